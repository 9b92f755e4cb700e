// Runtime core: device memory pool, stream, and the Cartesian grid with its
// helper operators, built on the device once per runtime.
//
// Grid numbering is OPM's UnstructuredGrid for Cartesian grids (used by the
// reference through Opm::GridManager, EquelleRuntimeCPU.cpp:20-49; 2D
// numbering pinned by backends/cuda/test/gridTest.cpp:104-144): I faces
// (i fastest, then j, then k), then J faces, then K faces; face_cells =
// (lower/left neighbour or -1, upper/right neighbour or -1).  Geometry is
// computed from node coordinates x_i = i*dx as the grid builder does, with
// explicitly rounded operations so no fused multiply-add changes a value.
// Helper operators follow Opm::HelperOps (restated in
// backends/cuda/src/deviceHelperOps.cpp:84-148): grad = -ngrad with ngrad
// rows (+1 first, -1 second) over interior faces, div = ngrad^T, fulldiv =
// fullngrad^T over all faces.
#include "eqg_internal.cuh"

#include <cub/cub.cuh>

#include <algorithm>
#include <cctype>
#include <cerrno>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <vector>

namespace eqg {

DevBuf::~DevBuf()
{
    if (ptr && core) core->free(ptr, bytes);
}

Core::Core()
{
    EQG_CUDA(cudaGetDevice(&device));
    EQG_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    EQG_CUDA(cudaDeviceGetDefaultMemPool(&pool, device));
    uint64_t threshold = UINT64_MAX;  // keep freed blocks cached in the pool
    EQG_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &threshold));
    EQG_CUDA(cudaMallocHost(&pinned, 64 * sizeof(double)));
    EQG_CUDA(cudaStreamCreateWithFlags(&copy_stream, cudaStreamNonBlocking));
}

// Drops the device buffers of output copies that were released (possibly
// by another thread); runs on the runtime's thread, the only one that may
// touch the allocator.
void Core::reap_outputs()
{
    std::vector<OutputCopy> done;
    {
        std::lock_guard<std::mutex> lock(output_mutex);
        done.swap(output_released);
    }
    done.clear();
}

Core::~Core()
{
    // Finish and drop outstanding output copies, then the pinned pool.
    {
        std::lock_guard<std::mutex> lock(output_mutex);
        for (auto& kv : output_copies) {
            cudaEventSynchronize(kv.second.done);
            cudaEventDestroy(kv.second.done);
            cudaFreeHost(kv.second.host);
        }
        output_copies.clear();
        for (auto& kv : pinned_pool) cudaFreeHost(kv.second);
        pinned_pool.clear();
    }
    reap_outputs();
    if (copy_stream) cudaStreamDestroy(copy_stream);
    // Release cached device objects before the stream goes away.
    for (auto& kv : derived_sets) eqg_set_release(kv.second);
    derived_sets.clear();
    fuse_state.reset();
    flush_buf.reset();
    pattern_cache.clear();
    opmat_cache.clear();
    identity_patterns.clear();
    ones_cache.clear();
    grad.reset();
    ngrad.reset();
    div_interior.reset();
    div_full.reset();
    face_cells.reset();
    face_normals.reset();
    face_areas.reset();
    face_centroids.reset();
    cell_volumes.reset();
    cell_centroids.reset();
    red_partials.reset();
    red_counter.reset();
    releasing = true;
    release_cached();
    for (auto& m : marks) cudaEventDestroy(m.ev);
    for (auto& pr : timer_pairs) {
        cudaEventDestroy(pr.a);
        cudaEventDestroy(pr.b);
    }
    residual_clock.clear();
    factor_clock.clear();
    krylov_clock.clear();
    if (stream) {
        cudaStreamSynchronize(stream);
        cudaStreamDestroy(stream);
    }
    if (pinned) cudaFreeHost(pinned);
    for (int k = 0; k < 2; ++k) {
        if (stage[k]) cudaFreeHost(stage[k]);
        if (stage_done[k]) cudaEventDestroy(stage_done[k]);
    }
}

// Size classes of the caching allocator: multiples of 256 B up to 64 KiB,
// then four classes per power of two (at most 25% slack).
size_t Core::size_class(size_t bytes)
{
    if (bytes <= 65536) return (bytes + 255) & ~(size_t)255;
    size_t p = 65536;
    while (p * 2 < bytes) p *= 2;
    const size_t step = p / 4;
    return ((bytes + step - 1) / step) * step;
}

// Every buffer of a runtime is used on its one stream only, so a freed
// block can serve the next request at once: work that still reads it was
// enqueued earlier on the same stream.  Blocks return to per-class free
// lists and go back to the pool only when the runtime ends (or when an
// allocation fails), so time steps allocate without driver calls.
Buf Core::alloc(size_t bytes)
{
    if (bytes == 0) bytes = 16;
    const size_t cls = size_class(bytes);
    void* p = nullptr;
    auto it = free_blocks.find(cls);
    if (it != free_blocks.end() && !it->second.empty()) {
        p = it->second.back();
        it->second.pop_back();
        cached_bytes -= (int64_t)cls;
    } else {
        cudaError_t e = cudaMallocAsync(&p, cls, stream);
        if (e == cudaErrorMemoryAllocation) {
            cudaGetLastError();
            release_cached();
            e = cudaMallocAsync(&p, cls, stream);
        }
        if (e != cudaSuccess) {
            cudaGetLastError();
            fail(e == cudaErrorMemoryAllocation ? EQG_ERR_MEMORY : EQG_ERR_DEVICE,
                 std::string("device allocation of ") + std::to_string(bytes) + " bytes failed: " +
                     cudaGetErrorString(e));
        }
    }
    bytes_in_use += (int64_t)cls;
    if (bytes_in_use > bytes_peak) bytes_peak = bytes_in_use;
    auto b = std::make_shared<DevBuf>();
    b->core = this;
    b->ptr = p;
    b->bytes = cls;
    return b;
}

void Core::free(void* p, size_t bytes)
{
    bytes_in_use -= (int64_t)bytes;
    if (releasing) {
        cudaFreeAsync(p, stream);
        return;
    }
    free_blocks[bytes].push_back(p);
    cached_bytes += (int64_t)bytes;
}

void Core::release_cached()
{
    for (auto& kv : free_blocks)
        for (void* q : kv.second) cudaFreeAsync(q, stream);
    free_blocks.clear();
    cached_bytes = 0;
}

void Core::sync() { EQG_CUDA(cudaStreamSynchronize(stream)); }

void Core::checkLaunch(const char* what)
{
    launches++;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) fail(EQG_ERR_DEVICE, std::string("kernel ") + what + " failed to launch: " + cudaGetErrorString(e));
}

double Core::param_d(const std::string& k, double d) const
{
    auto it = params.find(k);
    return it == params.end() ? d : std::stod(it->second);
}

int Core::param_i(const std::string& k, int d) const
{
    auto it = params.find(k);
    if (it == params.end()) return d;
    if (it->second == "true" || it->second == "yes") return 1;
    if (it->second == "false" || it->second == "no") return 0;
    return (int)std::stol(it->second);
}

std::string Core::param_s(const std::string& k, const std::string& d) const
{
    auto it = params.find(k);
    return it == params.end() ? d : it->second;
}

namespace {
constexpr size_t kStageBytes = 16u << 20;

void ensure_stage(Core& c)
{
    for (int k = 0; k < 2; ++k) {
        if (!c.stage[k]) EQG_CUDA(cudaMallocHost((void**)&c.stage[k], kStageBytes));
        if (!c.stage_done[k]) EQG_CUDA(cudaEventCreateWithFlags(&c.stage_done[k], cudaEventDisableTiming));
    }
}
}  // namespace

void Core::copy_to_device(void* dst, const void* src, size_t bytes)
{
    if (bytes < (1u << 20)) {  // small: one pageable copy
        if (bytes) EQG_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, stream));
        sync();
        return;
    }
    ensure_stage(*this);
    size_t off = 0;
    for (int k = 0; off < bytes; k ^= 1) {
        const size_t n = std::min(kStageBytes, bytes - off);
        EQG_CUDA(cudaEventSynchronize(stage_done[k]));  // its previous chunk has left the buffer
        std::memcpy(stage[k], (const char*)src + off, n);
        EQG_CUDA(cudaMemcpyAsync((char*)dst + off, stage[k], n, cudaMemcpyHostToDevice, stream));
        EQG_CUDA(cudaEventRecord(stage_done[k], stream));
        off += n;
    }
    sync();
}

void Core::copy_to_host(void* dst, const void* src, size_t bytes)
{
    if (bytes < (1u << 20)) {
        if (bytes) EQG_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, stream));
        sync();
        return;
    }
    ensure_stage(*this);
    const size_t chunks = (bytes + kStageBytes - 1) / kStageBytes;
    auto start = [&](size_t i) {
        const size_t off = i * kStageBytes, n = std::min(kStageBytes, bytes - off);
        EQG_CUDA(cudaMemcpyAsync(stage[i & 1], (const char*)src + off, n, cudaMemcpyDeviceToHost, stream));
        EQG_CUDA(cudaEventRecord(stage_done[i & 1], stream));
    };
    start(0);
    for (size_t i = 0; i < chunks; ++i) {
        if (i + 1 < chunks) start(i + 1);  // the next chunk's DMA while this one is copied out
        EQG_CUDA(cudaEventSynchronize(stage_done[i & 1]));
        const size_t off = i * kStageBytes, n = std::min(kStageBytes, bytes - off);
        std::memcpy((char*)dst + off, stage[i & 1], n);
    }
}

// ---------------------------------------------------------------------------
// Grid construction kernels.
// ---------------------------------------------------------------------------
namespace {

#define GRID_STRIDE(i, n) \
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < (n); i += (int64_t)gridDim.x * blockDim.x)

struct Dims {
    int dim, nx, ny, nz;
    double dx, dy, dz;
    int fx, fy, fz, nf, nc;
};

__device__ __forceinline__ double node(int i, double h) { return __dmul_rn((double)i, h); }
__device__ __forceinline__ double width(int i, double h) { return __dsub_rn(node(i + 1, h), node(i, h)); }
__device__ __forceinline__ double mid(int i, double h) { return __dmul_rn(0.5, __dadd_rn(node(i, h), node(i + 1, h))); }
__device__ __forceinline__ int cell_of(const Dims& d, int i, int j, int k) { return i + d.nx * (j + d.ny * k); }

__global__ void faces_kernel(Dims d, int32_t* face_cells, double* areas, double* centroids, uint8_t* interior)
{
    GRID_STRIDE(f, d.nf)
    {
        int axis, i, j, k;
        if (f < d.fx) {
            axis = 0;
            i = (int)(f % (d.nx + 1));
            const int r = (int)(f / (d.nx + 1));
            j = r % d.ny;
            k = r / d.ny;
        } else if (f < d.fx + d.fy) {
            axis = 1;
            const int g = (int)(f - d.fx);
            i = g % d.nx;
            const int r = g / d.nx;
            j = r % (d.ny + 1);
            k = r / (d.ny + 1);
        } else {
            axis = 2;
            const int h = (int)(f - d.fx - d.fy);
            i = h % d.nx;
            const int r = h / d.nx;
            j = r % d.ny;
            k = r / d.ny;
        }
        int c0, c1;
        double area, cx, cy, cz;
        if (axis == 0) {
            c0 = i > 0 ? cell_of(d, i - 1, j, k) : -1;
            c1 = i < d.nx ? cell_of(d, i, j, k) : -1;
            area = d.dim == 3 ? __dmul_rn(width(j, d.dy), width(k, d.dz)) : width(j, d.dy);
            cx = node(i, d.dx);
            cy = mid(j, d.dy);
            cz = mid(k, d.dz);
        } else if (axis == 1) {
            c0 = j > 0 ? cell_of(d, i, j - 1, k) : -1;
            c1 = j < d.ny ? cell_of(d, i, j, k) : -1;
            area = d.dim == 3 ? __dmul_rn(width(i, d.dx), width(k, d.dz)) : width(i, d.dx);
            cx = mid(i, d.dx);
            cy = node(j, d.dy);
            cz = mid(k, d.dz);
        } else {
            c0 = k > 0 ? cell_of(d, i, j, k - 1) : -1;
            c1 = k < d.nz ? cell_of(d, i, j, k) : -1;
            area = __dmul_rn(width(i, d.dx), width(j, d.dy));
            cx = mid(i, d.dx);
            cy = mid(j, d.dy);
            cz = node(k, d.dz);
        }
        face_cells[2 * f] = c0;
        face_cells[2 * f + 1] = c1;
        areas[f] = area;
        centroids[f] = cx;
        centroids[(int64_t)d.nf + f] = cy;
        if (d.dim == 3) centroids[2 * (int64_t)d.nf + f] = cz;
        interior[f] = (c0 >= 0 && c1 >= 0) ? 1 : 0;
    }
}

__global__ void cells_kernel(Dims d, double* volumes, double* centroids, uint8_t* boundary)
{
    GRID_STRIDE(c, d.nc)
    {
        const int i = (int)(c % d.nx);
        const int r = (int)(c / d.nx);
        const int j = r % d.ny;
        const int k = r / d.ny;
        double vol = __dmul_rn(width(i, d.dx), width(j, d.dy));
        if (d.dim == 3) vol = __dmul_rn(vol, width(k, d.dz));
        volumes[c] = vol;
        centroids[c] = mid(i, d.dx);
        centroids[(int64_t)d.nc + c] = mid(j, d.dy);
        if (d.dim == 3) centroids[2 * (int64_t)d.nc + c] = mid(k, d.dz);
        bool b = i == 0 || i == d.nx - 1 || j == 0 || j == d.ny - 1;
        if (d.dim == 3) b = b || k == 0 || k == d.nz - 1;
        boundary[c] = b ? 1 : 0;
    }
}

// The 2*dim faces of a cell in ascending face order, with the sign of the
// cell in fullngrad^T: +1 where the cell is the face's first cell.
__device__ __forceinline__ void cell_faces(const Dims& d, int64_t c, int32_t* faces, double* sign)
{
    const int i = (int)(c % d.nx);
    const int r = (int)(c / d.nx);
    const int j = r % d.ny;
    const int k = r / d.ny;
    faces[0] = i + (d.nx + 1) * (j + d.ny * k);
    faces[1] = faces[0] + 1;
    faces[2] = d.fx + i + d.nx * (j + (d.ny + 1) * k);
    faces[3] = faces[2] + d.nx;
    sign[0] = -1.0;
    sign[1] = 1.0;
    sign[2] = -1.0;
    sign[3] = 1.0;
    if (d.dim == 3) {
        faces[4] = d.fx + d.fy + i + d.nx * (j + d.ny * k);
        faces[5] = faces[4] + d.nx * d.ny;
        sign[4] = -1.0;
        sign[5] = 1.0;
    }
}

__global__ void div_full_kernel(Dims d, int32_t* ptr, int32_t* src, double* w)
{
    const int nfc = 2 * d.dim;
    GRID_STRIDE(c, d.nc)
    {
        int32_t faces[6];
        double sign[6];
        cell_faces(d, c, faces, sign);
        for (int t = 0; t < nfc; ++t) {
            src[c * nfc + t] = faces[t];
            w[c * nfc + t] = sign[t];
        }
        ptr[c] = (int32_t)(c * nfc);
        if (c == d.nc - 1) ptr[d.nc] = (int32_t)(d.nc * nfc);
    }
}

template <bool FILL>
__global__ void div_interior_kernel(Dims d, const int32_t* ipos, int64_t* cnt, const int32_t* ptr, int32_t* src,
                                    double* w)
{
    const int nfc = 2 * d.dim;
    GRID_STRIDE(c, d.nc)
    {
        int32_t faces[6];
        double sign[6];
        cell_faces(d, c, faces, sign);
        int o = FILL ? ptr[c] : 0;
        int64_t n = 0;
        for (int t = 0; t < nfc; ++t) {
            const int32_t p = ipos[faces[t]];
            if (p < 0) continue;
            if (FILL) {
                src[o] = p;
                w[o] = sign[t];
                ++o;
            } else {
                ++n;
            }
        }
        if (!FILL) cnt[c] = n;
    }
}

__global__ void grad_kernel(int nif, const int32_t* ifaces, const int32_t* face_cells, double s0, int32_t* ptr,
                            int32_t* src, double* w)
{
    GRID_STRIDE(i, nif)
    {
        const int32_t f = ifaces[i];
        int32_t c0 = face_cells[2 * f], c1 = face_cells[2 * f + 1];
        double w0 = s0, w1 = -s0;
        if (c1 < c0) {
            const int32_t t = c0;
            c0 = c1;
            c1 = t;
            const double u = w0;
            w0 = w1;
            w1 = u;
        }
        ptr[i] = (int32_t)(2 * i);
        src[2 * i] = c0;
        src[2 * i + 1] = c1;
        w[2 * i] = w0;
        w[2 * i + 1] = w1;
        if (i == nif - 1) ptr[nif] = 2 * nif;
    }
}

__global__ void iota_kernel(int32_t* out, int64_t n)
{
    GRID_STRIDE(i, n) out[i] = (int32_t)i;
}

__global__ void scatter_pos_kernel(const int32_t* list, int64_t n, int32_t* pos)
{
    GRID_STRIDE(i, n) pos[list[i]] = (int32_t)i;
}

__global__ void negate_u8_kernel(const uint8_t* a, uint8_t* out, int64_t n)
{
    GRID_STRIDE(i, n) out[i] = !a[i];
}

// ---------------------------------------------------------------------------
// Cartesian stencils: ngrad/grad over the interior faces and fulldiv/div
// over the cells, applied to values by face and cell index arithmetic
// instead of through their CSR operator matrices.  Interior faces come in
// ascending face order: x faces with 0 < i < nx (i fastest), then y faces
// with 0 < j < ny, then z faces with 0 < k < nz.  Each value is the CSR
// row's sum in its order (ascending column), with the weights +-1:
//   ngrad x (face) = x[first] - x[second], grad = -ngrad;
//   div f (cell)   = sum over the cell's faces in ascending face order of
//                    -f (the cell is the face's second cell) or +f (first).
// ---------------------------------------------------------------------------
struct InteriorCounts {
    int64_t x, y, z;
};

__host__ __device__ inline InteriorCounts interior_counts(const Dims& d)
{
    InteriorCounts n;
    n.x = (int64_t)(d.nx - 1) * d.ny * d.nz;
    n.y = (int64_t)d.nx * (d.ny - 1) * d.nz;
    n.z = d.dim == 3 ? (int64_t)d.nx * d.ny * (d.nz - 1) : 0;
    return n;
}

__global__ void stencil_grad_kernel(Dims d, InteriorCounts ni, int first_minus_second, const double* __restrict__ x,
                                    double* __restrict__ y, int64_t n)
{
    GRID_STRIDE(t, n)
    {
        int64_t c0, step;
        if (t < ni.x) {
            const int64_t i = t % (d.nx - 1) + 1, r = t / (d.nx - 1);
            c0 = (i - 1) + (int64_t)d.nx * r;
            step = 1;
        } else if (t < ni.x + ni.y) {
            const int64_t u = t - ni.x, i = u % d.nx, r = u / d.nx;
            const int64_t j = r % (d.ny - 1) + 1, k = r / (d.ny - 1);
            c0 = i + (int64_t)d.nx * ((j - 1) + (int64_t)d.ny * k);
            step = d.nx;
        } else {
            const int64_t u = t - ni.x - ni.y, i = u % d.nx, r = u / d.nx;
            const int64_t j = r % d.ny, k = r / d.ny + 1;
            c0 = i + (int64_t)d.nx * (j + (int64_t)d.ny * (k - 1));
            step = (int64_t)d.nx * d.ny;
        }
        const double a = x[c0], b = x[c0 + step];
        y[t] = first_minus_second ? a - b : b - a;
    }
}

template <bool INTERIOR>
__global__ void stencil_div_kernel(Dims d, InteriorCounts ni, const double* __restrict__ f, double* __restrict__ y)
{
    GRID_STRIDE(c, d.nc)
    {
        const int64_t i = c % d.nx, r = c / d.nx, j = r % d.ny, k = r / d.ny;
        double acc = 0.0;
        if (!INTERIOR) {
            const int64_t xl = i + (int64_t)(d.nx + 1) * (j + (int64_t)d.ny * k);
            const int64_t yl = d.fx + i + (int64_t)d.nx * (j + (int64_t)(d.ny + 1) * k);
            acc = acc - f[xl];
            acc = acc + f[xl + 1];
            acc = acc - f[yl];
            acc = acc + f[yl + d.nx];
            if (d.dim == 3) {
                const int64_t zl = (int64_t)d.fx + d.fy + i + (int64_t)d.nx * (j + (int64_t)d.ny * k);
                acc = acc - f[zl];
                acc = acc + f[zl + (int64_t)d.nx * d.ny];
            }
        } else {
            // interior position of the x face at i (0 < i < nx), of the y face
            // at j (0 < j < ny), of the z face at k (0 < k < nz)
            const int64_t xr = (int64_t)(d.nx - 1) * (j + (int64_t)d.ny * k);
            if (i > 0) acc = acc - f[(i - 1) + xr];
            if (i < d.nx - 1) acc = acc + f[i + xr];
            const int64_t yr = ni.x + i + (int64_t)d.nx * ((int64_t)(d.ny - 1) * k);
            if (j > 0) acc = acc - f[yr + (int64_t)d.nx * (j - 1)];
            if (j < d.ny - 1) acc = acc + f[yr + (int64_t)d.nx * j];
            if (d.dim == 3) {
                const int64_t zr = ni.x + ni.y + i + (int64_t)d.nx * j;
                const int64_t plane = (int64_t)d.nx * d.ny;
                if (k > 0) acc = acc - f[zr + plane * (k - 1)];
                if (k < d.nz - 1) acc = acc + f[zr + plane * k];
            }
        }
        y[c] = acc;
    }
}

}  // namespace

// Indices i in [0, n) with flags[i] != 0, ascending.
Buf compact_indices(Core& c, const uint8_t* flags, int64_t n, int64_t& count)
{
    Buf out = c.allocN<int32_t>(n > 0 ? n : 1);
    Buf num = c.allocN<int64_t>(1);
    cub::CountingInputIterator<int32_t> it(0);
    size_t tmp_bytes = 0;
    EQG_CUDA(cub::DeviceSelect::Flagged(nullptr, tmp_bytes, it, flags, out->as<int32_t>(), num->as<int64_t>(), n,
                                        c.stream));
    Buf tmp = c.alloc(tmp_bytes);
    EQG_CUDA(cub::DeviceSelect::Flagged(tmp->ptr, tmp_bytes, it, flags, out->as<int32_t>(), num->as<int64_t>(), n,
                                        c.stream));
    c.launches++;
    EQG_CUDA(cudaMemcpyAsync(c.pinned, num->ptr, sizeof(int64_t), cudaMemcpyDeviceToHost, c.stream));
    c.sync();
    std::memcpy(&count, c.pinned, sizeof(int64_t));
    return out;
}

namespace {

// The six built-in index sets from the face-interior and cell-boundary
// flags; returns the interior faces (ascending) and their count.
Buf make_index_sets(Core& c, const Buf& face_interior, const Buf& cell_boundary, eqg_set** builtin, int64_t& n_if)
{
    const int64_t nc64 = c.nc, nf64 = c.nf;
    // index sets
    auto make = [&](int entity, Buf idx, int64_t n, bool identity) {
        auto* s = new eqg_set;
        s->entity = entity;
        s->n = n;
        s->idx = idx;
        s->identity = identity;
        s->sorted = 1;
        return s;
    };
    Buf all_c = c.allocN<int32_t>(nc64), all_f = c.allocN<int32_t>(nf64);
    launch(c, "iota", [&] { iota_kernel<<<blocksFor(nc64), kThreads, 0, c.stream>>>(all_c->as<int32_t>(), nc64); });
    launch(c, "iota", [&] { iota_kernel<<<blocksFor(nf64), kThreads, 0, c.stream>>>(all_f->as<int32_t>(), nf64); });
    int64_t n_bc = 0, n_ic = 0, n_bf = 0;
    n_if = 0;
    Buf bc = compact_indices(c, cell_boundary->as<uint8_t>(), nc64, n_bc);
    Buf not_b = c.allocN<uint8_t>(nc64 > nf64 ? nc64 : nf64);
    launch(c, "negate", [&] { negate_u8_kernel<<<blocksFor(nc64), kThreads, 0, c.stream>>>(cell_boundary->as<uint8_t>(), not_b->as<uint8_t>(),
                                                                 nc64); });
    Buf ic = compact_indices(c, not_b->as<uint8_t>(), nc64, n_ic);
    Buf iff = compact_indices(c, face_interior->as<uint8_t>(), nf64, n_if);
    launch(c, "negate", [&] { negate_u8_kernel<<<blocksFor(nf64), kThreads, 0, c.stream>>>(face_interior->as<uint8_t>(), not_b->as<uint8_t>(),
                                                                 nf64); });
    Buf bf = compact_indices(c, not_b->as<uint8_t>(), nf64, n_bf);
    c.nif = (int)n_if;
    builtin[EQG_ALL_CELLS] = make(EQG_CELLS, all_c, nc64, true);
    builtin[EQG_BOUNDARY_CELLS] = make(EQG_CELLS, bc, n_bc, false);
    builtin[EQG_INTERIOR_CELLS] = make(EQG_CELLS, ic, n_ic, false);
    builtin[EQG_ALL_FACES] = make(EQG_FACES, all_f, nf64, true);
    builtin[EQG_BOUNDARY_FACES] = make(EQG_FACES, bf, n_bf, false);
    builtin[EQG_INTERIOR_FACES] = make(EQG_FACES, iff, n_if, false);

    return iff;
}

OpMatrixP new_opmatrix(Core& c, int n_out, int n_src, int max_row, int64_t nnz)
{
    auto m = std::make_shared<OpMatrix>();
    m->id = c.newId();
    m->n_out = n_out;
    m->n_src = n_src;
    m->max_row = max_row;
    m->nnz = nnz;
    m->ptr = c.allocN<int32_t>((size_t)n_out + 1);
    m->src = c.allocN<int32_t>(nnz > 0 ? nnz : 1);
    m->w = c.allocN<double>(nnz > 0 ? nnz : 1);
    return m;
}

// grad = -ngrad and ngrad over the interior faces, from face_cells.
void make_grad_ops(Core& c, const Buf& iff, int64_t n_if)
{
    c.grad = new_opmatrix(c, c.nif, c.nc, 2, 2 * n_if);
    c.ngrad = new_opmatrix(c, c.nif, c.nc, 2, 2 * n_if);
    if (c.nif > 0) {
        launch(c, "grad_op", [&] { grad_kernel<<<blocksFor(n_if), kThreads, 0, c.stream>>>(c.nif, iff->as<int32_t>(), c.face_cells->as<int32_t>(),
                                                                -1.0, c.grad->ptr->as<int32_t>(),
                                                                c.grad->src->as<int32_t>(), c.grad->w->as<double>()); });
        launch(c, "ngrad_op", [&] { grad_kernel<<<blocksFor(n_if), kThreads, 0, c.stream>>>(c.nif, iff->as<int32_t>(), c.face_cells->as<int32_t>(),
                                                                1.0, c.ngrad->ptr->as<int32_t>(),
                                                                c.ngrad->src->as<int32_t>(), c.ngrad->w->as<double>()); });
    } else {
        k_fill_i32(c, c.grad->ptr->as<int32_t>(), 0, 1);
        k_fill_i32(c, c.ngrad->ptr->as<int32_t>(), 0, 1);
    }
}

}  // namespace

void build_grid(Core& c, eqg_set** builtin)
{
    if (c.dim != 2 && c.dim != 3) fail(EQG_ERR_ARG, "Cannot handle " + std::to_string(c.dim) + " dimensions.");
    if (c.nx < 1 || c.ny < 1 || c.nz < 1) fail(EQG_ERR_ARG, "grid dimensions must be positive");
    if (c.dim == 2) {
        c.nz = 1;
        c.dz = 1.0;
    }
    Dims d;
    d.dim = c.dim;
    d.nx = c.nx;
    d.ny = c.ny;
    d.nz = c.nz;
    d.dx = c.dx;
    d.dy = c.dy;
    d.dz = c.dz;
    const int64_t fx = (int64_t)(c.nx + 1) * c.ny * c.nz;
    const int64_t fy = (int64_t)c.nx * (c.ny + 1) * c.nz;
    const int64_t fz = c.dim == 3 ? (int64_t)c.nx * c.ny * (c.nz + 1) : 0;
    const int64_t nc64 = (int64_t)c.nx * c.ny * c.nz;
    const int64_t nf64 = fx + fy + fz;
    if (nf64 * 2 > (int64_t)INT32_MAX || nc64 * 6 > (int64_t)INT32_MAX)
        fail(EQG_ERR_UNSUPPORTED, "grid too large for 32-bit indices");
    d.fx = (int)fx;
    d.fy = (int)fy;
    d.fz = (int)fz;
    d.nf = (int)nf64;
    d.nc = (int)nc64;
    c.nc = d.nc;
    c.nf = d.nf;

    c.face_cells = c.allocN<int32_t>(2 * nf64);
    c.face_areas = c.allocN<double>(nf64);
    c.face_centroids = c.allocN<double>(c.dim * nf64);
    Buf face_interior = c.allocN<uint8_t>(nf64);
    launch(c, "grid_faces", [&] { faces_kernel<<<blocksFor(nf64), kThreads, 0, c.stream>>>(d, c.face_cells->as<int32_t>(), c.face_areas->as<double>(),
                                                             c.face_centroids->as<double>(),
                                                             face_interior->as<uint8_t>()); });
    c.cell_volumes = c.allocN<double>(nc64);
    c.cell_centroids = c.allocN<double>(c.dim * nc64);
    Buf cell_boundary = c.allocN<uint8_t>(nc64);
    launch(c, "grid_cells", [&] { cells_kernel<<<blocksFor(nc64), kThreads, 0, c.stream>>>(d, c.cell_volumes->as<double>(),
                                                             c.cell_centroids->as<double>(),
                                                             cell_boundary->as<uint8_t>()); });

    int64_t n_if = 0;
    Buf iff = make_index_sets(c, face_interior, cell_boundary, builtin, n_if);
    make_grad_ops(c, iff, n_if);
    c.div_full = new_opmatrix(c, c.nc, c.nf, 2 * c.dim, (int64_t)2 * c.dim * nc64);
    launch(c, "div_full_op", [&] { div_full_kernel<<<blocksFor(nc64), kThreads, 0, c.stream>>>(d, c.div_full->ptr->as<int32_t>(),
                                                                c.div_full->src->as<int32_t>(),
                                                                c.div_full->w->as<double>()); });

    Buf ipos = c.allocN<int32_t>(nf64);
    k_fill_i32(c, ipos->as<int32_t>(), -1, nf64);
    if (n_if > 0) {
        launch(c, "interior_pos", [&] { scatter_pos_kernel<<<blocksFor(n_if), kThreads, 0, c.stream>>>(iff->as<int32_t>(), n_if, ipos->as<int32_t>()); });
    }
    {
        auto m = std::make_shared<OpMatrix>();
        m->id = c.newId();
        m->n_out = c.nc;
        m->n_src = c.nif;
        m->max_row = 2 * c.dim;
        Buf cnt = c.allocN<int64_t>(nc64);
        launch(c, "div_interior_count", [&] { div_interior_kernel<false><<<blocksFor(nc64), kThreads, 0, c.stream>>>(d, ipos->as<int32_t>(),
                                                                               cnt->as<int64_t>(), nullptr, nullptr,
                                                                               nullptr); });
        const int64_t nnz = counts_to_rowptr(c, cnt, c.nc, m->ptr);
        m->nnz = nnz;
        m->src = c.allocN<int32_t>(nnz > 0 ? nnz : 1);
        m->w = c.allocN<double>(nnz > 0 ? nnz : 1);
        launch(c, "div_interior_fill", [&] { div_interior_kernel<true><<<blocksFor(nc64), kThreads, 0, c.stream>>>(d, ipos->as<int32_t>(), nullptr,
                                                                              m->ptr->as<int32_t>(),
                                                                              m->src->as<int32_t>(),
                                                                              m->w->as<double>()); });
        c.div_interior = m;
    }
    c.grad->stencil = STENCIL_GRAD;
    c.ngrad->stencil = STENCIL_NGRAD;
    c.div_full->stencil = STENCIL_DIV_FULL;
    c.div_interior->stencil = STENCIL_DIV_INTERIOR;
    c.sync();
}

namespace {

Dims core_dims(const Core& c)
{
    Dims d;
    d.dim = c.dim;
    d.nx = c.nx;
    d.ny = c.ny;
    d.nz = c.nz;
    d.dx = c.dx;
    d.dy = c.dy;
    d.dz = c.dz;
    d.fx = (c.nx + 1) * c.ny * c.nz;
    d.fy = c.nx * (c.ny + 1) * c.nz;
    d.fz = c.dim == 3 ? c.nx * c.ny * (c.nz + 1) : 0;
    d.nf = c.nf;
    d.nc = c.nc;
    return d;
}

}  // namespace

bool stencil_apply_values(Core& c, int kind, const double* x, double* y)
{
    if (!c.cartesian) return false;
    const Dims d = core_dims(c);
    const InteriorCounts ni = interior_counts(d);
    switch (kind) {
    case STENCIL_GRAD:
    case STENCIL_NGRAD:
        if (c.nif <= 0) return true;
        // the interior face values written, two cell values read per face
        launch(c, "stencil_grad", [&] {
            stencil_grad_kernel<<<blocksFor(c.nif), kThreads, 0, c.stream>>>(d, ni, kind == STENCIL_NGRAD ? 1 : 0, x,
                                                                           y, c.nif);
        }, 8.0 * c.nif + 8.0 * c.nc);
        return true;
    case STENCIL_DIV_FULL:
        launch(c, "stencil_div", [&] {
            stencil_div_kernel<false><<<blocksFor(c.nc), kThreads, 0, c.stream>>>(d, ni, x, y);
        }, 8.0 * c.nf + 8.0 * c.nc);
        return true;
    case STENCIL_DIV_INTERIOR:
        launch(c, "stencil_div", [&] {
            stencil_div_kernel<true><<<blocksFor(c.nc), kThreads, 0, c.stream>>>(d, ni, x, y);
        }, 8.0 * c.nif + 8.0 * c.nc);
        return true;
    default:
        return false;
    }
}

// ---------------------------------------------------------------------------
// Grids read from a file (parameter grid_filename; the reference builds
// Opm::GridManager(grid_filename), EquelleRuntimeCPU.cpp:20-24).
//
// The file holds the arrays of an UnstructuredGrid that the runtime uses, as
// whitespace-separated text, each array after its keyword:
//
//   eqg-grid 1
//   dimensions <2|3>  cells <nc>  faces <nf>
//   face_cells      2 nf integers: first and second cell of each face (-1: outside)
//   cell_facepos    nc + 1 integers: cell c's faces are cell_faces[facepos[c] .. facepos[c+1])
//   cell_faces      facepos[nc] integers
//   face_areas      nf reals
//   face_centroids  dim nf reals, face by face (x y [z] of face 0, then face 1, ...)
//   face_normals    dim nf reals, face by face, scaled by the face area, from the
//                   first cell toward the second
//   cell_volumes    nc reals
//   cell_centroids  dim nc reals, cell by cell
//
// equelle_b200/grids.py writes it.  Every face must have at least one cell
// and two different cells when it has two, and each cell's face list must
// hold exactly the faces that name the cell.
// ---------------------------------------------------------------------------
namespace {

struct FileGrid {
    int dim = 0;
    int64_t nc = 0, nf = 0;
    std::vector<int32_t> face_cells, cell_facepos, cell_faces;
    std::vector<double> face_areas, face_centroids, face_normals, cell_volumes, cell_centroids;
};

class GridTokens {
public:
    GridTokens(const std::string& path) : path_(path)
    {
        std::ifstream f(path.c_str(), std::ios::binary);
        if (!f) fail(EQG_ERR_ARG, "Failed to read grid from file " + path);
        std::ostringstream ss;
        ss << f.rdbuf();
        text_ = ss.str();
        p_ = text_.c_str();
    }
    std::string word()
    {
        skip();
        const char* b = p_;
        while (*p_ && !std::isspace((unsigned char)*p_)) ++p_;
        return std::string(b, p_);
    }
    void expect(const char* key)
    {
        const std::string w = word();
        if (w != key) fail(EQG_ERR_ARG, "grid file " + path_ + ": expected '" + key + "', found '" + w + "'");
    }
    long long integer()
    {
        skip();
        char* e = nullptr;
        errno = 0;
        const long long v = std::strtoll(p_, &e, 10);
        if (e == p_ || errno) fail(EQG_ERR_ARG, "grid file " + path_ + ": expected an integer");
        p_ = e;
        return v;
    }
    double real()
    {
        skip();
        char* e = nullptr;
        const double v = std::strtod(p_, &e);
        if (e == p_) fail(EQG_ERR_ARG, "grid file " + path_ + ": expected a number");
        p_ = e;
        return v;
    }
    template <class T>
    void ints(const char* key, int64_t n, std::vector<T>& out)
    {
        expect(key);
        out.resize(n);
        for (int64_t i = 0; i < n; ++i) out[i] = (T)integer();
    }
    void reals(const char* key, int64_t n, std::vector<double>& out)
    {
        expect(key);
        out.resize(n);
        for (int64_t i = 0; i < n; ++i) out[i] = real();
    }

private:
    void skip()
    {
        while (*p_ && std::isspace((unsigned char)*p_)) ++p_;
    }
    std::string path_, text_;
    const char* p_ = nullptr;
};

FileGrid read_grid_file(const std::string& path)
{
    GridTokens t(path);
    FileGrid g;
    t.expect("eqg-grid");
    if (t.integer() != 1) fail(EQG_ERR_ARG, "grid file " + path + ": unknown format version");
    t.expect("dimensions");
    g.dim = (int)t.integer();
    t.expect("cells");
    g.nc = t.integer();
    t.expect("faces");
    g.nf = t.integer();
    if (g.dim != 2 && g.dim != 3) fail(EQG_ERR_ARG, "Cannot handle " + std::to_string(g.dim) + " dimensions.");
    if (g.nc < 1 || g.nf < 1 || 2 * g.nf > (int64_t)INT32_MAX || g.nc > (int64_t)INT32_MAX)
        fail(EQG_ERR_ARG, "grid file " + path + ": cell or face count out of range");
    t.ints("face_cells", 2 * g.nf, g.face_cells);
    t.ints("cell_facepos", g.nc + 1, g.cell_facepos);
    if (g.cell_facepos[0] != 0) fail(EQG_ERR_ARG, "grid file " + path + ": cell_facepos must start at 0");
    for (int64_t c = 0; c < g.nc; ++c)
        if (g.cell_facepos[c + 1] < g.cell_facepos[c])
            fail(EQG_ERR_ARG, "grid file " + path + ": cell_facepos must not decrease");
    t.ints("cell_faces", g.cell_facepos[g.nc], g.cell_faces);
    t.reals("face_areas", g.nf, g.face_areas);
    t.reals("face_centroids", g.dim * g.nf, g.face_centroids);
    t.reals("face_normals", g.dim * g.nf, g.face_normals);
    t.reals("cell_volumes", g.nc, g.cell_volumes);
    t.reals("cell_centroids", g.dim * g.nc, g.cell_centroids);
    // topology checks: faces name valid, distinct cells; each cell's list
    // holds exactly the faces naming it
    std::vector<int64_t> named(g.nc, 0);
    for (int64_t f = 0; f < g.nf; ++f) {
        const int32_t a = g.face_cells[2 * f], b = g.face_cells[2 * f + 1];
        if (a < -1 || a >= g.nc || b < -1 || b >= g.nc || (a < 0 && b < 0) || a == b)
            fail(EQG_ERR_ARG, "grid file " + path + ": face " + std::to_string(f) + " has invalid cells");
        if (a >= 0) named[a]++;
        if (b >= 0) named[b]++;
    }
    for (int64_t c = 0; c < g.nc; ++c) {
        if (g.cell_facepos[c + 1] - g.cell_facepos[c] != named[c])
            fail(EQG_ERR_ARG, "grid file " + path + ": face list of cell " + std::to_string(c) +
                                 " does not match face_cells");
        for (int32_t k = g.cell_facepos[c]; k < g.cell_facepos[c + 1]; ++k) {
            const int32_t f = g.cell_faces[k];
            if (f < 0 || f >= g.nf || (g.face_cells[2 * (int64_t)f] != c && g.face_cells[2 * (int64_t)f + 1] != c))
                fail(EQG_ERR_ARG, "grid file " + path + ": face list of cell " + std::to_string(c) +
                                     " does not match face_cells");
        }
    }
    return g;
}

// face by face (f dim + d) -> component-major (d n + f)
std::vector<double> component_major(const std::vector<double>& v, int dim, int64_t n)
{
    std::vector<double> out(v.size());
    for (int64_t i = 0; i < n; ++i)
        for (int d = 0; d < dim; ++d) out[(size_t)d * n + i] = v[(size_t)i * dim + d];
    return out;
}

template <class T>
Buf upload(Core& c, const std::vector<T>& v)
{
    Buf b = c.allocN<T>(v.empty() ? 1 : v.size());
    if (!v.empty()) EQG_CUDA(cudaMemcpyAsync(b->ptr, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, c.stream));
    return b;
}

}  // namespace

void build_grid_from_file(Core& c, const std::string& path, eqg_set** builtin)
{
    const FileGrid g = read_grid_file(path);
    c.cartesian = false;
    c.dim = g.dim;
    c.nx = c.ny = c.nz = 0;
    c.dx = c.dy = c.dz = 0.0;
    c.nc = (int)g.nc;
    c.nf = (int)g.nf;
    c.face_cells = upload(c, g.face_cells);
    c.face_areas = upload(c, g.face_areas);
    c.face_centroids = upload(c, component_major(g.face_centroids, g.dim, g.nf));
    c.face_normals = upload(c, component_major(g.face_normals, g.dim, g.nf));
    c.cell_volumes = upload(c, g.cell_volumes);
    c.cell_centroids = upload(c, component_major(g.cell_centroids, g.dim, g.nc));
    // interior faces: two cells; boundary cells: a face with an outside side
    // (EquelleRuntimeCPU::boundaryCell, EquelleRuntimeCPU.cpp:94-104)
    std::vector<uint8_t> interior(g.nf), boundary(g.nc, 0);
    for (int64_t f = 0; f < g.nf; ++f) {
        const int32_t a = g.face_cells[2 * f], b = g.face_cells[2 * f + 1];
        interior[f] = (a >= 0 && b >= 0) ? 1 : 0;
        if (!interior[f]) boundary[a >= 0 ? a : b] = 1;
    }
    Buf face_interior = upload(c, interior), cell_boundary = upload(c, boundary);
    int64_t n_if = 0;
    Buf iff = make_index_sets(c, face_interior, cell_boundary, builtin, n_if);
    make_grad_ops(c, iff, n_if);
    // fulldiv = fullngrad^T and div = ngrad^T: row c holds the faces of cell
    // c in ascending order, +1 where c is the face's first cell, -1 where it
    // is the second (the transpose of a face-by-face matrix has its columns
    // in ascending order)
    std::vector<int32_t> ipos(g.nf, -1);
    {
        int32_t k = 0;
        for (int64_t f = 0; f < g.nf; ++f)
            if (interior[f]) ipos[f] = k++;
    }
    std::vector<int32_t> fptr(g.nc + 1, 0), fsrc, iptr(g.nc + 1, 0), isrc;
    std::vector<double> fw, iw;
    int max_row = 0;
    for (int64_t cc = 0; cc < g.nc; ++cc) {
        std::vector<int32_t> faces(g.cell_faces.begin() + g.cell_facepos[cc],
                                   g.cell_faces.begin() + g.cell_facepos[cc + 1]);
        std::sort(faces.begin(), faces.end());
        max_row = std::max(max_row, (int)faces.size());
        for (int32_t f : faces) {
            const double sign = g.face_cells[2 * (int64_t)f] == cc ? 1.0 : -1.0;
            fsrc.push_back(f);
            fw.push_back(sign);
            if (ipos[f] >= 0) {
                isrc.push_back(ipos[f]);
                iw.push_back(sign);
            }
        }
        fptr[cc + 1] = (int32_t)fsrc.size();
        iptr[cc + 1] = (int32_t)isrc.size();
    }
    c.div_full = opmat_from_host(c, c.nc, c.nf, fptr, fsrc, fw);
    c.div_interior = opmat_from_host(c, c.nc, c.nif, iptr, isrc, iw);
    c.sync();
}

}  // namespace eqg

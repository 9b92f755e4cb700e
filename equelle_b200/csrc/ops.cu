// Value kernels: elementwise arithmetic, comparisons, selections, gathers,
// index location and reductions.  Each is a grid-stride loop over dense
// arrays (coalesced, bandwidth bound; no shared-memory staging is needed
// for a single pass over contiguous data).
#include "eqg_internal.cuh"

#include <cfloat>
#include <climits>

namespace eqg {

namespace {

#define GRID_STRIDE(i, n) \
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < (n); i += (int64_t)gridDim.x * blockDim.x)

__global__ void fill_kernel(double* out, double v, int64_t n)
{
    GRID_STRIDE(i, n) out[i] = v;
}

__global__ void fill_i32_kernel(int32_t* out, int32_t v, int64_t n)
{
    GRID_STRIDE(i, n) out[i] = v;
}

__device__ __forceinline__ double apply_op(int op, double a, double b)
{
    switch (op) {
    case EW_ADD: return a + b;
    case EW_SUB: return a - b;
    case EW_MUL: return a * b;
    default: return a / b;
    }
}

template <int OP>
__global__ void binary_kernel(const double* __restrict__ a, const double* __restrict__ b, double* __restrict__ out,
                              int64_t n)
{
    GRID_STRIDE(i, n) out[i] = apply_op(OP, a[i], b[i]);
}

__global__ void binary_scalar_kernel(int op, const double* __restrict__ a, double s, int scalar_left,
                                     double* __restrict__ out, int64_t n)
{
    GRID_STRIDE(i, n) out[i] = scalar_left ? apply_op(op, s, a[i]) : apply_op(op, a[i], s);
}

__global__ void unary_kernel(int op, const double* __restrict__ a, double* __restrict__ out, int64_t n)
{
    GRID_STRIDE(i, n)
    {
        const double x = a[i];
        double r;
        if (op == EQG_NEG) r = 0.0 - x;          // V::Zero(n) - x
        else if (op == EQG_SQRT) r = sqrt(x);
        else r = (x >= 0.0 ? 1.0 : -1.0) * x;    // factors * x
        out[i] = r;
    }
}

__device__ __forceinline__ uint8_t cmp(int op, double a, double b)
{
    switch (op) {
    case EQG_LT: return a < b;
    case EQG_LE: return a <= b;
    case EQG_GT: return a > b;
    case EQG_GE: return a >= b;
    case EQG_EQ: return a == b;
    default: return a != b;
    }
}

__global__ void compare_kernel(int op, const double* a, const double* b, uint8_t* out, int64_t n)
{
    GRID_STRIDE(i, n) out[i] = cmp(op, a[i], b[i]);
}

__global__ void compare_scalar_kernel(int op, const double* a, double s, int scalar_left, uint8_t* out, int64_t n)
{
    GRID_STRIDE(i, n) out[i] = scalar_left ? cmp(op, s, a[i]) : cmp(op, a[i], s);
}

// iftrue * trueones + iffalse * falseones (EquelleRuntimeCPU_impl.hpp:170-178)
__global__ void select_kernel(const uint8_t* m, const double* a, const double* b, double* out, int64_t n)
{
    GRID_STRIDE(i, n)
    {
        const double t = m[i] ? 1.0 : 0.0;
        const double f = m[i] ? 0.0 : 1.0;
        out[i] = a[i] * t + b[i] * f;
    }
}

__global__ void mask_logic_kernel(int op, const uint8_t* a, const uint8_t* b, uint8_t* out, int64_t n)
{
    GRID_STRIDE(i, n)
    {
        if (op == EQG_AND) out[i] = a[i] && b[i];
        else if (op == EQG_OR) out[i] = a[i] || b[i];
        else out[i] = !a[i];
    }
}

__global__ void set_select_kernel(const uint8_t* m, const int32_t* a, const int32_t* b, int32_t* out, int64_t n)
{
    GRID_STRIDE(i, n) out[i] = m[i] ? a[i] : b[i];
}

__global__ void is_empty_kernel(const int32_t* s, uint8_t* out, int64_t n)
{
    GRID_STRIDE(i, n) out[i] = s[i] < 0;
}

__global__ void face_neighbour_kernel(const int32_t* face_cells, const int32_t* faces, int side, int32_t* out,
                                      int64_t n, int nf, int32_t* err)
{
    GRID_STRIDE(i, n)
    {
        const int32_t f = faces[i];
        if (f < 0 || f >= nf) {
            *err = 1;
            out[i] = -1;
        } else {
            out[i] = face_cells[2 * (int64_t)f + side];
        }
    }
}

__global__ void gather_i32_kernel(const int32_t* data, const int32_t* map, int32_t* out, int64_t n, int32_t fill)
{
    GRID_STRIDE(i, n)
    {
        const int32_t m = map[i];
        out[i] = m >= 0 ? data[m] : fill;
    }
}

__global__ void gather_f64_kernel(const double* data, const int32_t* idx, int stride, int comp, double* out,
                                  int64_t n, int32_t* err)
{
    GRID_STRIDE(i, n)
    {
        const int32_t e = idx[i];
        if (e < 0) {
            *err = 1;
            out[i] = 0.0;
        } else {
            out[i] = data[(int64_t)comp * stride + e];
        }
    }
}

// Unit normal component: n[comp] / sqrt(sum_d n[d]^2) of the area-scaled
// normal (EquelleRuntimeCPU.cpp:306-308).  Cartesian faces have one nonzero
// component equal to the face area.
__global__ void normal_kernel(const int32_t* faces, const double* areas, double* out, int comp, int dim, int nf,
                              int fx, int fy, int64_t n, int32_t* err)
{
    GRID_STRIDE(i, n)
    {
        const int32_t f = faces[i];
        if (f < 0 || f >= nf) {
            *err = 1;
            out[i] = 0.0;
            continue;
        }
        const int axis = f < fx ? 0 : (f < fx + fy ? 1 : 2);
        const double a = areas[f];
        double nn = 0.0;
        for (int d = 0; d < dim; ++d) {
            const double v = d == axis ? a : 0.0;
            nn += v * v;
        }
        out[i] = (comp == axis ? a : 0.0) / sqrt(nn);
    }
}

// Unit normal component of grids read from a file: the area-scaled normal
// over its Euclidean norm (EquelleRuntimeCPU::normal,
// EquelleRuntimeCPU.cpp:295-314), the squares summed in component order.
__global__ void normal_file_kernel(const int32_t* faces, const double* normals, double* out, int comp, int dim,
                                   int nf, int64_t n, int32_t* err)
{
    GRID_STRIDE(i, n)
    {
        const int32_t f = faces[i];
        if (f < 0 || f >= nf) {
            *err = 1;
            out[i] = 0.0;
            continue;
        }
        // separately rounded products and sums (no fused multiply-add), as
        // the reference's Eigen row norm computes them
        double nn = 0.0;
        for (int d = 0; d < dim; ++d) {
            const double v = normals[(int64_t)d * nf + f];
            nn = __dadd_rn(nn, __dmul_rn(v, v));
        }
        out[i] = normals[(int64_t)comp * nf + f] / sqrt(nn);
    }
}

// Position of each key in a strictly ascending array (binary search), or in
// the identity enumeration 0..identity_n-1 when sorted == nullptr.
__global__ void locate_kernel(const int32_t* sorted, int64_t n_sorted, const int32_t* keys, int32_t* pos,
                              int64_t n_keys, int identity_n, int32_t* err)
{
    GRID_STRIDE(i, n_keys)
    {
        const int32_t k = keys[i];
        int32_t p = -1;
        if (!sorted) {
            if (k >= 0 && k < identity_n) p = k;
        } else {
            int64_t lo = 0, hi = n_sorted;
            while (lo < hi) {
                const int64_t mid = (lo + hi) >> 1;
                if (sorted[mid] < k) lo = mid + 1;
                else hi = mid;
            }
            if (lo < n_sorted && sorted[lo] == k) p = (int32_t)lo;
        }
        if (p < 0) *err = 1;
        pos[i] = p;
    }
}

__global__ void scatter_inverse_kernel(const int32_t* pos, int64_t n, int32_t* inv, int32_t* err)
{
    GRID_STRIDE(i, n)
    {
        const int32_t p = pos[i];
        if (p >= 0) {
            const int32_t old = atomicExch(&inv[p], (int32_t)i);
            if (old >= 0) *err = 2;  // two source rows land on one target row
        }
    }
}

__global__ void strictly_sorted_kernel(const int32_t* a, int64_t n, int32_t* flag)
{
    GRID_STRIDE(i, n - 1)
    {
        if (!(a[i] < a[i + 1])) *flag = 0;
    }
}

// ---- deterministic reductions: fixed grid, block partials, one final block.
template <int OP>
__device__ __forceinline__ double red_identity()
{
    return OP == EQG_MIN ? DBL_MAX : (OP == EQG_MAX ? -DBL_MAX : (OP == EQG_SUM ? 0.0 : 1.0));
}

template <int OP>
__device__ __forceinline__ double red_combine(double a, double b)
{
    return OP == EQG_MIN ? fmin(a, b) : (OP == EQG_MAX ? fmax(a, b) : (OP == EQG_SUM ? a + b : a * b));
}

template <int OP, bool SQUARE>
__global__ void reduce_partials_kernel(const double* a, int64_t n, double* partials)
{
    __shared__ double sh[kThreads];
    double acc = red_identity<OP>();
    GRID_STRIDE(i, n)
    {
        const double x = a[i];
        acc = red_combine<OP>(acc, SQUARE ? x * x : x);
    }
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) sh[threadIdx.x] = red_combine<OP>(sh[threadIdx.x], sh[threadIdx.x + s]);
        __syncthreads();
    }
    if (threadIdx.x == 0) partials[blockIdx.x] = sh[0];
}

template <int OP, bool SQRT>
__global__ void reduce_final_kernel(const double* partials, int nparts, double* out)
{
    __shared__ double sh[kThreads];
    double acc = red_identity<OP>();
    for (int i = threadIdx.x; i < nparts; i += blockDim.x) acc = red_combine<OP>(acc, partials[i]);
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) sh[threadIdx.x] = red_combine<OP>(sh[threadIdx.x], sh[threadIdx.x + s]);
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = SQRT ? sqrt(sh[0]) : sh[0];
}

template <int OP, bool SQUARE>
double run_reduce(Core& c, const double* a, int64_t n)
{
    double* partials = c.red_partials->as<double>();
    const int nb = blocksFor(n, kThreads, kRedBlocks);
    launch(c, "reduce_partials", [&] { reduce_partials_kernel<OP, SQUARE><<<nb, kThreads, 0, c.stream>>>(a, n, partials); }, 8.0 * n);
    launch(c, "reduce_final", [&] { reduce_final_kernel<OP, SQUARE><<<1, kThreads, 0, c.stream>>>(partials, nb, partials + kRedBlocks); });
    EQG_CUDA(cudaMemcpyAsync(c.pinned, partials + kRedBlocks, sizeof(double), cudaMemcpyDeviceToHost, c.stream));
    c.sync();
    return c.pinned[0];
}

}  // namespace

void k_fill(Core& c, double* out, double v, int64_t n)
{
    if (n <= 0) return;
    launch(c, "fill", [&] { fill_kernel<<<blocksFor(n), kThreads, 0, c.stream>>>(out, v, n); }, 8.0 * n);
}

void k_fill_i32(Core& c, int32_t* out, int32_t v, int64_t n)
{
    if (n <= 0) return;
    launch(c, "fill_i32", [&] { fill_i32_kernel<<<blocksFor(n), kThreads, 0, c.stream>>>(out, v, n); });
}

void k_binary(Core& c, int op, const double* a, const double* b, double* out, int64_t n)
{
    if (n <= 0) return;
    const int nb = blocksFor(n);
    switch (op) {
    case EW_ADD: launch(c, "binary", [&] { binary_kernel<EW_ADD><<<nb, kThreads, 0, c.stream>>>(a, b, out, n); }, 24.0 * n); break;
    case EW_SUB: launch(c, "binary", [&] { binary_kernel<EW_SUB><<<nb, kThreads, 0, c.stream>>>(a, b, out, n); }, 24.0 * n); break;
    case EW_MUL: launch(c, "binary", [&] { binary_kernel<EW_MUL><<<nb, kThreads, 0, c.stream>>>(a, b, out, n); }, 24.0 * n); break;
    case EW_DIV: launch(c, "binary", [&] { binary_kernel<EW_DIV><<<nb, kThreads, 0, c.stream>>>(a, b, out, n); }, 24.0 * n); break;
    default: fail(EQG_ERR_ARG, "unknown binary operator");
    }
}

void k_binary_scalar(Core& c, int op, const double* a, double s, int scalar_left, double* out, int64_t n)
{
    if (n <= 0) return;
    launch(c, "binary_scalar", [&] { binary_scalar_kernel<<<blocksFor(n), kThreads, 0, c.stream>>>(op, a, s, scalar_left, out, n); }, 16.0 * n);
}

void k_unary_value(Core& c, int op, const double* a, double* out, int64_t n)
{
    if (n <= 0) return;
    launch(c, "unary", [&] { unary_kernel<<<blocksFor(n), kThreads, 0, c.stream>>>(op, a, out, n); }, 16.0 * n);
}

void k_compare(Core& c, int op, const double* a, const double* b, uint8_t* out, int64_t n)
{
    if (n <= 0) return;
    launch(c, "compare", [&] { compare_kernel<<<blocksFor(n), kThreads, 0, c.stream>>>(op, a, b, out, n); }, 17.0 * n);
}

void k_compare_scalar(Core& c, int op, const double* a, double s, int scalar_left, uint8_t* out, int64_t n)
{
    if (n <= 0) return;
    launch(c, "compare_scalar", [&] { compare_scalar_kernel<<<blocksFor(n), kThreads, 0, c.stream>>>(op, a, s, scalar_left, out, n); }, 9.0 * n);
}

void k_select_value(Core& c, const uint8_t* m, const double* a, const double* b, double* out, int64_t n)
{
    if (n <= 0) return;
    launch(c, "select", [&] { select_kernel<<<blocksFor(n), kThreads, 0, c.stream>>>(m, a, b, out, n); }, 25.0 * n);
}

void k_mask_logic(Core& c, int op, const uint8_t* a, const uint8_t* b, uint8_t* out, int64_t n)
{
    if (n <= 0) return;
    launch(c, "mask_logic", [&] { mask_logic_kernel<<<blocksFor(n), kThreads, 0, c.stream>>>(op, a, b, out, n); }, 3.0 * n);
}

void k_set_select(Core& c, const uint8_t* m, const int32_t* a, const int32_t* b, int32_t* out, int64_t n)
{
    if (n <= 0) return;
    launch(c, "set_select", [&] { set_select_kernel<<<blocksFor(n), kThreads, 0, c.stream>>>(m, a, b, out, n); });
}

void k_is_empty(Core& c, const int32_t* s, uint8_t* out, int64_t n)
{
    if (n <= 0) return;
    launch(c, "is_empty", [&] { is_empty_kernel<<<blocksFor(n), kThreads, 0, c.stream>>>(s, out, n); });
}

void k_face_neighbour(Core& c, const int32_t* faces, int side, int32_t* out, int64_t n, int32_t* err)
{
    if (n <= 0) return;
    launch(c, "face_neighbour", [&] { face_neighbour_kernel<<<blocksFor(n), kThreads, 0, c.stream>>>(c.face_cells->as<int32_t>(), faces, side, out, n,
                                                                   c.nf, err); });
}

void k_gather_i32(Core& c, const int32_t* data, const int32_t* map, int32_t* out, int64_t n, int32_t fill)
{
    if (n <= 0) return;
    launch(c, "gather_i32", [&] { gather_i32_kernel<<<blocksFor(n), kThreads, 0, c.stream>>>(data, map, out, n, fill); });
}

void k_gather_f64(Core& c, const double* data, const int32_t* idx, int stride, int comp, double* out, int64_t n,
                  int32_t* err)
{
    if (n <= 0) return;
    launch(c, "gather_f64", [&] { gather_f64_kernel<<<blocksFor(n), kThreads, 0, c.stream>>>(data, idx, stride, comp, out, n, err); }, 20.0 * n);
}

void k_normal(Core& c, const int32_t* faces, double* out, int comp, int64_t n, int32_t* err)
{
    if (n <= 0) return;
    if (!c.cartesian) {
        launch(c, "normal", [&] {
            normal_file_kernel<<<blocksFor(n), kThreads, 0, c.stream>>>(faces, c.face_normals->as<double>(), out, comp,
                                                                       c.dim, c.nf, n, err);
        });
        return;
    }
    const int fx = (c.nx + 1) * c.ny * c.nz;
    const int fy = c.nx * (c.ny + 1) * c.nz;
    launch(c, "normal", [&] { normal_kernel<<<blocksFor(n), kThreads, 0, c.stream>>>(faces, c.face_areas->as<double>(), out, comp, c.dim, c.nf,
                                                           fx, fy, n, err); });
}

void k_locate(Core& c, const int32_t* sorted, int64_t n_sorted, const int32_t* keys, int32_t* pos, int64_t n_keys,
              int identity_n, int32_t* err)
{
    if (n_keys <= 0) return;
    launch(c, "locate", [&] { locate_kernel<<<blocksFor(n_keys), kThreads, 0, c.stream>>>(sorted, n_sorted, keys, pos, n_keys, identity_n, err); });
}

void k_scatter_inverse(Core& c, const int32_t* pos, int64_t n, int32_t* inv, int32_t* err)
{
    if (n <= 0) return;
    launch(c, "scatter_inverse", [&] { scatter_inverse_kernel<<<blocksFor(n), kThreads, 0, c.stream>>>(pos, n, inv, err); });
}

void k_is_strictly_sorted(Core& c, const int32_t* a, int64_t n, int32_t* flag)
{
    if (n <= 1) return;
    launch(c, "strictly_sorted", [&] { strictly_sorted_kernel<<<blocksFor(n), kThreads, 0, c.stream>>>(a, n, flag); });
}

double k_reduce(Core& c, int op, const double* a, int64_t n)
{
    switch (op) {
    case EQG_MIN: return run_reduce<EQG_MIN, false>(c, a, n);
    case EQG_MAX: return run_reduce<EQG_MAX, false>(c, a, n);
    case EQG_SUM: return run_reduce<EQG_SUM, false>(c, a, n);
    case EQG_PROD: return run_reduce<EQG_PROD, false>(c, a, n);
    }
    fail(EQG_ERR_ARG, "unknown reduction");
}

double k_two_norm(Core& c, const double* a, int64_t n)
{
    double* partials = c.red_partials->as<double>();
    const int nb = blocksFor(n, kThreads, kRedBlocks);
    launch(c, "norm_partials", [&] { reduce_partials_kernel<EQG_SUM, true><<<nb, kThreads, 0, c.stream>>>(a, n, partials); }, 8.0 * n);
    launch(c, "norm_final", [&] { reduce_final_kernel<EQG_SUM, true><<<1, kThreads, 0, c.stream>>>(partials, nb, partials + kRedBlocks); });
    EQG_CUDA(cudaMemcpyAsync(c.pinned, partials + kRedBlocks, sizeof(double), cudaMemcpyDeviceToHost, c.stream));
    c.sync();
    return c.pinned[0];
}

}  // namespace eqg

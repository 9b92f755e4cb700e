// Linear solve J du = F for the Newton update (the reference calls
// Opm::LinearSolverFactory::solve from solveForUpdate,
// EquelleRuntimeCPU.cpp:413-440).
//
// Method: BiCGStab (van der Vorst 1992) right-preconditioned with ILU(0)
// (Saad, Iterative Methods for Sparse Linear Systems, Alg. 10.4), from x = 0,
// converged when ||b - A x|| <= tol * ||b||, with a fixed pseudo-random
// shadow residual (shadow_entry).
//
// Parallel ILU(0): rows are reordered symmetrically so that each "stage" is a
// contiguous block of rows with no couplings inside it; factorization and
// both triangular solves then run one kernel per stage, a thread per row.
//   - ordering "natural": stages are the wavefront levels of the natural
//     order (symmetrised pattern), which reproduces natural-order ILU(0)
//     exactly (the oracle's preconditioner), at the price of many stages;
//   - ordering "multicolor" (default): greedy colouring of the symmetrised
//     pattern; a 7-point stencil gives 2 colours per unknown block, so a
//     handful of stages of ~n/colors rows each.
// The analysis (ordering, permuted pattern, value map) is computed on the
// host once per Jacobian pattern and cached with it.
//
// Precision "mixed": the inner BiCGStab and the ILU(0) factors run in FP32,
// inside FP64 iterative refinement (r = b - A x in FP64 with FP64 A).
//
// Every kernel of an iteration reads a device-side status word first and
// returns at once after convergence or breakdown, so the host enqueues
// several iterations between convergence checks without a round trip.
#include "eqg_internal.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>

namespace eqg {

namespace {

#define GRID_STRIDE(i, n) \
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < (n); i += (int64_t)gridDim.x * blockDim.x)

struct KScal {
    double rho, rho_new, alpha, omega;
    double thr;      // tol^2 * ||b||^2
    double rv, ss, ts, tt, rr, rhat_r;
    int status;      // 0 running, 1 converged, 2 breakdown
    int s_conv;      // converged on the half step
    int iterations;
    int pad;
};

enum { ST_RUN = 0, ST_CONV = 1, ST_BREAK = 2 };

__device__ __forceinline__ bool stopped(const KScal* sc) { return sc->status != ST_RUN; }

// Block-wide sum of NV values; returns sums to thread 0.
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV])
{
    __shared__ double sh[NV][kThreads / 32];
#pragma unroll
    for (int k = 0; k < NV; ++k) {
        double x = v[k];
        for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
        if ((threadIdx.x & 31) == 0) sh[k][threadIdx.x >> 5] = x;
    }
    __syncthreads();
    if (threadIdx.x < 32) {
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            double x = threadIdx.x < (kThreads / 32) ? sh[k][threadIdx.x] : 0.0;
            for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
            v[k] = x;
        }
    }
}

// Writes block partials; returns true in exactly one thread of the last
// block to finish, after which `partials` holds all blocks' sums.
template <int NV>
__device__ __forceinline__ bool publish_partials(double (&v)[NV], double* partials, unsigned int* counter)
{
    block_sum<NV>(v);
    __shared__ bool last;
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) partials[blockIdx.x * NV + k] = v[k];
        __threadfence();
        const unsigned int done = atomicAdd(counter, 1u);
        last = (done == gridDim.x - 1);
    }
    __syncthreads();
    return last && threadIdx.x == 0;
}

template <int NV>
__device__ __forceinline__ void final_sums(const double* partials, int nblocks, double (&out)[NV],
                                           unsigned int* counter)
{
    __threadfence();
#pragma unroll
    for (int k = 0; k < NV; ++k) out[k] = 0.0;
    for (int b = 0; b < nblocks; ++b)
#pragma unroll
        for (int k = 0; k < NV; ++k) out[k] += ((volatile double*)partials)[b * NV + k];
    *counter = 0u;
}

// ---- matrix kernels ---------------------------------------------------------
template <class T>
__device__ __forceinline__ double row_dot(int r, const int* __restrict__ rowptr, const int* __restrict__ col,
                                          const T* __restrict__ a, const T* __restrict__ x)
{
    double acc = 0.0;
    const int e1 = rowptr[r + 1];
    for (int e = rowptr[r]; e < e1; ++e) acc += (double)a[e] * (double)x[col[e]];
    return acc;
}

__global__ void gather_values_kernel(const double* __restrict__ src, const int* __restrict__ vmap,
                                     double* __restrict__ dst, int64_t nnz)
{
    GRID_STRIDE(e, nnz) dst[e] = src[vmap[e]];
}

__global__ void to_float_kernel(const double* __restrict__ a, float* __restrict__ b, int64_t n)
{
    GRID_STRIDE(i, n) b[i] = (float)a[i];
}

__global__ void permute_kernel(const double* __restrict__ src, const int* __restrict__ perm, double* __restrict__ dst,
                               int n)
{
    GRID_STRIDE(i, n) dst[i] = src[perm[i]];
}

__global__ void unpermute_kernel(const double* __restrict__ src, const int* __restrict__ perm,
                                 double* __restrict__ dst, int n)
{
    GRID_STRIDE(i, n) dst[perm[i]] = src[i];
}

// ILU(0) of the rows [r0, r1) of one stage (their L parts reference only
// finished rows of earlier stages).
__global__ void ilu0_factor_stage_kernel(int r0, int r1, const int* __restrict__ rowptr, const int* __restrict__ col,
                                         const int* __restrict__ diag, double* lu, int* status)
{
    for (int64_t rr = r0 + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; rr < r1;
         rr += (int64_t)gridDim.x * blockDim.x) {
        const int r = (int)rr;
        const int dpos = diag[r];
        const int end = rowptr[r + 1];
        for (int e = rowptr[r]; e < dpos; ++e) {
            const int k = col[e];
            const double piv = lu[diag[k]];
            if (piv == 0.0) {
                *status = 1;
                return;
            }
            const double lik = lu[e] / piv;
            lu[e] = lik;
            int p = e + 1;
            const int q1 = rowptr[k + 1];
            for (int q = diag[k] + 1; q < q1; ++q) {
                const int cq = col[q];
                while (p < end && col[p] < cq) ++p;
                if (p < end && col[p] == cq) lu[p] -= lik * lu[q];
            }
        }
        if (lu[dpos] == 0.0) *status = 1;
    }
}

template <class T>
__global__ void ilu0_lower_stage_kernel(int r0, int r1, const int* __restrict__ rowptr, const int* __restrict__ col,
                                        const int* __restrict__ diag, const T* __restrict__ lu,
                                        const T* __restrict__ b, T* __restrict__ y, const KScal* sc, int skip_if_s)
{
    if (stopped(sc) || (skip_if_s && sc->s_conv)) return;
    for (int64_t rr = r0 + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; rr < r1;
         rr += (int64_t)gridDim.x * blockDim.x) {
        const int r = (int)rr;
        double s = (double)b[r];
        const int dpos = diag[r];
        for (int e = rowptr[r]; e < dpos; ++e) s -= (double)lu[e] * (double)y[col[e]];
        y[r] = (T)s;
    }
}

template <class T>
__global__ void ilu0_upper_stage_kernel(int r0, int r1, const int* __restrict__ rowptr, const int* __restrict__ col,
                                        const int* __restrict__ diag, const T* __restrict__ lu, T* __restrict__ x,
                                        const KScal* sc, int skip_if_s)
{
    if (stopped(sc) || (skip_if_s && sc->s_conv)) return;
    for (int64_t rr = r0 + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; rr < r1;
         rr += (int64_t)gridDim.x * blockDim.x) {
        const int r = (int)rr;
        const int dpos = diag[r];
        double s = (double)x[r];
        const int e1 = rowptr[r + 1];
        for (int e = dpos + 1; e < e1; ++e) s -= (double)lu[e] * (double)x[col[e]];
        x[r] = (T)(s / (double)lu[dpos]);
    }
}

// ---- BiCGStab steps -----------------------------------------------------------
// Shadow residual: a fixed, dense pseudo-random vector in [-1, 1) from a
// 32-bit hash of the row index (the textbook rhat = r0 breaks down when r0
// is nearly a unit vector, as at the first Newton iteration of well-driven
// flow).  The CPU oracle uses the same entries.
__device__ __forceinline__ double shadow_entry(int64_t i)
{
    uint32_t x = (uint32_t)((uint64_t)i * 0x9E3779B1ull);
    x ^= x >> 16;
    x *= 0x85EBCA6Bu;
    x ^= x >> 13;
    return 2.0 * ((double)x / 4294967296.0) - 1.0;
}

template <class T>
__global__ void bicg_init_kernel(const T* __restrict__ b, T* r, T* rhat, T* p, T* v, T* x, int n, double* partials,
                                 unsigned int* counter, KScal* sc, double tol2)
{
    double d[2] = {0.0, 0.0};
    GRID_STRIDE(i, n)
    {
        const T bi = b[i];
        const T hi = (T)shadow_entry(i);
        r[i] = bi;
        rhat[i] = hi;
        p[i] = (T)0;
        v[i] = (T)0;
        x[i] = (T)0;
        d[0] += (double)bi * (double)bi;
        d[1] += (double)hi * (double)bi;
    }
    if (publish_partials<2>(d, partials, counter)) {
        double s[2];
        final_sums<2>(partials, gridDim.x, s, counter);
        sc->rho = 1.0;
        sc->alpha = 1.0;
        sc->omega = 1.0;
        sc->rho_new = s[1];
        sc->rr = s[0];
        sc->thr = tol2 * s[0];
        sc->s_conv = 0;
        sc->iterations = 0;
        sc->status = s[0] == 0.0 ? ST_CONV : ST_RUN;
    }
}

template <class T>
__global__ void bicg_p_kernel(const T* __restrict__ r, const T* __restrict__ v, T* __restrict__ p, int n,
                              const KScal* sc)
{
    if (stopped(sc)) return;
    const double beta = (sc->rho_new / sc->rho) * (sc->alpha / sc->omega);
    const double omega = sc->omega;
    GRID_STRIDE(i, n) p[i] = (T)((double)r[i] + beta * ((double)p[i] - omega * (double)v[i]));
}

// v = A ph ; alpha = rho_new / (rhat . v)
template <class T>
__global__ void bicg_spmv_alpha_kernel(const int* __restrict__ rowptr, const int* __restrict__ col,
                                       const T* __restrict__ a, const T* __restrict__ ph, const T* __restrict__ rhat,
                                       T* __restrict__ v, int n, double* partials, unsigned int* counter, KScal* sc)
{
    if (stopped(sc)) return;
    double d[1] = {0.0};
    GRID_STRIDE(i, n)
    {
        const double vi = row_dot<T>((int)i, rowptr, col, a, ph);
        v[i] = (T)vi;
        d[0] += (double)rhat[i] * (double)(T)vi;
    }
    if (publish_partials<1>(d, partials, counter)) {
        double s[1];
        final_sums<1>(partials, gridDim.x, s, counter);
        sc->rv = s[0];
        if (s[0] == 0.0 || !isfinite(s[0])) sc->status = ST_BREAK;
        else sc->alpha = sc->rho_new / s[0];
    }
}

// s = r - alpha v ; ss = s . s
template <class T>
__global__ void bicg_s_kernel(const T* __restrict__ r, const T* __restrict__ v, T* __restrict__ s, int n,
                              double* partials, unsigned int* counter, KScal* sc)
{
    if (stopped(sc)) return;
    const double alpha = sc->alpha;
    double d[1] = {0.0};
    GRID_STRIDE(i, n)
    {
        const T si = (T)((double)r[i] - alpha * (double)v[i]);
        s[i] = si;
        d[0] += (double)si * (double)si;
    }
    if (publish_partials<1>(d, partials, counter)) {
        double t[1];
        final_sums<1>(partials, gridDim.x, t, counter);
        sc->ss = t[0];
        sc->s_conv = t[0] <= sc->thr ? 1 : 0;
    }
}

// t = A sh ; omega = (t . s) / (t . t)
template <class T>
__global__ void bicg_spmv_omega_kernel(const int* __restrict__ rowptr, const int* __restrict__ col,
                                       const T* __restrict__ a, const T* __restrict__ sh, const T* __restrict__ s,
                                       T* __restrict__ t, int n, double* partials, unsigned int* counter, KScal* sc)
{
    if (stopped(sc) || sc->s_conv) return;
    double d[2] = {0.0, 0.0};
    GRID_STRIDE(i, n)
    {
        const T ti = (T)row_dot<T>((int)i, rowptr, col, a, sh);
        t[i] = ti;
        d[0] += (double)ti * (double)s[i];
        d[1] += (double)ti * (double)ti;
    }
    if (publish_partials<2>(d, partials, counter)) {
        double u[2];
        final_sums<2>(partials, gridDim.x, u, counter);
        sc->ts = u[0];
        sc->tt = u[1];
        if (u[1] == 0.0 || !isfinite(u[1])) sc->status = ST_BREAK;
        else sc->omega = u[0] / u[1];
    }
}

// x += alpha ph + omega sh ; r = s - omega t ; rr = r.r ; rho_new = rhat.r
template <class T>
__global__ void bicg_xr_kernel(const T* __restrict__ ph, const T* __restrict__ sh, const T* __restrict__ s,
                               const T* __restrict__ t, const T* __restrict__ rhat, T* __restrict__ x,
                               T* __restrict__ r, int n, double* partials, unsigned int* counter, KScal* sc)
{
    if (stopped(sc)) return;
    const double alpha = sc->alpha;
    const int half = sc->s_conv;
    const double omega = half ? 0.0 : sc->omega;
    double d[2] = {0.0, 0.0};
    GRID_STRIDE(i, n)
    {
        if (half) {
            x[i] = (T)((double)x[i] + alpha * (double)ph[i]);
        } else {
            x[i] = (T)((double)x[i] + alpha * (double)ph[i] + omega * (double)sh[i]);
            const T ri = (T)((double)s[i] - omega * (double)t[i]);
            r[i] = ri;
            d[0] += (double)ri * (double)ri;
            d[1] += (double)rhat[i] * (double)ri;
        }
    }
    if (publish_partials<2>(d, partials, counter)) {
        double u[2];
        final_sums<2>(partials, gridDim.x, u, counter);
        sc->iterations += 1;
        if (half) {
            sc->rr = sc->ss;
            sc->status = ST_CONV;
            return;
        }
        sc->rr = u[0];
        sc->rhat_r = u[1];
        sc->rho = sc->rho_new;
        sc->rho_new = u[1];
        if (u[0] <= sc->thr) sc->status = ST_CONV;
        else if (u[1] == 0.0 || sc->omega == 0.0 || !isfinite(u[0])) sc->status = ST_BREAK;
    }
}

// Refinement: r = b - A x (FP64) with rr = r.r ; also r32 = float(r).
__global__ void residual_kernel(const int* __restrict__ rowptr, const int* __restrict__ col,
                                const double* __restrict__ a, const double* __restrict__ x,
                                const double* __restrict__ b, double* __restrict__ r, float* __restrict__ r32, int n,
                                double* partials, unsigned int* counter, double* out_rr)
{
    double d[1] = {0.0};
    GRID_STRIDE(i, n)
    {
        const double ri = b[i] - row_dot<double>((int)i, rowptr, col, a, x);
        r[i] = ri;
        r32[i] = (float)ri;
        d[0] += ri * ri;
    }
    if (publish_partials<1>(d, partials, counter)) {
        double u[1];
        final_sums<1>(partials, gridDim.x, u, counter);
        *out_rr = u[0];
    }
}

__global__ void add_float_kernel(double* __restrict__ x, const float* __restrict__ d, int n)
{
    GRID_STRIDE(i, n) x[i] += (double)d[i];
}

__global__ void sumsq_kernel(const double* __restrict__ a, int n, double* partials, unsigned int* counter,
                             double* out)
{
    double d[1] = {0.0};
    GRID_STRIDE(i, n) d[0] += a[i] * a[i];
    if (publish_partials<1>(d, partials, counter)) {
        double u[1];
        final_sums<1>(partials, gridDim.x, u, counter);
        *out = u[0];
    }
}

}  // namespace

// ---------------------------------------------------------------------------
// Host analysis, cached per Jacobian pattern.
// ---------------------------------------------------------------------------
struct SolverAnalysis {
    int n = 0;
    int64_t nnz = 0;
    bool natural = false;
    bool ok = true;                 // every row has a diagonal entry
    std::vector<int> stage_ptr;     // stage boundaries in the new order
    Buf perm, rowptr, col, vmap, diag;
    // workspaces
    Buf a64, lu64, a32, lu32;
    Buf vec64;   // 10 double vectors
    Buf vec32;   // 9 float vectors
    Buf scal;    // KScal
    Buf partials, counter, factor_status;
};

namespace {

std::shared_ptr<SolverAnalysis> analyse(Core& c, const Pattern& p, bool natural)
{
    auto an = std::make_shared<SolverAnalysis>();
    const int n = p.rows;
    an->n = n;
    an->nnz = p.nnz;
    an->natural = natural;
    std::vector<int> rp(n + 1), ci(p.nnz > 0 ? p.nnz : 1);
    EQG_CUDA(cudaMemcpyAsync(rp.data(), p.rowptr->ptr, (size_t)(n + 1) * 4, cudaMemcpyDeviceToHost, c.stream));
    if (p.nnz > 0)
        EQG_CUDA(cudaMemcpyAsync(ci.data(), p.colind->ptr, (size_t)p.nnz * 4, cudaMemcpyDeviceToHost, c.stream));
    c.sync();
    // symmetrised adjacency (without the diagonal)
    std::vector<int> tp(n + 1, 0);
    for (int64_t e = 0; e < p.nnz; ++e) tp[ci[e] + 1]++;
    for (int i = 0; i < n; ++i) tp[i + 1] += tp[i];
    std::vector<int> tr(p.nnz > 0 ? p.nnz : 1);
    {
        std::vector<int> pos(tp.begin(), tp.end() - 1);
        for (int i = 0; i < n; ++i)
            for (int e = rp[i]; e < rp[i + 1]; ++e) tr[pos[ci[e]]++] = i;
    }
    for (int i = 0; i < n; ++i) {
        bool has = false;
        for (int e = rp[i]; e < rp[i + 1]; ++e) has |= (ci[e] == i);
        if (!has) an->ok = false;
    }
    std::vector<int> key(n, 0);
    if (natural) {
        // wavefront level over the earlier neighbours
        for (int i = 0; i < n; ++i) {
            int lv = 0;
            for (int e = rp[i]; e < rp[i + 1]; ++e)
                if (ci[e] < i) lv = std::max(lv, key[ci[e]] + 1);
            for (int e = tp[i]; e < tp[i + 1]; ++e)
                if (tr[e] < i) lv = std::max(lv, key[tr[e]] + 1);
            key[i] = lv;
        }
    } else {
        // greedy colouring in natural order
        std::vector<int> mark(64, -1);
        for (int i = 0; i < n; ++i) {
            auto see = [&](int j) {
                if (j < i) {
                    const int cj = key[j];
                    if (cj >= (int)mark.size()) mark.resize(cj + 1, -1);
                    mark[cj] = i;
                }
            };
            for (int e = rp[i]; e < rp[i + 1]; ++e) see(ci[e]);
            for (int e = tp[i]; e < tp[i + 1]; ++e) see(tr[e]);
            int col = 0;
            while (col < (int)mark.size() && mark[col] == i) ++col;
            key[i] = col;
        }
    }
    const int nstages = n > 0 ? *std::max_element(key.begin(), key.end()) + 1 : 0;
    an->stage_ptr.assign(nstages + 1, 0);
    for (int i = 0; i < n; ++i) an->stage_ptr[key[i] + 1]++;
    for (int s = 0; s < nstages; ++s) an->stage_ptr[s + 1] += an->stage_ptr[s];
    std::vector<int> perm(n), iperm(n);
    {
        std::vector<int> pos(an->stage_ptr.begin(), an->stage_ptr.end() - 1);
        for (int i = 0; i < n; ++i) perm[pos[key[i]]++] = i;  // stable within a stage
    }
    for (int r = 0; r < n; ++r) iperm[perm[r]] = r;
    // permuted pattern with ascending new columns
    std::vector<int> nrp(n + 1, 0), ncol(p.nnz > 0 ? p.nnz : 1), vmap(p.nnz > 0 ? p.nnz : 1), diag(n, -1);
    std::vector<std::pair<int, int>> row;
    for (int r = 0; r < n; ++r) {
        const int i = perm[r];
        row.clear();
        for (int e = rp[i]; e < rp[i + 1]; ++e) row.emplace_back(iperm[ci[e]], e);
        std::sort(row.begin(), row.end());
        nrp[r + 1] = nrp[r] + (int)row.size();
        int o = nrp[r];
        for (auto& ce : row) {
            if (ce.first == r) diag[r] = o;
            ncol[o] = ce.first;
            vmap[o] = ce.second;
            ++o;
        }
    }
    auto up = [&](const std::vector<int>& v) {
        Buf b = c.allocN<int>(v.size());
        EQG_CUDA(cudaMemcpyAsync(b->ptr, v.data(), v.size() * 4, cudaMemcpyHostToDevice, c.stream));
        return b;
    };
    an->perm = up(perm);
    an->rowptr = up(nrp);
    an->col = up(ncol);
    an->vmap = up(vmap);
    std::vector<int> diag_safe(diag);
    for (auto& d : diag_safe)
        if (d < 0) d = 0;
    an->diag = up(diag_safe);
    const size_t nz = (size_t)(p.nnz > 0 ? p.nnz : 1);
    an->a64 = c.allocN<double>(nz);
    an->lu64 = c.allocN<double>(nz);
    an->vec64 = c.allocN<double>((size_t)10 * (n > 0 ? n : 1));
    an->scal = c.alloc(sizeof(KScal));
    an->partials = c.allocN<double>((size_t)kRedBlocks * 2);
    an->counter = c.allocN<unsigned int>(1);
    an->factor_status = c.allocN<int>(1);
    EQG_CUDA(cudaMemsetAsync(an->counter->ptr, 0, sizeof(unsigned int), c.stream));
    c.sync();
    return an;
}

template <class T>
struct Vecs {
    T *x, *r, *rhat, *p, *v, *s, *t, *ph, *sh, *b;
};

template <class T>
Vecs<T> vecs(T* base, int n)
{
    Vecs<T> v;
    T* q[10];
    for (int k = 0; k < 10; ++k) q[k] = base + (size_t)k * (n > 0 ? n : 1);
    v.x = q[0];
    v.r = q[1];
    v.rhat = q[2];
    v.p = q[3];
    v.v = q[4];
    v.s = q[5];
    v.t = q[6];
    v.ph = q[7];
    v.sh = q[8];
    v.b = q[9];
    return v;
}

template <class T>
void precondition(Core& c, const SolverAnalysis& an, const T* lu, const T* in, T* out, const KScal* sc, int skip_if_s)
{
    const int ns = (int)an.stage_ptr.size() - 1;
    for (int s = 0; s < ns; ++s) {
        const int r0 = an.stage_ptr[s], r1 = an.stage_ptr[s + 1];
        launch(c, "ilu0_lower", [&] { ilu0_lower_stage_kernel<T><<<blocksFor(r1 - r0), kThreads, 0, c.stream>>>(
            r0, r1, an.rowptr->as<int>(), an.col->as<int>(), an.diag->as<int>(), lu, in, out, sc, skip_if_s); });
    }
    for (int s = ns - 1; s >= 0; --s) {
        const int r0 = an.stage_ptr[s], r1 = an.stage_ptr[s + 1];
        launch(c, "ilu0_upper", [&] { ilu0_upper_stage_kernel<T><<<blocksFor(r1 - r0), kThreads, 0, c.stream>>>(
            r0, r1, an.rowptr->as<int>(), an.col->as<int>(), an.diag->as<int>(), lu, out, sc, skip_if_s); });
    }
}

// BiCGStab on the permuted system with values a and factors lu; v.b holds the
// right-hand side.  Returns (converged, iterations, rr/bb).
template <class T>
SolveResult bicgstab(Core& c, SolverAnalysis& an, const T* a, const T* lu, Vecs<T> v, double tol, int max_iter,
                     int check_every)
{
    const int n = an.n;
    KScal* sc = an.scal->as<KScal>();
    double* part = an.partials->as<double>();
    unsigned int* cnt = an.counter->as<unsigned int>();
    const int nb = blocksFor(n, kThreads, kRedBlocks);
    launch(c, "bicg_init", [&] { bicg_init_kernel<T><<<nb, kThreads, 0, c.stream>>>(v.b, v.r, v.rhat, v.p, v.v, v.x, n, part, cnt, sc, tol * tol); });
    SolveResult res;
    KScal h{};
    double bb = 0.0;
    int enq = 0;
    for (;;) {
        const int chunk = std::min(check_every, max_iter - enq);
        for (int k = 0; k < chunk; ++k) {
            launch(c, "bicg_p", [&] { bicg_p_kernel<T><<<blocksFor(n), kThreads, 0, c.stream>>>(v.r, v.v, v.p, n, sc); });
            precondition<T>(c, an, lu, v.p, v.ph, sc, 0);
            launch(c, "bicg_spmv_alpha", [&] { bicg_spmv_alpha_kernel<T><<<nb, kThreads, 0, c.stream>>>(an.rowptr->as<int>(), an.col->as<int>(), a, v.ph,
                                                                    v.rhat, v.v, n, part, cnt, sc); });
            launch(c, "bicg_s", [&] { bicg_s_kernel<T><<<nb, kThreads, 0, c.stream>>>(v.r, v.v, v.s, n, part, cnt, sc); });
            precondition<T>(c, an, lu, v.s, v.sh, sc, 1);
            launch(c, "bicg_spmv_omega", [&] { bicg_spmv_omega_kernel<T><<<nb, kThreads, 0, c.stream>>>(an.rowptr->as<int>(), an.col->as<int>(), a, v.sh,
                                                                    v.s, v.t, n, part, cnt, sc); });
            launch(c, "bicg_xr", [&] { bicg_xr_kernel<T><<<nb, kThreads, 0, c.stream>>>(v.ph, v.sh, v.s, v.t, v.rhat, v.x, v.r, n, part, cnt, sc); });
        }
        enq += chunk;
        EQG_CUDA(cudaMemcpyAsync(c.pinned, sc, sizeof(KScal), cudaMemcpyDeviceToHost, c.stream));
        c.sync();
        std::memcpy(&h, c.pinned, sizeof(KScal));
        if (bb == 0.0) bb = h.thr / (tol * tol > 0 ? tol * tol : 1.0);
        if (h.status != ST_RUN || enq >= max_iter) break;
    }
    res.converged = h.status == ST_CONV;
    res.iterations = h.iterations;
    const double b2 = tol > 0 ? h.thr / (tol * tol) : 0.0;
    res.rel_residual = b2 > 0 ? std::sqrt(h.rr / b2) : 0.0;
    return res;
}

}  // namespace

SolveResult linear_solve(Core& c, const PatternP& p, const double* jval, const double* rhs, double* xout)
{
    if (p->rows != p->cols) fail(EQG_ERR_ARG, "solveForUpdate: Jacobian is not square");
    const std::string ordering = c.param_s("linsolver_ordering", "multicolor");
    const bool natural = ordering == "natural";
    if (!natural && ordering != "multicolor") fail(EQG_ERR_ARG, "linsolver_ordering must be natural or multicolor");
    const std::string precision = c.param_s("linsolver_precision", "double");
    const bool mixed = precision == "mixed";
    if (!mixed && precision != "double") fail(EQG_ERR_ARG, "linsolver_precision must be double or mixed");
    const double tol = c.param_d("linsolver_residual_tolerance", 1e-8);
    const int max_iter = c.param_i("linsolver_max_iterations", 1000);
    const int check_every = std::max(1, c.param_i("linsolver_check_every", 8));

    if (!p->analysis || p->analysis->natural != natural) p->analysis = analyse(c, *p, natural);
    SolverAnalysis& an = *p->analysis;
    SolveResult res;
    if (!an.ok) return res;  // structurally missing diagonal: ILU(0) cannot factor
    const int n = an.n;
    if (n == 0) {
        res.converged = true;
        return res;
    }
    // permuted matrix and factorization (FP64)
    c.factor_clock.start(c.stream);
    launch(c, "gather_values", [&] { gather_values_kernel<<<blocksFor(an.nnz), kThreads, 0, c.stream>>>(jval, an.vmap->as<int>(), an.a64->as<double>(),
                                                                       an.nnz); });
    EQG_CUDA(cudaMemcpyAsync(an.lu64->ptr, an.a64->ptr, (size_t)an.nnz * 8, cudaMemcpyDeviceToDevice, c.stream));
    EQG_CUDA(cudaMemsetAsync(an.factor_status->ptr, 0, sizeof(int), c.stream));
    const int ns = (int)an.stage_ptr.size() - 1;
    for (int s = 0; s < ns; ++s) {
        const int r0 = an.stage_ptr[s], r1 = an.stage_ptr[s + 1];
        launch(c, "ilu0_factor", [&] { ilu0_factor_stage_kernel<<<blocksFor(r1 - r0), kThreads, 0, c.stream>>>(
            r0, r1, an.rowptr->as<int>(), an.col->as<int>(), an.diag->as<int>(), an.lu64->as<double>(),
            an.factor_status->as<int>()); });
    }
    Vecs<double> v = vecs<double>(an.vec64->as<double>(), n);
    launch(c, "permute", [&] { permute_kernel<<<blocksFor(n), kThreads, 0, c.stream>>>(rhs, an.perm->as<int>(), v.b, n); });
    if (mixed) {
        if (!an.a32) {
            an.a32 = c.allocN<float>((size_t)an.nnz);
            an.lu32 = c.allocN<float>((size_t)an.nnz);
            an.vec32 = c.allocN<float>((size_t)10 * n);
        }
        launch(c, "to_float", [&] { to_float_kernel<<<blocksFor(an.nnz), kThreads, 0, c.stream>>>(an.a64->as<double>(), an.a32->as<float>(), an.nnz); });
        launch(c, "to_float", [&] { to_float_kernel<<<blocksFor(an.nnz), kThreads, 0, c.stream>>>(an.lu64->as<double>(), an.lu32->as<float>(), an.nnz); });
    }
    c.factor_clock.stop(c.stream);
    int fstat = 0;
    EQG_CUDA(cudaMemcpyAsync(c.pinned, an.factor_status->ptr, sizeof(int), cudaMemcpyDeviceToHost, c.stream));
    c.sync();
    std::memcpy(&fstat, c.pinned, sizeof(int));
    if (fstat) return res;  // zero pivot
    c.krylov_clock.start(c.stream);

    if (!mixed) {
        res = bicgstab<double>(c, an, an.a64->as<double>(), an.lu64->as<double>(), v, tol, max_iter, check_every);
        res.sweeps = 1;
    } else {
        Vecs<float> w = vecs<float>(an.vec32->as<float>(), n);
        const double inner_tol = c.param_d("linsolver_inner_tolerance", 1e-4);
        const int max_sweeps = c.param_i("linsolver_max_sweeps", 60);
        double* part = an.partials->as<double>();
        unsigned int* cnt = an.counter->as<unsigned int>();
        const int nb = blocksFor(n, kThreads, kRedBlocks);
        // x = 0, r = b
        k_fill(c, v.x, 0.0, n);
        Buf rr_dev = c.allocN<double>(2);
        launch(c, "sumsq", [&] { sumsq_kernel<<<nb, kThreads, 0, c.stream>>>(v.b, n, part, cnt, rr_dev->as<double>()); });
        launch(c, "residual", [&] { residual_kernel<<<nb, kThreads, 0, c.stream>>>(an.rowptr->as<int>(), an.col->as<int>(), an.a64->as<double>(),
                                                       v.x, v.b, v.r, w.b, n, part, cnt, rr_dev->as<double>() + 1); });
        EQG_CUDA(cudaMemcpyAsync(c.pinned, rr_dev->ptr, 2 * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
        c.sync();
        const double bb = c.pinned[0];
        double rr = c.pinned[1];
        int total_iter = 0, sweeps = 0;
        bool conv = bb == 0.0 || rr <= tol * tol * bb;
        while (!conv && sweeps < max_sweeps && total_iter < max_iter) {
            SolveResult inner = bicgstab<float>(c, an, an.a32->as<float>(), an.lu32->as<float>(), w, inner_tol,
                                                max_iter - total_iter, check_every);
            total_iter += inner.iterations;
            ++sweeps;
            launch(c, "add_float", [&] { add_float_kernel<<<blocksFor(n), kThreads, 0, c.stream>>>(v.x, w.x, n); });
            launch(c, "residual", [&] { residual_kernel<<<nb, kThreads, 0, c.stream>>>(an.rowptr->as<int>(), an.col->as<int>(),
                                                           an.a64->as<double>(), v.x, v.b, v.r, w.b, n, part, cnt,
                                                           rr_dev->as<double>() + 1); });
            EQG_CUDA(cudaMemcpyAsync(c.pinned, rr_dev->as<double>() + 1, sizeof(double), cudaMemcpyDeviceToHost,
                                     c.stream));
            c.sync();
            rr = c.pinned[0];
            conv = rr <= tol * tol * bb;
            if (inner.iterations == 0 && !inner.converged) break;  // inner breakdown
        }
        res.converged = conv;
        res.iterations = total_iter;
        res.sweeps = sweeps;
        res.rel_residual = bb > 0 ? std::sqrt(rr / bb) : 0.0;
    }
    c.krylov_clock.stop(c.stream);
    launch(c, "unpermute", [&] { unpermute_kernel<<<blocksFor(n), kThreads, 0, c.stream>>>(v.x, an.perm->as<int>(), xout, n); });
    return res;
}

}  // namespace eqg

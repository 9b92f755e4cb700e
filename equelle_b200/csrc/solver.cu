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
// Preconditioner "multigrid" (default; see the analysis section below):
// geometric-aggregation V-cycle with these ILU(0) sweeps as smoothers, which
// keeps the iteration count of the elliptic pressure part from growing with
// the grid; "ilu0": the staged ILU(0) alone.
//
// Precision "mixed": BiCGStab in FP64, the preconditioner (V-cycle or ILU
// sweeps, with FP32 copies of the factors and level matrices) in FP32.
// Precision "refine": the inner BiCGStab and the preconditioner in FP32,
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

// Writes this block's sums to `partials`; returns true, in every thread of
// the block, for the last block to finish.
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
    return last;
}

// Grid-wide sums of NV values, deterministic: block sums in fixed slots, the
// last block to finish adds them up in a fixed order with all its threads.
// Returns true in thread 0 of that block, with the sums in `out`.
template <int NV>
__device__ __forceinline__ bool grid_sum(double (&v)[NV], double* partials, unsigned int* counter, double (&out)[NV])
{
    if (!publish_partials<NV>(v, partials, counter)) return false;
    __threadfence();
    double acc[NV];
#pragma unroll
    for (int k = 0; k < NV; ++k) acc[k] = 0.0;
    for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x)
#pragma unroll
        for (int k = 0; k < NV; ++k) acc[k] += ((volatile double*)partials)[b * NV + k];
    __syncthreads();
    block_sum<NV>(acc);
    if (threadIdx.x != 0) return false;
#pragma unroll
    for (int k = 0; k < NV; ++k) out[k] = acc[k];
    *counter = 0u;
    return true;
}

// ---- matrix kernels ---------------------------------------------------------
// Level matrices used by the sweeps are in a sliced ELL layout: rows in
// slices of 32 (one warp), each slice stored column-major and padded to its
// longest row, so that a warp's k-th loads of its 32 rows are one contiguous
// 256-byte (FP64) segment.  Within a row, entries are in ascending column
// order, so the ILU(0) lower part is k < dk[r] and the upper part k > dk[r].
struct SellView {
    const int* __restrict__ slice_ptr;  // first slot of each slice
    const int* __restrict__ col;        // column of each slot
    const int* __restrict__ len;        // entries of each row
    const int* __restrict__ dk;         // position of the diagonal in each row
};

__device__ __forceinline__ int sell_base(const SellView& m, int r) { return m.slice_ptr[r >> 5] + (r & 31); }

// sum_{k0 <= k < k1} a[row, k] x[col[row, k]], added in ascending k.  With
// KM > 0 (rows of at most KM entries) the loop is unrolled so that a thread
// issues all its column and value loads before the dependent gathers of x:
// the kernels using it are bound by the latency of that load chain.
template <int KM, class T>
__device__ __forceinline__ double sell_dot(const SellView& m, int base, int k0, int k1, const T* __restrict__ a,
                                           const T* __restrict__ x)
{
    double acc = 0.0;
    if (KM == 0) {
        for (int k = k0; k < k1; ++k) {
            const int idx = base + (k << 5);
            acc += (double)a[idx] * (double)x[m.col[idx]];
        }
        return acc;
    }
    int ci[KM > 0 ? KM : 1];
    T av[KM > 0 ? KM : 1];
#pragma unroll
    for (int k = 0; k < KM; ++k) {
        const bool on = k >= k0 && k < k1;
        const int idx = base + (k << 5);
        ci[k] = on ? m.col[idx] : 0;
        av[k] = on ? a[idx] : (T)0;
    }
#pragma unroll
    for (int k = 0; k < KM; ++k)
        if (k >= k0 && k < k1) acc += (double)av[k] * (double)x[ci[k]];
    return acc;
}

// Dispatches on a level's longest row as KK (4, 8, 16; 0 = plain loop).
#define WITH_KMAX(kmax, ...)                        \
    if ((kmax) <= 4) {                              \
        constexpr int KK = 4;                       \
        __VA_ARGS__;                                \
    } else if ((kmax) <= 8) {                       \
        constexpr int KK = 8;                       \
        __VA_ARGS__;                                \
    } else if ((kmax) <= 16) {                      \
        constexpr int KK = 16;                      \
        __VA_ARGS__;                                \
    } else {                                        \
        constexpr int KK = 0;                       \
        __VA_ARGS__;                                \
    }

// dst (sliced ELL) <- src (CSR) through the slot map; padding slots get 0.
__global__ void sell_scatter_kernel(int64_t size, const int* __restrict__ map, const double* __restrict__ src,
                                    double* __restrict__ dst)
{
    GRID_STRIDE(i, size)
    {
        const int e = map[i];
        dst[i] = e >= 0 ? src[e] : 0.0;
    }
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

template <int KM, class T>
__global__ void ilu0_lower_stage_kernel(int r0, int r1, SellView m, const T* __restrict__ lu,
                                        const T* __restrict__ b, T* __restrict__ y, const KScal* sc, int skip_if_s)
{
    if (stopped(sc) || (skip_if_s && sc->s_conv)) return;
    for (int64_t rr = r0 + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; rr < r1;
         rr += (int64_t)gridDim.x * blockDim.x) {
        const int r = (int)rr;
        const double s = sell_dot<KM, T>(m, sell_base(m, r), 0, m.dk[r], lu, y);
        y[r] = (T)((double)b[r] - s);
    }
}

template <int KM, class T>
__global__ void ilu0_upper_stage_kernel(int r0, int r1, SellView m, const T* __restrict__ lu, T* __restrict__ x,
                                        const KScal* sc, int skip_if_s)
{
    if (stopped(sc) || (skip_if_s && sc->s_conv)) return;
    for (int64_t rr = r0 + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; rr < r1;
         rr += (int64_t)gridDim.x * blockDim.x) {
        const int r = (int)rr;
        const int base = sell_base(m, r);
        const int d = m.dk[r];
        const double s = sell_dot<KM, T>(m, base, d + 1, m.len[r], lu, x);
        x[r] = (T)(((double)x[r] - s) / (double)lu[base + (d << 5)]);
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
    double s[2];
    if (grid_sum<2>(d, partials, counter, s)) {
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
template <int KM, class T>
__global__ void bicg_spmv_alpha_kernel(SellView m, const T* __restrict__ a, const T* __restrict__ ph,
                                       const T* __restrict__ rhat, T* __restrict__ v, int n, double* partials,
                                       unsigned int* counter, KScal* sc)
{
    if (stopped(sc)) return;
    double d[1] = {0.0};
    GRID_STRIDE(i, n)
    {
        const double vi = sell_dot<KM, T>(m, sell_base(m, (int)i), 0, m.len[i], a, ph);
        v[i] = (T)vi;
        d[0] += (double)rhat[i] * (double)(T)vi;
    }
    double s[1];
    if (grid_sum<1>(d, partials, counter, s)) {
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
    double t[1];
    if (grid_sum<1>(d, partials, counter, t)) {
        sc->ss = t[0];
        sc->s_conv = t[0] <= sc->thr ? 1 : 0;
    }
}

// t = A sh ; omega = (t . s) / (t . t)
template <int KM, class T>
__global__ void bicg_spmv_omega_kernel(SellView m, const T* __restrict__ a, const T* __restrict__ sh,
                                       const T* __restrict__ s, T* __restrict__ t, int n, double* partials,
                                       unsigned int* counter, KScal* sc)
{
    if (stopped(sc) || sc->s_conv) return;
    double d[2] = {0.0, 0.0};
    GRID_STRIDE(i, n)
    {
        const T ti = (T)sell_dot<KM, T>(m, sell_base(m, (int)i), 0, m.len[i], a, sh);
        t[i] = ti;
        d[0] += (double)ti * (double)s[i];
        d[1] += (double)ti * (double)ti;
    }
    double u[2];
    if (grid_sum<2>(d, partials, counter, u)) {
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
    double u[2];
    if (grid_sum<2>(d, partials, counter, u)) {
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
template <int KM>
__global__ void residual_kernel(SellView m, const double* __restrict__ a, const double* __restrict__ x,
                                const double* __restrict__ b, double* __restrict__ r, float* __restrict__ r32, int n,
                                double* partials, unsigned int* counter, double* out_rr)
{
    double d[1] = {0.0};
    GRID_STRIDE(i, n)
    {
        const double ri = b[i] - sell_dot<KM, double>(m, sell_base(m, (int)i), 0, m.len[i], a, x);
        r[i] = ri;
        r32[i] = (float)ri;
        d[0] += ri * ri;
    }
    double u[1];
    if (grid_sum<1>(d, partials, counter, u)) {
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
    double u[1];
    if (grid_sum<1>(d, partials, counter, u)) {
        *out = u[0];
    }
}

// ---- multilevel preconditioner kernels -------------------------------------
// Coarse-level values: each coarse entry is the sum of the finer level's
// entries that aggregate onto it (Galerkin product R A R^T with a 0/1
// aggregation R), gathered in a fixed order.
__global__ void galerkin_kernel(int64_t nnz_c, const int* __restrict__ gptr, const int* __restrict__ gidx,
                                const double* __restrict__ fine, double* __restrict__ coarse)
{
    GRID_STRIDE(c, nnz_c)
    {
        double s = 0.0;
        const int k1 = gptr[c + 1];
        for (int k = gptr[c]; k < k1; ++k) s += fine[gidx[k]];
        coarse[c] = s;
    }
}

__device__ __forceinline__ bool mg_skip(const KScal* sc, int skip_if_s)
{
    return stopped(sc) || (skip_if_s && sc->s_conv);
}

// out = b - A x
template <int KM, class T>
__global__ void mg_residual_kernel(int n, SellView m, const T* __restrict__ a, const T* __restrict__ x,
                                   const T* __restrict__ b, T* __restrict__ out, const KScal* sc, int skip_if_s)
{
    if (mg_skip(sc, skip_if_s)) return;
    GRID_STRIDE(i, n) out[i] = (T)((double)b[i] - sell_dot<KM, T>(m, sell_base(m, (int)i), 0, m.len[i], a, x));
}

// rc[P] = sum of t over the members of aggregate P
template <class T>
__global__ void mg_restrict_kernel(int nc, const int* __restrict__ mptr, const int* __restrict__ midx,
                                   const T* __restrict__ t, T* __restrict__ rc, const KScal* sc, int skip_if_s)
{
    if (mg_skip(sc, skip_if_s)) return;
    GRID_STRIDE(P, nc)
    {
        double s = 0.0;
        const int k1 = mptr[P + 1];
        for (int k = mptr[P]; k < k1; ++k) s += (double)t[midx[k]];
        rc[P] = (T)s;
    }
}

// z[i] += ec[agg[i]] (piecewise-constant prolongation)
template <class T>
__global__ void mg_prolong_kernel(int n, const int* __restrict__ agg, const T* __restrict__ ec, T* __restrict__ z,
                                  const KScal* sc, int skip_if_s)
{
    if (mg_skip(sc, skip_if_s)) return;
    GRID_STRIDE(i, n) z[i] = (T)((double)z[i] + (double)ec[agg[i]]);
}

template <class T>
__global__ void mg_add_kernel(int n, const T* __restrict__ w, T* __restrict__ z, const KScal* sc, int skip_if_s)
{
    if (mg_skip(sc, skip_if_s)) return;
    GRID_STRIDE(i, n) z[i] = (T)((double)z[i] + (double)w[i]);
}

// Inverse of the coarsest matrix (n <= kCoarsest) by Gauss-Jordan with
// partial pivoting on [A | I], one block.
constexpr int kCoarsest = 128;

__global__ void dense_inverse_kernel(int n, const int* __restrict__ rowptr, const int* __restrict__ col,
                                     const double* __restrict__ a, double* __restrict__ work,
                                     double* __restrict__ inv, int* status)
{
    __shared__ double factor[kCoarsest];
    __shared__ int piv;
    __shared__ double pval;
    const int w2 = 2 * n;
    for (int idx = threadIdx.x; idx < n * w2; idx += blockDim.x) work[idx] = 0.0;
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        for (int e = rowptr[i]; e < rowptr[i + 1]; ++e) work[i * w2 + col[e]] = a[e];
        work[i * w2 + n + i] = 1.0;
    }
    __syncthreads();
    for (int k = 0; k < n; ++k) {
        if (threadIdx.x == 0) {
            int best = k;
            double bv = fabs(work[k * w2 + k]);
            for (int r = k + 1; r < n; ++r) {
                const double v = fabs(work[r * w2 + k]);
                if (v > bv) {
                    bv = v;
                    best = r;
                }
            }
            piv = best;
            if (bv == 0.0) *status = 1;
        }
        __syncthreads();
        if (piv != k)
            for (int j = threadIdx.x; j < w2; j += blockDim.x) {
                const double t = work[k * w2 + j];
                work[k * w2 + j] = work[piv * w2 + j];
                work[piv * w2 + j] = t;
            }
        __syncthreads();
        if (threadIdx.x == 0) pval = work[k * w2 + k];
        __syncthreads();
        for (int j = threadIdx.x; j < w2; j += blockDim.x) work[k * w2 + j] /= pval;
        __syncthreads();
        for (int r = threadIdx.x; r < n; r += blockDim.x) factor[r] = work[r * w2 + k];
        __syncthreads();
        for (int idx = threadIdx.x; idx < n * w2; idx += blockDim.x) {
            const int r = idx / w2, j = idx - r * w2;
            if (r != k) work[idx] -= factor[r] * work[k * w2 + j];
        }
        __syncthreads();
    }
    for (int idx = threadIdx.x; idx < n * n; idx += blockDim.x) {
        const int r = idx / n, j = idx - r * n;
        inv[idx] = work[r * w2 + n + j];
    }
}

template <class T>
__global__ void dense_apply_kernel(int n, const T* __restrict__ inv, const T* __restrict__ r, T* __restrict__ z,
                                   const KScal* sc, int skip_if_s)
{
    if (mg_skip(sc, skip_if_s)) return;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        double s = 0.0;
        for (int j = 0; j < n; ++j) s += (double)inv[i * n + j] * (double)r[j];
        z[i] = (T)s;
    }
}

// FP64 <-> FP32 copies around an FP32 preconditioner.
__global__ void pc_to_f32_kernel(const double* __restrict__ a, float* __restrict__ b, int n, const KScal* sc,
                                 int skip_if_s)
{
    if (mg_skip(sc, skip_if_s)) return;
    GRID_STRIDE(i, n) b[i] = (float)a[i];
}

__global__ void pc_to_f64_kernel(const float* __restrict__ a, double* __restrict__ b, int n, const KScal* sc,
                                 int skip_if_s)
{
    if (mg_skip(sc, skip_if_s)) return;
    GRID_STRIDE(i, n) b[i] = (double)a[i];
}

}  // namespace

// ---------------------------------------------------------------------------
// Host analysis, cached per Jacobian pattern.
//
// Multilevel preconditioner (the default when the system is laid out as
// `ncomp` blocks of one unknown per grid cell, as newtonSolve and
// newtonSolveSystem stack them): geometric aggregation of 2x2x2 cells per
// unknown block, Galerkin coarse matrices R A R^T, a V(1,1) cycle with one
// ILU(0) sweep before and after the coarse correction on every level, and a
// dense inverse on the coarsest level (<= 128 unknowns).  Otherwise plain
// ILU(0).
// ---------------------------------------------------------------------------
struct HostCsr {
    int n = 0;
    std::vector<int> ptr, col;
};

struct Level {
    int n = 0;
    int64_t nnz = 0;
    int cx = 1, cy = 1, cz = 1;    // cells of this level's grid
    bool coarsest = false;
    std::vector<int> stage_ptr;    // stages (colours or wavefronts) in the permuted order
    Buf perm, rowptr, col, diag;   // permuted pattern
    Buf gptr, gidx;                // Galerkin gather from the finer level (levels > 0)
    Buf agg, mptr, midx;           // to the next coarser level
    Buf a64, lu64;                 // CSR values: matrix, ILU(0) factors
    int64_t sell_size = 0;         // sliced ELL copies used by the sweeps
    int kmax = 0;                  // longest row
    Buf sell_ptr, sell_col, sell_len, sell_dk, sell_map;
    Buf as64, lus64, as32, lus32;
    Buf v64, v32;                  // 4 work vectors: r, z, t, w
    SellView view() const
    {
        return SellView{sell_ptr->as<int>(), sell_col->as<int>(), sell_len->as<int>(), sell_dk->as<int>()};
    }
    Buf work64, inv64, inv32;      // coarsest level
};

struct SolverAnalysis {
    int n = 0;
    int64_t nnz = 0;
    bool natural = false;
    bool ok = true;  // every row has a diagonal entry
    bool multigrid = false;
    std::vector<Level> levels;
    Buf vmap;        // level-0 permuted entry <- Jacobian entry
    Buf vec64, vec32, scal, partials, counter, factor_status;
    Buf pc32;        // FP32 input and output of an FP32 preconditioner
    // CUDA graphs of `chunk` BiCGStab iterations: [0] FP64, [1] FP32, [2] FP64
    // with an FP32 preconditioner
    struct IterGraph {
        cudaGraphExec_t exec = nullptr;
        int chunk = 0;
        int64_t kernels = 0;
    } graph[3];
    ~SolverAnalysis()
    {
        for (auto& g : graph)
            if (g.exec) cudaGraphExecDestroy(g.exec);
    }
};

namespace {

// Stage key of every row: wavefront level of the natural order, or greedy
// colour, over the symmetrised pattern.
std::vector<int> stage_keys(const HostCsr& A, bool natural)
{
    const int n = A.n;
    const int64_t nnz = A.ptr[n];
    std::vector<int> tp(n + 1, 0), tr(nnz > 0 ? nnz : 1);
    for (int64_t e = 0; e < nnz; ++e) tp[A.col[e] + 1]++;
    for (int i = 0; i < n; ++i) tp[i + 1] += tp[i];
    {
        std::vector<int> pos(tp.begin(), tp.end() - 1);
        for (int i = 0; i < n; ++i)
            for (int e = A.ptr[i]; e < A.ptr[i + 1]; ++e) tr[pos[A.col[e]]++] = i;
    }
    std::vector<int> key(n, 0);
    if (natural) {
        for (int i = 0; i < n; ++i) {
            int lv = 0;
            for (int e = A.ptr[i]; e < A.ptr[i + 1]; ++e)
                if (A.col[e] < i) lv = std::max(lv, key[A.col[e]] + 1);
            for (int e = tp[i]; e < tp[i + 1]; ++e)
                if (tr[e] < i) lv = std::max(lv, key[tr[e]] + 1);
            key[i] = lv;
        }
    } else {
        std::vector<int> mark(64, -1);
        for (int i = 0; i < n; ++i) {
            auto see = [&](int j) {
                if (j < i) {
                    const int cj = key[j];
                    if (cj >= (int)mark.size()) mark.resize(cj + 1, -1);
                    mark[cj] = i;
                }
            };
            for (int e = A.ptr[i]; e < A.ptr[i + 1]; ++e) see(A.col[e]);
            for (int e = tp[i]; e < tp[i + 1]; ++e) see(tr[e]);
            int cc = 0;
            while (cc < (int)mark.size() && mark[cc] == i) ++cc;
            key[i] = cc;
        }
    }
    return key;
}

Buf upload_ints(Core& c, const std::vector<int>& v)
{
    Buf b = c.allocN<int>(v.empty() ? 1 : v.size());
    if (!v.empty()) EQG_CUDA(cudaMemcpyAsync(b->ptr, v.data(), v.size() * 4, cudaMemcpyHostToDevice, c.stream));
    return b;
}

// Orders the rows of `A` by stage, builds the permuted pattern with
// ascending columns, and returns the host permutation (new -> old), its
// inverse and, for every permuted entry, its entry index in `A`.
void order_level(Core& c, const HostCsr& A, bool natural, Level& L, std::vector<int>& perm, std::vector<int>& iperm,
                 std::vector<int>& pcsr_ptr, std::vector<int>& pcsr_col, std::vector<int>& emap, bool& ok)
{
    const int n = A.n;
    const int64_t nnz = A.ptr[n];
    const std::vector<int> key = stage_keys(A, natural);
    const int nst = n > 0 ? *std::max_element(key.begin(), key.end()) + 1 : 0;
    L.stage_ptr.assign(nst + 1, 0);
    for (int i = 0; i < n; ++i) L.stage_ptr[key[i] + 1]++;
    for (int s = 0; s < nst; ++s) L.stage_ptr[s + 1] += L.stage_ptr[s];
    perm.assign(n, 0);
    iperm.assign(n, 0);
    {
        std::vector<int> pos(L.stage_ptr.begin(), L.stage_ptr.end() - 1);
        for (int i = 0; i < n; ++i) perm[pos[key[i]]++] = i;
    }
    for (int r = 0; r < n; ++r) iperm[perm[r]] = r;
    pcsr_ptr.assign(n + 1, 0);
    pcsr_col.assign(nnz > 0 ? nnz : 1, 0);
    emap.assign(nnz > 0 ? nnz : 1, 0);
    std::vector<int> diag(n, 0);
    std::vector<std::pair<int, int>> row;
    for (int r = 0; r < n; ++r) {
        const int i = perm[r];
        row.clear();
        for (int e = A.ptr[i]; e < A.ptr[i + 1]; ++e) row.emplace_back(iperm[A.col[e]], e);
        std::sort(row.begin(), row.end());
        pcsr_ptr[r + 1] = pcsr_ptr[r] + (int)row.size();
        int o = pcsr_ptr[r];
        bool has = false;
        for (auto& ce : row) {
            if (ce.first == r) {
                diag[r] = o;
                has = true;
            }
            pcsr_col[o] = ce.first;
            emap[o] = ce.second;
            ++o;
        }
        if (!has) ok = false;
    }
    L.n = n;
    L.nnz = nnz;
    {
        // sliced ELL, 32 rows per slice (one thread per row)
        const int nsl = (n + 31) / 32;
        std::vector<int> sp(nsl + 1, 0), len(n), dk(n);
        for (int sl = 0; sl < nsl; ++sl) {
            int w = 0;
            for (int r = sl * 32; r < std::min(n, sl * 32 + 32); ++r) w = std::max(w, pcsr_ptr[r + 1] - pcsr_ptr[r]);
            sp[sl + 1] = sp[sl] + 32 * w;
        }
        const int64_t size = sp[nsl];
        std::vector<int> scol(size > 0 ? size : 1, 0), smap(size > 0 ? size : 1, -1);
        for (int r = 0; r < n; ++r) {
            const int base = sp[r / 32] + (r % 32);
            len[r] = pcsr_ptr[r + 1] - pcsr_ptr[r];
            dk[r] = diag[r] - pcsr_ptr[r];
            const int w = (sp[r / 32 + 1] - sp[r / 32]) / 32;
            for (int k = 0; k < w; ++k) {
                const int idx = base + 32 * k;
                if (k < len[r]) {
                    scol[idx] = pcsr_col[pcsr_ptr[r] + k];
                    smap[idx] = pcsr_ptr[r] + k;
                } else {
                    scol[idx] = r;  // padding: a valid column, value 0, never read by the sweeps
                }
            }
        }
        L.sell_size = size;
        L.kmax = 0;
        for (int r = 0; r < n; ++r) L.kmax = std::max(L.kmax, len[r]);
        L.sell_ptr = upload_ints(c, sp);
        L.sell_col = upload_ints(c, scol);
        L.sell_len = upload_ints(c, len);
        L.sell_dk = upload_ints(c, dk);
        L.sell_map = upload_ints(c, smap);
        L.as64 = c.allocN<double>((size_t)(size > 0 ? size : 1));
        L.lus64 = c.allocN<double>((size_t)(size > 0 ? size : 1));
    }
    L.perm = upload_ints(c, perm);
    L.rowptr = upload_ints(c, pcsr_ptr);
    L.col = upload_ints(c, pcsr_col);
    L.diag = upload_ints(c, diag);
    const size_t nz = (size_t)(nnz > 0 ? nnz : 1);
    L.a64 = c.allocN<double>(nz);
    L.lu64 = c.allocN<double>(nz);
    L.v64 = c.allocN<double>((size_t)4 * (n > 0 ? n : 1));
}

std::shared_ptr<SolverAnalysis> analyse(Core& c, const Pattern& p, bool natural)
{
    auto an = std::make_shared<SolverAnalysis>();
    const int n = p.rows;
    an->n = n;
    an->nnz = p.nnz;
    an->natural = natural;
    HostCsr A;
    A.n = n;
    A.ptr.resize(n + 1);
    A.col.resize(p.nnz > 0 ? p.nnz : 1);
    EQG_CUDA(cudaMemcpyAsync(A.ptr.data(), p.rowptr->ptr, (size_t)(n + 1) * 4, cudaMemcpyDeviceToHost, c.stream));
    if (p.nnz > 0)
        EQG_CUDA(cudaMemcpyAsync(A.col.data(), p.colind->ptr, (size_t)p.nnz * 4, cudaMemcpyDeviceToHost, c.stream));
    c.sync();

    std::vector<int> perm, iperm, pptr, pcol, emap;
    an->levels.emplace_back();
    order_level(c, A, natural, an->levels[0], perm, iperm, pptr, pcol, emap, an->ok);
    an->vmap = upload_ints(c, emap);

    const std::string pre = c.param_s("linsolver_preconditioner", "multigrid");
    if (pre != "multigrid" && pre != "ilu0") fail(EQG_ERR_ARG, "linsolver_preconditioner must be multigrid or ilu0");
    const int ncomp = (c.nc > 0 && n % c.nc == 0) ? n / c.nc : 0;
    an->multigrid = pre == "multigrid" && ncomp >= 1 && ncomp <= 8 && n > kCoarsest && an->ok;
    an->levels[0].cx = c.nx;
    an->levels[0].cy = c.ny;
    an->levels[0].cz = c.nz;
    if (an->multigrid) {
        // the finer level in its natural ordering, with its permutation
        HostCsr fine = A;
        std::vector<int> fperm = perm, fiperm = iperm, fptr = pptr, fcol = pcol;
        for (;;) {
            Level& F = an->levels.back();
            const int fcx = F.cx, fcy = F.cy, fcz = F.cz;
            const int fcells = fcx * fcy * fcz;
            const int ccx = (fcx + 1) / 2, ccy = (fcy + 1) / 2, ccz = fcz > 1 ? (fcz + 1) / 2 : 1;
            const int ccells = ccx * ccy * ccz;
            const int nc_unk = ncomp * ccells;
            // aggregate of every fine unknown (natural indices)
            std::vector<int> agg_nat(fine.n);
            for (int u = 0; u < fine.n; ++u) {
                const int comp = u / fcells, cell = u - comp * fcells;
                const int i = cell % fcx, j = (cell / fcx) % fcy, k = cell / (fcx * fcy);
                agg_nat[u] = comp * ccells + (i / 2) + ccx * ((j / 2) + ccy * (fcz > 1 ? k / 2 : 0));
            }
            // coarse pattern (natural ordering)
            HostCsr C;
            C.n = nc_unk;
            {
                std::vector<std::vector<int>> rows(nc_unk);
                std::vector<int> mark(nc_unk, -1);
                std::vector<std::vector<int>> members(nc_unk);
                for (int u = 0; u < fine.n; ++u) members[agg_nat[u]].push_back(u);
                C.ptr.assign(nc_unk + 1, 0);
                std::vector<int> cols;
                for (int U = 0; U < nc_unk; ++U) {
                    for (int u : members[U])
                        for (int e = fine.ptr[u]; e < fine.ptr[u + 1]; ++e) {
                            const int V = agg_nat[fine.col[e]];
                            if (mark[V] != U) {
                                mark[V] = U;
                                rows[U].push_back(V);
                            }
                        }
                    std::sort(rows[U].begin(), rows[U].end());
                    C.ptr[U + 1] = C.ptr[U] + (int)rows[U].size();
                }
                C.col.resize(C.ptr[nc_unk] > 0 ? C.ptr[nc_unk] : 1);
                for (int U = 0; U < nc_unk; ++U) std::copy(rows[U].begin(), rows[U].end(), C.col.begin() + C.ptr[U]);
            }
            an->levels.emplace_back();
            Level& Lc = an->levels.back();
            Level& Lf = an->levels[an->levels.size() - 2];
            Lc.cx = ccx;
            Lc.cy = ccy;
            Lc.cz = ccz;
            std::vector<int> cperm, ciperm, cptr, ccol, cemap;
            bool cok = true;
            order_level(c, C, natural, Lc, cperm, ciperm, cptr, ccol, cemap, cok);
            if (!cok) fail(EQG_ERR_DEVICE, "coarse level without a diagonal entry");
            // aggregation in permuted indices, and aggregate members
            std::vector<int> aggp(fine.n);
            for (int pf = 0; pf < fine.n; ++pf) aggp[pf] = ciperm[agg_nat[fperm[pf]]];
            std::vector<int> mptr(nc_unk + 1, 0), midx(fine.n);
            for (int pf = 0; pf < fine.n; ++pf) mptr[aggp[pf] + 1]++;
            for (int P = 0; P < nc_unk; ++P) mptr[P + 1] += mptr[P];
            {
                std::vector<int> pos(mptr.begin(), mptr.end() - 1);
                for (int pf = 0; pf < fine.n; ++pf) midx[pos[aggp[pf]]++] = pf;
            }
            Lf.agg = upload_ints(c, aggp);
            Lf.mptr = upload_ints(c, mptr);
            Lf.midx = upload_ints(c, midx);
            // Galerkin gather: coarse permuted entry <- fine permuted entries
            const int64_t fnnz = fptr[fine.n];
            std::vector<int> target(fnnz > 0 ? fnnz : 1);
            for (int pf = 0; pf < fine.n; ++pf) {
                const int P = aggp[pf];
                for (int e = fptr[pf]; e < fptr[pf + 1]; ++e) {
                    const int Q = aggp[fcol[e]];
                    const int* lo = ccol.data() + cptr[P];
                    const int* hi = ccol.data() + cptr[P + 1];
                    const int* q = std::lower_bound(lo, hi, Q);
                    target[e] = (int)(q - ccol.data());
                }
            }
            const int64_t cnnz = cptr[nc_unk];
            std::vector<int> gptr(cnnz + 1, 0), gidx(fnnz > 0 ? fnnz : 1);
            for (int64_t e = 0; e < fnnz; ++e) gptr[target[e] + 1]++;
            for (int64_t k = 0; k < cnnz; ++k) gptr[k + 1] += gptr[k];
            {
                std::vector<int> pos(gptr.begin(), gptr.end() - 1);
                for (int64_t e = 0; e < fnnz; ++e) gidx[pos[target[e]]++] = (int)e;
            }
            Lc.gptr = upload_ints(c, gptr);
            Lc.gidx = upload_ints(c, gidx);
            if (nc_unk <= kCoarsest || (ccx == 1 && ccy == 1 && ccz == 1)) {
                if (nc_unk > kCoarsest) {
                    an->multigrid = false;  // cannot coarsen further and too large to invert
                    an->levels.resize(1);
                    break;
                }
                Lc.coarsest = true;
                Lc.work64 = c.allocN<double>((size_t)2 * nc_unk * nc_unk);
                Lc.inv64 = c.allocN<double>((size_t)nc_unk * nc_unk);
                break;
            }
            fine = std::move(C);
            fperm = std::move(cperm);
            fiperm = std::move(ciperm);
            fptr = std::move(cptr);
            fcol = std::move(ccol);
        }
    }
    an->vec64 = c.allocN<double>((size_t)10 * (n > 0 ? n : 1));
    an->scal = c.alloc(sizeof(KScal));
    an->partials = c.allocN<double>((size_t)kRedBlocks * 2);
    an->counter = c.allocN<unsigned int>(1);
    an->factor_status = c.allocN<int>(1);
    EQG_CUDA(cudaMemsetAsync(an->counter->ptr, 0, sizeof(unsigned int), c.stream));
    c.sync();
    if (c.verbose > 2 && an->multigrid) {
        std::printf("        multigrid levels:");
        for (auto& L : an->levels) std::printf(" %d(%zu stages)", L.n, L.stage_ptr.size() - 1);
        std::printf("\n");
    }
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
const T* level_a(const Level& L);
template <>
const double* level_a<double>(const Level& L) { return L.as64->as<double>(); }
template <>
const float* level_a<float>(const Level& L) { return L.as32->as<float>(); }
template <class T>
const T* level_lu(const Level& L);
template <>
const double* level_lu<double>(const Level& L) { return L.lus64->as<double>(); }
template <>
const float* level_lu<float>(const Level& L) { return L.lus32->as<float>(); }
template <class T>
T* level_vec(const Level& L, int k);
template <>
double* level_vec<double>(const Level& L, int k) { return L.v64->as<double>() + (size_t)k * (L.n > 0 ? L.n : 1); }
template <>
float* level_vec<float>(const Level& L, int k) { return L.v32->as<float>() + (size_t)k * (L.n > 0 ? L.n : 1); }
template <class T>
const T* level_inv(const Level& L);
template <>
const double* level_inv<double>(const Level& L) { return L.inv64->as<double>(); }
template <>
const float* level_inv<float>(const Level& L) { return L.inv32->as<float>(); }

// out = M^{-1} in for the ILU(0) factors of one level.
template <class T>
void ilu_apply(Core& c, const Level& L, const T* in, T* out, const KScal* sc, int skip_if_s)
{
    const T* lu = level_lu<T>(L);
    const int ns = (int)L.stage_ptr.size() - 1;
    for (int s = 0; s < ns; ++s) {
        const int r0 = L.stage_ptr[s], r1 = L.stage_ptr[s + 1];
        WITH_KMAX(L.kmax, launch(c, "ilu0_lower", [&] {
            ilu0_lower_stage_kernel<KK, T><<<blocksFor(r1 - r0), kThreads, 0, c.stream>>>(r0, r1, L.view(), lu, in,
                                                                                          out, sc, skip_if_s);
        }));
    }
    for (int s = ns - 1; s >= 0; --s) {
        const int r0 = L.stage_ptr[s], r1 = L.stage_ptr[s + 1];
        WITH_KMAX(L.kmax, launch(c, "ilu0_upper", [&] {
            ilu0_upper_stage_kernel<KK, T><<<blocksFor(r1 - r0), kThreads, 0, c.stream>>>(r0, r1, L.view(), lu, out,
                                                                                          sc, skip_if_s);
        }));
    }
}

// z = V-cycle(r) on level l.
template <class T>
void vcycle(Core& c, const SolverAnalysis& an, size_t l, const T* r, T* z, const KScal* sc, int skip)
{
    const Level& L = an.levels[l];
    const int n = L.n;
    if (L.coarsest) {
        launch(c, "mg_dense_apply",
               [&] { dense_apply_kernel<T><<<1, kThreads, 0, c.stream>>>(n, level_inv<T>(L), r, z, sc, skip); });
        return;
    }
    const Level& C = an.levels[l + 1];
    T* t = level_vec<T>(L, 2);
    T* w = level_vec<T>(L, 3);
    T* rc = level_vec<T>(C, 0);
    T* zc = level_vec<T>(C, 1);
    const T* a = level_a<T>(L);
    ilu_apply<T>(c, L, r, z, sc, skip);
    WITH_KMAX(L.kmax, launch(c, "mg_residual", [&] {
        mg_residual_kernel<KK, T><<<blocksFor(n), kThreads, 0, c.stream>>>(n, L.view(), a, z, r, t, sc, skip);
    }));
    launch(c, "mg_restrict", [&] {
        mg_restrict_kernel<T><<<blocksFor(C.n), kThreads, 0, c.stream>>>(C.n, L.mptr->as<int>(), L.midx->as<int>(), t,
                                                                          rc, sc, skip);
    });
    vcycle<T>(c, an, l + 1, rc, zc, sc, skip);
    launch(c, "mg_prolong", [&] {
        mg_prolong_kernel<T><<<blocksFor(n), kThreads, 0, c.stream>>>(n, L.agg->as<int>(), zc, z, sc, skip);
    });
    WITH_KMAX(L.kmax, launch(c, "mg_residual", [&] {
        mg_residual_kernel<KK, T><<<blocksFor(n), kThreads, 0, c.stream>>>(n, L.view(), a, z, r, t, sc, skip);
    }));
    ilu_apply<T>(c, L, t, w, sc, skip);
    launch(c, "mg_add", [&] { mg_add_kernel<T><<<blocksFor(n), kThreads, 0, c.stream>>>(n, w, z, sc, skip); });
}

template <class T>
void precondition(Core& c, const SolverAnalysis& an, const T* in, T* out, const KScal* sc, int skip_if_s)
{
    if (an.multigrid) vcycle<T>(c, an, 0, in, out, sc, skip_if_s);
    else ilu_apply<T>(c, an.levels[0], in, out, sc, skip_if_s);
}

// out = M^{-1} in with the FP32 copy of the preconditioner, for FP64 vectors.
void precondition_f32(Core& c, const SolverAnalysis& an, const double* in, double* out, const KScal* sc, int skip_if_s)
{
    const int n = an.n;
    float* in32 = an.pc32->as<float>();
    float* out32 = in32 + n;
    launch(c, "pc_to_f32",
           [&] { pc_to_f32_kernel<<<blocksFor(n), kThreads, 0, c.stream>>>(in, in32, n, sc, skip_if_s); });
    precondition<float>(c, an, in32, out32, sc, skip_if_s);
    launch(c, "pc_to_f64",
           [&] { pc_to_f64_kernel<<<blocksFor(n), kThreads, 0, c.stream>>>(out32, out, n, sc, skip_if_s); });
}

template <class T>
void apply_pc(Core& c, const SolverAnalysis& an, const T* in, T* out, const KScal* sc, int skip_if_s, bool pc32)
{
    if constexpr (sizeof(T) == sizeof(double)) {
        if (pc32) {
            precondition_f32(c, an, in, out, sc, skip_if_s);
            return;
        }
    }
    precondition<T>(c, an, in, out, sc, skip_if_s);
}

// BiCGStab on the permuted system with values a; v.b holds the right-hand
// side.
template <class T>
SolveResult bicgstab(Core& c, SolverAnalysis& an, const T* a, Vecs<T> v, double tol, int max_iter, int check_every,
                     bool pc32 = false)
{
    const int n = an.n;
    const Level& L0 = an.levels[0];
    KScal* sc = an.scal->as<KScal>();
    double* part = an.partials->as<double>();
    unsigned int* cnt = an.counter->as<unsigned int>();
    const int nb = blocksFor(n, kThreads, kRedBlocks);
    launch(c, "bicg_init", [&] {
        bicg_init_kernel<T><<<nb, kThreads, 0, c.stream>>>(v.b, v.r, v.rhat, v.p, v.v, v.x, n, part, cnt, sc, tol * tol);
    });
    auto iteration = [&] {
        launch(c, "bicg_p", [&] { bicg_p_kernel<T><<<blocksFor(n), kThreads, 0, c.stream>>>(v.r, v.v, v.p, n, sc); });
        apply_pc<T>(c, an, v.p, v.ph, sc, 0, pc32);
        WITH_KMAX(L0.kmax, launch(c, "bicg_spmv_alpha", [&] {
            bicg_spmv_alpha_kernel<KK, T><<<nb, kThreads, 0, c.stream>>>(L0.view(), a, v.ph, v.rhat, v.v, n, part, cnt,
                                                                        sc);
        }));
        launch(c, "bicg_s", [&] { bicg_s_kernel<T><<<nb, kThreads, 0, c.stream>>>(v.r, v.v, v.s, n, part, cnt, sc); });
        apply_pc<T>(c, an, v.s, v.sh, sc, 1, pc32);
        WITH_KMAX(L0.kmax, launch(c, "bicg_spmv_omega", [&] {
            bicg_spmv_omega_kernel<KK, T><<<nb, kThreads, 0, c.stream>>>(L0.view(), a, v.sh, v.s, v.t, n, part, cnt,
                                                                        sc);
        }));
        launch(c, "bicg_xr", [&] {
            bicg_xr_kernel<T><<<nb, kThreads, 0, c.stream>>>(v.ph, v.sh, v.s, v.t, v.rhat, v.x, v.r, n, part, cnt, sc);
        });
    };
    // Graph of `check_every` iterations, captured once per analysis and
    // precision; kernel arguments are fixed (buffers of the analysis,
    // scalars in device memory).  Kernel timing (time_kernel) needs one
    // event pair per launch, so timed runs launch eagerly.
    const bool graphs = c.timed_kernel.empty() && c.param_i("linsolver_graphs", 1) != 0;
    SolverAnalysis::IterGraph& g = an.graph[sizeof(T) == sizeof(double) ? (pc32 ? 2 : 0) : 1];
    if (graphs && (!g.exec || g.chunk != check_every)) {
        if (g.exec) {
            cudaGraphExecDestroy(g.exec);
            g.exec = nullptr;
        }
        const int64_t before = c.launches.load();
        cudaGraph_t graph = nullptr;
        EQG_CUDA(cudaStreamBeginCapture(c.stream, cudaStreamCaptureModeThreadLocal));
        try {
            for (int k = 0; k < check_every; ++k) iteration();
        } catch (...) {
            cudaStreamEndCapture(c.stream, &graph);
            if (graph) cudaGraphDestroy(graph);
            throw;
        }
        EQG_CUDA(cudaStreamEndCapture(c.stream, &graph));
        const cudaError_t ie = cudaGraphInstantiate(&g.exec, graph, 0);
        cudaGraphDestroy(graph);
        if (ie != cudaSuccess) fail(EQG_ERR_DEVICE, std::string("graph instantiation failed: ") + cudaGetErrorString(ie));
        g.kernels = c.launches.load() - before;
        c.launches -= g.kernels;  // captured, not executed
        g.chunk = check_every;
    }
    SolveResult res;
    KScal h{};
    int enq = 0;
    for (;;) {
        const int chunk = std::min(check_every, max_iter - enq);
        if (graphs && chunk == g.chunk) {
            EQG_CUDA(cudaGraphLaunch(g.exec, c.stream));
            c.launches += g.kernels;
        } else {
            for (int k = 0; k < chunk; ++k) iteration();
        }
        enq += chunk;
        EQG_CUDA(cudaMemcpyAsync(c.pinned, sc, sizeof(KScal), cudaMemcpyDeviceToHost, c.stream));
        c.sync();
        std::memcpy(&h, c.pinned, sizeof(KScal));
        if (h.status != ST_RUN || enq >= max_iter) break;
    }
    res.converged = h.status == ST_CONV;
    res.iterations = h.iterations;
    const double b2 = tol > 0 ? h.thr / (tol * tol) : 0.0;
    res.rel_residual = b2 > 0 ? std::sqrt(h.rr / b2) : 0.0;
    return res;
}

void factor_level(Core& c, const Level& L, int* status)
{
    EQG_CUDA(cudaMemcpyAsync(L.lu64->ptr, L.a64->ptr, (size_t)L.nnz * 8, cudaMemcpyDeviceToDevice, c.stream));
    const int ns = (int)L.stage_ptr.size() - 1;
    for (int s = 0; s < ns; ++s) {
        const int r0 = L.stage_ptr[s], r1 = L.stage_ptr[s + 1];
        launch(c, "ilu0_factor", [&] {
            ilu0_factor_stage_kernel<<<blocksFor(r1 - r0), kThreads, 0, c.stream>>>(
                r0, r1, L.rowptr->as<int>(), L.col->as<int>(), L.diag->as<int>(), L.lu64->as<double>(), status);
        });
    }
}

void to_float(Core& c, const Buf& src, Buf& dst, int64_t n)
{
    if (!dst) dst = c.allocN<float>((size_t)(n > 0 ? n : 1));
    launch(c, "to_float",
           [&] { to_float_kernel<<<blocksFor(n), kThreads, 0, c.stream>>>(src->as<double>(), dst->as<float>(), n); });
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
    const bool refine = precision == "refine";
    if (!mixed && !refine && precision != "double")
        fail(EQG_ERR_ARG, "linsolver_precision must be double, mixed or refine");
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
    // level matrices and their factorizations (FP64)
    c.factor_clock.start(c.stream);
    const Level& L0 = an.levels[0];
    launch(c, "gather_values", [&] {
        gather_values_kernel<<<blocksFor(an.nnz), kThreads, 0, c.stream>>>(jval, an.vmap->as<int>(),
                                                                           L0.a64->as<double>(), an.nnz);
    });
    for (size_t l = 1; l < an.levels.size(); ++l) {
        const Level& F = an.levels[l - 1];
        const Level& C = an.levels[l];
        launch(c, "mg_galerkin", [&] {
            galerkin_kernel<<<blocksFor(C.nnz), kThreads, 0, c.stream>>>(C.nnz, C.gptr->as<int>(), C.gidx->as<int>(),
                                                                         F.a64->as<double>(), C.a64->as<double>());
        });
    }
    EQG_CUDA(cudaMemsetAsync(an.factor_status->ptr, 0, sizeof(int), c.stream));
    for (auto& L : an.levels) {
        launch(c, "sell_scatter", [&] {
            sell_scatter_kernel<<<blocksFor(L.sell_size), kThreads, 0, c.stream>>>(
                L.sell_size, L.sell_map->as<int>(), L.a64->as<double>(), L.as64->as<double>());
        });
        if (L.coarsest) {
            launch(c, "mg_dense_inverse", [&] {
                dense_inverse_kernel<<<1, 1024, 0, c.stream>>>(L.n, L.rowptr->as<int>(), L.col->as<int>(),
                                                               L.a64->as<double>(), L.work64->as<double>(),
                                                               L.inv64->as<double>(), an.factor_status->as<int>());
            });
        } else {
            factor_level(c, L, an.factor_status->as<int>());
            launch(c, "sell_scatter", [&] {
                sell_scatter_kernel<<<blocksFor(L.sell_size), kThreads, 0, c.stream>>>(
                    L.sell_size, L.sell_map->as<int>(), L.lu64->as<double>(), L.lus64->as<double>());
            });
        }
    }
    Vecs<double> v = vecs<double>(an.vec64->as<double>(), n);
    launch(c, "permute",
           [&] { permute_kernel<<<blocksFor(n), kThreads, 0, c.stream>>>(rhs, L0.perm->as<int>(), v.b, n); });
    if (mixed || refine) {
        for (auto& L : an.levels) {
            to_float(c, L.as64, L.as32, L.sell_size);
            if (L.coarsest) to_float(c, L.inv64, L.inv32, (int64_t)L.n * L.n);
            else to_float(c, L.lus64, L.lus32, L.sell_size);
            if (!L.v32) L.v32 = c.allocN<float>((size_t)4 * (L.n > 0 ? L.n : 1));
        }
        if (refine && !an.vec32) an.vec32 = c.allocN<float>((size_t)10 * n);
        if (mixed && !an.pc32) an.pc32 = c.allocN<float>((size_t)2 * n);
    }
    c.factor_clock.stop(c.stream);
    int fstat = 0;
    EQG_CUDA(cudaMemcpyAsync(c.pinned, an.factor_status->ptr, sizeof(int), cudaMemcpyDeviceToHost, c.stream));
    c.sync();
    std::memcpy(&fstat, c.pinned, sizeof(int));
    if (fstat) return res;  // zero pivot
    c.krylov_clock.start(c.stream);

    if (!refine) {
        res = bicgstab<double>(c, an, L0.as64->as<double>(), v, tol, max_iter, check_every, mixed);
        res.sweeps = 1;
    } else {
        Vecs<float> w = vecs<float>(an.vec32->as<float>(), n);
        const double inner_tol = c.param_d("linsolver_inner_tolerance", 1e-4);
        const int max_sweeps = c.param_i("linsolver_max_sweeps", 60);
        double* part = an.partials->as<double>();
        unsigned int* cnt = an.counter->as<unsigned int>();
        const int nb = blocksFor(n, kThreads, kRedBlocks);
        k_fill(c, v.x, 0.0, n);
        Buf rr_dev = c.allocN<double>(2);
        launch(c, "sumsq",
               [&] { sumsq_kernel<<<nb, kThreads, 0, c.stream>>>(v.b, n, part, cnt, rr_dev->as<double>()); });
        WITH_KMAX(L0.kmax, launch(c, "residual", [&] {
            residual_kernel<KK><<<nb, kThreads, 0, c.stream>>>(L0.view(), L0.as64->as<double>(), v.x, v.b, v.r, w.b, n,
                                                               part, cnt, rr_dev->as<double>() + 1);
        }));
        EQG_CUDA(cudaMemcpyAsync(c.pinned, rr_dev->ptr, 2 * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
        c.sync();
        const double bb = c.pinned[0];
        double rr = c.pinned[1];
        int total_iter = 0, sweeps = 0;
        bool conv = bb == 0.0 || rr <= tol * tol * bb;
        while (!conv && sweeps < max_sweeps && total_iter < max_iter) {
            SolveResult inner = bicgstab<float>(c, an, L0.as32->as<float>(), w, inner_tol, max_iter - total_iter,
                                                check_every);
            total_iter += inner.iterations;
            ++sweeps;
            launch(c, "add_float",
                   [&] { add_float_kernel<<<blocksFor(n), kThreads, 0, c.stream>>>(v.x, w.x, n); });
            WITH_KMAX(L0.kmax, launch(c, "residual", [&] {
                residual_kernel<KK><<<nb, kThreads, 0, c.stream>>>(L0.view(), L0.as64->as<double>(), v.x, v.b, v.r,
                                                                   w.b, n, part, cnt, rr_dev->as<double>() + 1);
            }));
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
    launch(c, "unpermute",
           [&] { unpermute_kernel<<<blocksFor(n), kThreads, 0, c.stream>>>(v.x, L0.perm->as<int>(), xout, n); });
    return res;
}

}  // namespace eqg

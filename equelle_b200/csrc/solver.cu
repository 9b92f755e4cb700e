// Linear solve J du = F for the Newton update (the reference calls
// Opm::LinearSolverFactory::solve from solveForUpdate,
// EquelleRuntimeCPU.cpp:413-440).
//
// Method: BiCGStab (van der Vorst 1992) right-preconditioned, from x = 0,
// converged when ||b - A x|| <= tol * ||b||, with a fixed pseudo-random
// shadow residual (shadow_entry).
//
// Block structure: Equelle's newtonSolveSystem stacks its unknowns as
// `ncomp` collections over all cells, so unknown comp * ncells + cell belongs
// to grid cell `cell`.  For ncomp = 2 or 3 the solver works on ncomp x ncomp
// blocks, one block row per cell (all unknowns of a cell together); with
// ncomp = 1, with the natural ordering, or when the unknowns do not cover
// every cell, the blocks are 1 x 1 (one block row per unknown).
//
// Preconditioner: block ILU(0) (Saad, Iterative Methods for Sparse Linear
// Systems, sec. 10.3, in its block form, as in OPM's BILU0), with the block
// rows reordered symmetrically so that each "stage" is a contiguous range of
// block rows with no couplings inside it:
//   - ordering "multicolor" (default): greedy colouring of the block graph;
//     the 7-point (5-point) cell graph takes two colours, so a sweep is two
//     stages;
//   - ordering "natural" (1 x 1 blocks): wavefront levels of the natural
//     order, which reproduces natural-order ILU(0), the oracle's
//     preconditioner, at the price of many stages.
// Factorization and both triangular sweeps run one kernel per stage, one
// thread per block row.  Rows of the first stage have no lower part (their
// forward-sweep value is the right-hand side itself) and rows of the last
// stage have no upper part (the forward sweep finishes them), so a sweep
// over S stages takes S kernels.
//
// Preconditioner "multigrid" (default; see the analysis section below):
// geometric-aggregation V-cycle with these block ILU(0) sweeps as smoothers,
// which keeps the iteration count of the elliptic pressure part from growing
// with the grid; "ilu0": the staged block ILU(0) alone.
//
// Precision "mixed": BiCGStab and every vector in FP64, the preconditioner's
// matrices (level matrices, block ILU(0) factors, coarsest inverse) stored
// in FP32: the V-cycle reads about half the bytes, in FP64 arithmetic.
// Precision "refine": the inner BiCGStab and the preconditioner in FP32,
// inside FP64 iterative refinement (r = b - A x in FP64 with FP64 A).
//
// Every kernel of an iteration reads a device-side status word first and
// returns at once after convergence or breakdown, so the host enqueues
// several iterations between convergence checks without a round trip.
#include "eqg_internal.cuh"

#include <algorithm>
#include <chrono>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <mutex>
#include <numeric>
#include <sstream>
#include <string>

#include <omp.h>

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

// Every kernel of a BiCGStab iteration calls this before it reads anything
// that an earlier kernel wrote (first thing, except for the fused coarse
// cycle's prefetches of constant data): those kernels are launched as
// programmatic dependent launches (launch_k), so their blocks may be
// scheduled while the kernel before them on the stream still runs; this
// waits until that kernel has completed and its writes are visible (at once
// when the kernel was launched normally).
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

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

// ---- block matrices -----------------------------------------------------------
// Level matrices are in a block sliced ELL layout: block rows in slices of
// 32 (one warp), each slice stored by position k in the row and padded to
// its longest row.  Slot q = slice_ptr[R / 32] + 32 k + R % 32 holds the
// block column col[q] of the k-th block of block row R, and the B x B values
// of that block (row-major, e = i B + j) are contiguous at q B^2 + e: a 2 x 2
// block is one 128-bit load in FP32 (two in FP64), and a warp's loads at
// position k are one contiguous segment.  Within a row, blocks are in
// ascending column order, so the ILU(0) lower part is k < dk[R] and the
// upper part k > dk[R].  Vectors are in block-row order: unknown c of block
// row R is at R B + c.  A level whose slices all have the same width (the
// small levels of the fused coarse cycle) also records that width: there the
// slot of (R, k) is known without a load, and the kernels read a row's
// columns and values in the same round trip as its length and diagonal
// position.  Padding slots hold a valid column (the row itself) and zero
// values.
struct SellView {
    const int* __restrict__ slice_ptr;  // first slot of each slice
    const int* __restrict__ col;        // block column of each slot
    const int* __restrict__ len;        // blocks of each block row
    const int* __restrict__ dk;         // position of the diagonal block in each row
    int width;                          // slots per row of every slice (0: slices differ)
};

// First slot of the slice of block row R; with U the level's slices all have
// m.width slots per row.
template <bool U>
__device__ __forceinline__ int slice_base(const SellView& m, int R)
{
    return U ? (R >> 5) * (m.width << 5) : m.slice_ptr[R >> 5];
}

// Block J of a vector.  With CG the loads bypass L1 (ld.global.cg): for
// vectors that other thread blocks of the same kernel wrote.
template <int B, class T, bool CG = false>
__device__ __forceinline__ void load_bvec(const T* __restrict__ x, int J, double (&v)[B])
{
    if constexpr (B == 2 && sizeof(T) == 8) {
        const double2* p = reinterpret_cast<const double2*>(x) + J;
        const double2 t = CG ? __ldcg(p) : *p;
        v[0] = t.x;
        v[1] = t.y;
    } else if constexpr (B == 2 && sizeof(T) == 4) {
        const float2* p = reinterpret_cast<const float2*>(x) + J;
        const float2 t = CG ? __ldcg(p) : *p;
        v[0] = (double)t.x;
        v[1] = (double)t.y;
    } else {
#pragma unroll
        for (int c = 0; c < B; ++c) v[c] = (double)(CG ? __ldcg(x + J * B + c) : x[J * B + c]);
    }
}

template <int B, class T>
__device__ __forceinline__ void store_bvec(T* __restrict__ x, int R, const double (&v)[B])
{
#pragma unroll
    for (int c = 0; c < B; ++c) x[R * B + c] = (T)v[c];
}

// The BB values of one block (contiguous; 16-byte aligned when BB = 4).
template <int BB, class M>
__device__ __forceinline__ void load_block(const M* __restrict__ p, M (&v)[BB])
{
    if constexpr (BB == 4 && sizeof(M) == 4) {
        const float4 t = *reinterpret_cast<const float4*>(p);
        v[0] = t.x;
        v[1] = t.y;
        v[2] = t.z;
        v[3] = t.w;
    } else if constexpr (BB == 4 && sizeof(M) == 8) {
        const double2 t0 = reinterpret_cast<const double2*>(p)[0];
        const double2 t1 = reinterpret_cast<const double2*>(p)[1];
        v[0] = t0.x;
        v[1] = t0.y;
        v[2] = t1.x;
        v[3] = t1.y;
    } else {
#pragma unroll
        for (int e = 0; e < BB; ++e) v[e] = p[e];
    }
}

// acc += sum_{k0 <= k < k1} A_{R,k} x_{col(R,k)}, blocks in ascending k and
// within a block in ascending j.  x_J is read from `x` when J < split and
// from `x2` otherwise.  With KM > 0 (rows of at most KM blocks) the loop is
// unrolled so that a thread issues its column loads before the dependent
// gathers of x: the kernels using it are bound by the latency of that chain.
//
// With U (slices of uniform width) the column and value loads cover every
// slot k < m.width, so they do not wait for k0 and k1 (the row's diagonal
// position or length); only the sums skip the slots outside [k0, k1).
template <int B, int KM, class T, class M, bool CG = false, bool U = false>
__device__ __forceinline__ void bdot(const SellView& m, int sbase, int lane, int k0, int k1, const M* __restrict__ a,
                                     const T* __restrict__ x, const T* __restrict__ x2, int split, double (&acc)[B])
{
    constexpr int BB = B * B;
    if constexpr (KM == 0) {
        for (int k = k0; k < k1; ++k) {
            const int q = sbase + (k << 5);
            const int J = m.col[q + lane];
            double xv[B];
            load_bvec<B, T, CG>(J < split ? x : x2, J, xv);
            M av[BB];
            load_block<BB, M>(a + (size_t)(q + lane) * BB, av);
#pragma unroll
            for (int i = 0; i < B; ++i)
#pragma unroll
                for (int j = 0; j < B; ++j) acc[i] += (double)av[i * B + j] * xv[j];
        }
    } else if constexpr (KM * BB <= 32) {
        // columns and values of the whole row first (predicated loads), then
        // the gathers of x
        int ci[KM];
        M av[KM][BB];
#pragma unroll
        for (int k = 0; k < KM; ++k) {
            const bool ld = U ? k < m.width : (k >= k0 && k < k1);
            const int q = sbase + (k << 5);
            ci[k] = ld ? m.col[q + lane] : 0;
#pragma unroll
            for (int e = 0; e < BB; ++e) av[k][e] = (M)0;
            if (ld) load_block<BB, M>(a + (size_t)(q + lane) * BB, av[k]);
        }
#pragma unroll
        for (int k = 0; k < KM; ++k) {
            if (k >= k0 && k < k1) {
                double xv[B];
                load_bvec<B, T, CG>(ci[k] < split ? x : x2, ci[k], xv);
#pragma unroll
                for (int i = 0; i < B; ++i)
#pragma unroll
                    for (int j = 0; j < B; ++j) acc[i] += (double)av[k][i * B + j] * xv[j];
            }
        }
    } else {
        int ci[KM];
#pragma unroll
        for (int k = 0; k < KM; ++k)
            ci[k] = (U ? k < m.width : (k >= k0 && k < k1)) ? m.col[sbase + (k << 5) + lane] : 0;
#pragma unroll
        for (int k = 0; k < KM; ++k) {
            if (k >= k0 && k < k1) {
                const int q = sbase + (k << 5);
                double xv[B];
                load_bvec<B, T, CG>(ci[k] < split ? x : x2, ci[k], xv);
                M av[BB];
                load_block<BB, M>(a + (size_t)(q + lane) * BB, av);
#pragma unroll
                for (int i = 0; i < B; ++i)
#pragma unroll
                    for (int j = 0; j < B; ++j) acc[i] += (double)av[i * B + j] * xv[j];
            }
        }
    }
}

// y = D x for the block at slot position `q` (its first value at
// a[q B^2 + lane], values 32 apart).
template <int B, class M>
__device__ __forceinline__ void bmatvec(const M* __restrict__ a, int q, int lane, const double (&x)[B], double (&y)[B])
{
    M av[B * B];
    load_block<B * B, M>(a + (size_t)(q + lane) * (B * B), av);
#pragma unroll
    for (int i = 0; i < B; ++i) {
        double s = 0.0;
#pragma unroll
        for (int j = 0; j < B; ++j) s += (double)av[i * B + j] * x[j];
        y[i] = s;
    }
}

// In-place inverse of a B x B block by Gauss-Jordan elimination with
// partial pivoting; false when a pivot is zero or not finite.
template <int B>
__device__ __forceinline__ bool invert_block(double (&a)[B * B])
{
    double v[B * B];
#pragma unroll
    for (int i = 0; i < B; ++i)
#pragma unroll
        for (int j = 0; j < B; ++j) v[i * B + j] = i == j ? 1.0 : 0.0;
#pragma unroll
    for (int c = 0; c < B; ++c) {
        int p = c;
        double best = fabs(a[c * B + c]);
#pragma unroll
        for (int r = c + 1; r < B; ++r)
            if (fabs(a[r * B + c]) > best) {
                best = fabs(a[r * B + c]);
                p = r;
            }
        if (!(best > 0.0) || !isfinite(best)) return false;
#pragma unroll
        for (int r = c + 1; r < B; ++r)
            if (r == p)
#pragma unroll
                for (int j = 0; j < B; ++j) {
                    const double t = a[c * B + j];
                    a[c * B + j] = a[r * B + j];
                    a[r * B + j] = t;
                    const double u = v[c * B + j];
                    v[c * B + j] = v[r * B + j];
                    v[r * B + j] = u;
                }
        const double piv = a[c * B + c];
#pragma unroll
        for (int j = 0; j < B; ++j) {
            a[c * B + j] /= piv;
            v[c * B + j] /= piv;
        }
#pragma unroll
        for (int r = 0; r < B; ++r)
            if (r != c) {
                const double f = a[r * B + c];
#pragma unroll
                for (int j = 0; j < B; ++j) {
                    a[r * B + j] -= f * a[c * B + j];
                    v[r * B + j] -= f * v[c * B + j];
                }
            }
    }
#pragma unroll
    for (int e = 0; e < B * B; ++e) a[e] = v[e];
    return true;
}

// Dispatches on a level's longest block row as KK (8, 16; 0 = plain loop).
#define WITH_KMAX(kmax, ...)                        \
    if ((kmax) <= 8) {                              \
        constexpr int KK = 8;                       \
        __VA_ARGS__;                                \
    } else if ((kmax) <= 16) {                      \
        constexpr int KK = 16;                      \
        __VA_ARGS__;                                \
    } else {                                        \
        constexpr int KK = 0;                       \
        __VA_ARGS__;                                \
    }

// Dispatches on the block size as BS (1, 2, 3).
#define WITH_BS(bs, ...)                            \
    if ((bs) == 1) {                                \
        constexpr int BS = 1;                       \
        __VA_ARGS__;                                \
    } else if ((bs) == 2) {                         \
        constexpr int BS = 2;                       \
        __VA_ARGS__;                                \
    } else {                                        \
        constexpr int BS = 3;                       \
        __VA_ARGS__;                                \
    }

// dst[p] = src[map[p]], or 0 where map[p] < 0 (padding, or an entry of a
// block that the Jacobian does not have).
__global__ void gather_values_kernel(const double* __restrict__ src, const int* __restrict__ map,
                                     double* __restrict__ dst, int64_t size)
{
    GRID_STRIDE(p, size)
    {
        const int e = map[p];
        dst[p] = e >= 0 ? src[e] : 0.0;
    }
}

// The same gather, one block row per thread over its slots: a thread's
// loads stay in the few Jacobian rows of its block row (the unknowns of one
// cell), which L1 then serves, and a warp's stores at one slot position are
// one contiguous segment.
template <int BB>
__global__ void gather_rows_kernel(int nb, const int* __restrict__ slice_ptr, const double* __restrict__ src,
                                   const int* __restrict__ map, double* __restrict__ dst)
{
    // every lane of the last slice, also past the last row (its slots are
    // padding: zero)
    GRID_STRIDE(r, ((int64_t)nb + 31) & ~(int64_t)31)
    {
        const int R = (int)r, lane = R & 31;
        const int s0 = slice_ptr[R >> 5], width = (slice_ptr[(R >> 5) + 1] - s0) >> 5;
        for (int k = 0; k < width; ++k) {
            const int64_t q = (int64_t)(s0 + (k << 5) + lane) * BB;
#pragma unroll
            for (int e = 0; e < BB; ++e) {
                const int j = map[q + e];
                dst[q + e] = j >= 0 ? src[j] : 0.0;
            }
        }
    }
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

// Block ILU(0) of the block rows [r0, r1) of one stage, in place in `lu`
// (the block values of the matrix on entry).  For each lower block (R, K),
// in ascending K: L_RK = A_RK D_K^{-1}, then A_RJ -= L_RK U_KJ for every
// upper block (K, J) of row K whose position (R, J) is in row R's pattern.
// The diagonal block is stored inverted (D_R^{-1}); rows of earlier stages
// are finished.  A singular diagonal block sets *status.
template <int B>
__global__ void bilu_factor_stage_kernel(int r0, int r1, SellView m, double* lu, int* status)
{
    constexpr int BB = B * B;
    for (int64_t rr = r0 + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; rr < r1;
         rr += (int64_t)gridDim.x * blockDim.x) {
        const int R = (int)rr;
        const int lane = R & 31, sb = m.slice_ptr[R >> 5], len = m.len[R], d = m.dk[R];
        auto at = [&](int sbase, int ln, int k, int e) -> double& {
            return lu[(size_t)(sbase + (k << 5) + ln) * BB + e];
        };
        for (int k = 0; k < d; ++k) {
            const int K = m.col[sb + (k << 5) + lane];
            const int lk = K & 31, sk = m.slice_ptr[K >> 5], lenk = m.len[K], dkk = m.dk[K];
            double l[BB];
#pragma unroll
            for (int i = 0; i < B; ++i)
#pragma unroll
                for (int j = 0; j < B; ++j) {
                    double s = 0.0;
#pragma unroll
                    for (int t = 0; t < B; ++t) s += at(sb, lane, k, i * B + t) * at(sk, lk, dkk, t * B + j);
                    l[i * B + j] = s;
                }
#pragma unroll
            for (int e = 0; e < BB; ++e) at(sb, lane, k, e) = l[e];
            int p = k + 1;
            for (int kk = dkk + 1; kk < lenk; ++kk) {
                const int J = m.col[sk + (kk << 5) + lk];
                while (p < len && m.col[sb + (p << 5) + lane] < J) ++p;
                if (p < len && m.col[sb + (p << 5) + lane] == J) {
#pragma unroll
                    for (int i = 0; i < B; ++i)
#pragma unroll
                        for (int j = 0; j < B; ++j) {
                            double s = 0.0;
#pragma unroll
                            for (int t = 0; t < B; ++t) s += l[i * B + t] * at(sk, lk, kk, t * B + j);
                            at(sb, lane, p, i * B + j) -= s;
                        }
                }
            }
        }
        double dg[BB];
#pragma unroll
        for (int e = 0; e < BB; ++e) dg[e] = at(sb, lane, d, e);
        if (!invert_block<B>(dg)) *status = 1;
#pragma unroll
        for (int e = 0; e < BB; ++e) at(sb, lane, d, e) = dg[e];
    }
}

__device__ __forceinline__ bool mg_skip(const KScal* sc, int skip_if_s)
{
    return stopped(sc) || (skip_if_s && sc->s_conv);
}

// zadd_R += z
template <int B, class T, bool CG = false>
__device__ __forceinline__ void update_z(T* __restrict__ zadd, int R, const double (&z)[B])
{
    double w[B];
    load_bvec<B, T, CG>(zadd, R, w);
#pragma unroll
    for (int c = 0; c < B; ++c) w[c] += z[c];
    store_bvec<B, T>(zadd, R, w);
}

// The multigrid steps below are written as loops over a row range for
// thread `tid` of `nth`, shared by the one-step kernels (CG = false) and by
// the fused coarse cycle (mg_tail_kernel, CG = true), so that both compute
// every element with the same operations.

// Forward sweep of stage [r0, r1), a stage after the first:
//   y_R = b_R - sum_{k < dk} L_Rk y_K,
// with y_K = b_K for rows of the first stage (K < r_first) and out_K
// otherwise.  The last stage has no upper part: there the row is finished,
// out_R = D_R^{-1} y_R (and zadd_R += out_R when zadd is given).
template <int B, int KM, class T, class M, bool CG, bool U = false>
__device__ __forceinline__ void lower_rows(int r0, int r1, int r_first, int last, const SellView& m,
                                           const M* __restrict__ lu, const T* __restrict__ b, T* __restrict__ out,
                                           T* __restrict__ zadd, int tid, int nth)
{
    for (int R = r0 + tid; R < r1; R += nth) {
        const int lane = R & 31, sb = slice_base<U>(m, R), d = m.dk[R];
        double acc[B];
#pragma unroll
        for (int c = 0; c < B; ++c) acc[c] = 0.0;
        bdot<B, KM, T, M, CG, U>(m, sb, lane, 0, d, lu, b, out, r_first, acc);
        double y[B];
        load_bvec<B, T, CG>(b, R, y);
#pragma unroll
        for (int c = 0; c < B; ++c) y[c] = (double)(T)(y[c] - acc[c]);
        if (last) {
            double z[B];
            bmatvec<B, M>(lu, sb + (d << 5), lane, y, z);
#pragma unroll
            for (int c = 0; c < B; ++c) z[c] = (double)(T)z[c];
            store_bvec<B, T>(out, R, z);
            if (zadd) update_z<B, T, CG>(zadd, R, z);
        } else {
            store_bvec<B, T>(out, R, y);
        }
    }
}

// Backward sweep of stage [r0, r1), a stage before the last:
//   out_R = D_R^{-1} (y_R - sum_{k > dk} U_Rk out_K),
// with y_R = b_R in the first stage and the forward-sweep value out_R
// otherwise; zadd_R += out_R when zadd is given.
template <int B, int KM, class T, class M, bool CG, bool U = false>
__device__ __forceinline__ void upper_rows(int r0, int r1, int first, const SellView& m, const M* __restrict__ lu,
                                           const T* __restrict__ b, T* __restrict__ out, T* __restrict__ zadd,
                                           int tid, int nth)
{
    for (int R = r0 + tid; R < r1; R += nth) {
        const int lane = R & 31, sb = slice_base<U>(m, R), d = m.dk[R];
        double acc[B];
#pragma unroll
        for (int c = 0; c < B; ++c) acc[c] = 0.0;
        bdot<B, KM, T, M, CG, U>(m, sb, lane, d + 1, m.len[R], lu, out, out, INT_MAX, acc);
        double y[B];
        load_bvec<B, T, CG>(first ? b : out, R, y);
#pragma unroll
        for (int c = 0; c < B; ++c) y[c] -= acc[c];
        double z[B];
        bmatvec<B, M>(lu, sb + (d << 5), lane, y, z);
#pragma unroll
        for (int c = 0; c < B; ++c) z[c] = (double)(T)z[c];
        store_bvec<B, T>(out, R, z);
        if (zadd) update_z<B, T, CG>(zadd, R, z);
    }
}

// out = b - A x.  Block rows below r_zero are not computed: after a full
// ILU(0) sweep their residual is zero (see vcycle).  With ZW they get 0;
// without, they are left as they are, for readers that skip them.
template <int B, int KM, class T, class M, bool CG, bool U = false, bool ZW = true>
__device__ __forceinline__ void residual_rows(int nb, int r_zero, const SellView& m, const M* __restrict__ a,
                                              const T* __restrict__ x, const T* __restrict__ b, T* __restrict__ out,
                                              int tid, int nth)
{
    for (int R = tid; R < nb; R += nth) {
        if (R < r_zero) {
            if (ZW)
#pragma unroll
                for (int c = 0; c < B; ++c) out[R * B + c] = (T)0;
            continue;
        }
        double acc[B];
#pragma unroll
        for (int c = 0; c < B; ++c) acc[c] = 0.0;
        bdot<B, KM, T, M, CG, U>(m, slice_base<U>(m, R), R & 31, 0, m.len[R], a, x, x, INT_MAX, acc);
        double y[B];
        load_bvec<B, T, CG>(b, R, y);
#pragma unroll
        for (int c = 0; c < B; ++c) y[c] -= acc[c];
        store_bvec<B, T>(out, R, y);
    }
}

// rc[P] = sum of t over the members of aggregate P, in member order.  An
// aggregate of at most kMembers members (2 x 2 x 2 cells) issues all its
// index loads, then all its gathers, before the sum: the step is bound by the
// latency of that chain, not by its bytes.
constexpr int kMembers = 8;

// Members below t_zero (positions whose t is zero and was not written, see
// residual_rows) are skipped: the same sums as adding their zeros.
template <class T, bool CG>
__device__ __forceinline__ void restrict_rows(int nc, const int* __restrict__ mptr, const int* __restrict__ midx,
                                              const T* __restrict__ t, int t_zero, T* __restrict__ rc, int tid,
                                              int nth)
{
    for (int P = tid; P < nc; P += nth) {
        double s = 0.0;
        const int k0 = mptr[P], k1 = mptr[P + 1];
        if (k1 - k0 <= kMembers) {
            int mi[kMembers];
#pragma unroll
            for (int j = 0; j < kMembers; ++j) mi[j] = k0 + j < k1 ? midx[k0 + j] : -1;
            double tv[kMembers];
#pragma unroll
            for (int j = 0; j < kMembers; ++j)
                tv[j] = mi[j] >= t_zero ? (double)(CG ? __ldcg(t + mi[j]) : t[mi[j]]) : 0.0;
#pragma unroll
            for (int j = 0; j < kMembers; ++j)
                if (mi[j] >= t_zero) s += tv[j];
        } else {
            for (int k = k0; k < k1; ++k)
                if (midx[k] >= t_zero) s += (double)(CG ? __ldcg(t + midx[k]) : t[midx[k]]);
        }
        rc[P] = (T)s;
    }
}

// restrict_rows with the members of each aggregate at P kMembers + j
// (-1 past the last): the member loads need no offsets first.  Same sums.
template <class T, bool CG>
__device__ __forceinline__ void restrict_padded_rows(int nc, const int* __restrict__ mpad, const T* __restrict__ t,
                                                     T* __restrict__ rc, int tid, int nth)
{
    for (int P = tid; P < nc; P += nth) {
        int mi[kMembers];
#pragma unroll
        for (int j = 0; j < kMembers; ++j) mi[j] = mpad[P * kMembers + j];
        double tv[kMembers];
#pragma unroll
        for (int j = 0; j < kMembers; ++j) tv[j] = mi[j] >= 0 ? (double)(CG ? __ldcg(t + mi[j]) : t[mi[j]]) : 0.0;
        double s = 0.0;
#pragma unroll
        for (int j = 0; j < kMembers; ++j)
            if (mi[j] >= 0) s += tv[j];
        rc[P] = (T)s;
    }
}

// z_R += alpha zc_{aggb[R]} (piecewise-constant prolongation, per block
// row, scaled by the over-correction factor alpha).  Piecewise-constant
// interpolation from aggregates underestimates the smooth error it
// corrects.  Measured on the two-phase cases, BiCGStab iterations per time
// step: 2 x 2 x 2 aggregates (128 x 128 x 64) 121 at 1.0, 97 at 1.25 to
// 1.45, 104 at 1.6, 127 at 1.9; 2 x 2 aggregates (512 x 512) 92 at 1.0, 49
// at 1.3, 29 at 1.6, 24 at 1.8, 22 at 2.0, 27 at 2.2.
constexpr double kMgAlpha3d = 1.4;
constexpr double kMgAlpha2d = 1.9;
template <int B, class T, bool CG>
__device__ __forceinline__ void prolong_rows(int nb, const int* __restrict__ aggb, const T* __restrict__ zc,
                                             T* __restrict__ z, double alpha, int tid, int nth)
{
    for (int R = tid; R < nb; R += nth) {
        double e[B];
        load_bvec<B, T, CG>(zc, aggb[R], e);
#pragma unroll
        for (int c = 0; c < B; ++c) e[c] *= alpha;
        update_z<B, T, CG>(z, R, e);
    }
}

// z = inv r with the dense inverse of the coarsest level: one warp per row,
// lane l summing columns l, l + 32, ... in order, then a butterfly over the
// warp (every lane ends with the same sum).  tid and nth are multiples of 32
// apart from the lane, so every lane of a warp takes the same rows.
template <class T, class M, bool CG>
__device__ __forceinline__ void dense_rows(int n, const M* __restrict__ inv, const T* __restrict__ r,
                                           T* __restrict__ z, int tid, int nth)
{
    const int lane = tid & 31;
    for (int i = tid >> 5; i < n; i += nth >> 5) {
        double s = 0.0;
        for (int j = lane; j < n; j += 32) s += (double)inv[i * n + j] * (double)(CG ? __ldcg(r + j) : r[j]);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) z[i] = (T)s;
    }
}

#define THREAD_RANGE                                                 \
    const int tid = (int)(blockIdx.x * blockDim.x + threadIdx.x); \
    const int nth = (int)(gridDim.x * blockDim.x)

template <int B, int KM, class T, class M>
__global__ void bilu_lower_kernel(int r0, int r1, int r_first, int last, SellView m, const M* __restrict__ lu,
                                  const T* __restrict__ b, T* __restrict__ out, T* __restrict__ zadd,
                                  const KScal* sc, int skip_if_s)
{
    pdl_wait();
    if (mg_skip(sc, skip_if_s)) return;
    THREAD_RANGE;
    lower_rows<B, KM, T, M, false>(r0, r1, r_first, last, m, lu, b, out, zadd, tid, nth);
}

template <int B, int KM, class T, class M>
__global__ void bilu_upper_kernel(int r0, int r1, int first, SellView m, const M* __restrict__ lu,
                                  const T* __restrict__ b, T* __restrict__ out, T* __restrict__ zadd,
                                  const KScal* sc, int skip_if_s)
{
    pdl_wait();
    if (mg_skip(sc, skip_if_s)) return;
    THREAD_RANGE;
    upper_rows<B, KM, T, M, false>(r0, r1, first, m, lu, b, out, zadd, tid, nth);
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

// The BiCGStab vectors in 16-byte chunks (two doubles or four floats); each
// vector starts on a 16-byte boundary (vec_stride), the elements past the
// last whole chunk are done one by one.
template <class T>
struct Chunk;
template <>
struct Chunk<double> {
    using V = double2;
    static constexpr int W = 2;
};
template <>
struct Chunk<float> {
    using V = float4;
    static constexpr int W = 4;
};

template <class T>
__device__ __forceinline__ void load_chunk(const T* __restrict__ p, int64_t c, double (&v)[Chunk<T>::W])
{
    const typename Chunk<T>::V t = reinterpret_cast<const typename Chunk<T>::V*>(p)[c];
    if constexpr (Chunk<T>::W == 2) {
        v[0] = t.x;
        v[1] = t.y;
    } else {
        v[0] = t.x;
        v[1] = t.y;
        v[2] = t.z;
        v[3] = t.w;
    }
}

template <class T>
__device__ __forceinline__ void store_chunk(T* __restrict__ p, int64_t c, const T (&v)[Chunk<T>::W])
{
    typename Chunk<T>::V t;
    if constexpr (Chunk<T>::W == 2) {
        t.x = v[0];
        t.y = v[1];
    } else {
        t.x = v[0];
        t.y = v[1];
        t.z = v[2];
        t.w = v[3];
    }
    reinterpret_cast<typename Chunk<T>::V*>(p)[c] = t;
}

// Elements between the starts of two BiCGStab vectors: a multiple of 4, so
// that every vector of a buffer from allocN starts on a 16-byte boundary.
inline size_t vec_stride(int n) { return ((size_t)(n > 0 ? n : 1) + 3) & ~(size_t)3; }

// Chunks c of n elements for this thread, then the remaining elements i.
#define CHUNK_STRIDE(c, n, W) GRID_STRIDE(c, (int64_t)(n) / (W))
#define REST_STRIDE(i, n, W)                                                                                  \
    for (int64_t i = (int64_t)(n) / (W) * (W) + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < (n); \
         i += (int64_t)gridDim.x * blockDim.x)

template <class T>
__global__ void bicg_p_kernel(const T* __restrict__ r, const T* __restrict__ v, T* __restrict__ p, int n,
                              const KScal* sc)
{
    pdl_wait();
    if (stopped(sc)) return;
    const double beta = (sc->rho_new / sc->rho) * (sc->alpha / sc->omega);
    const double omega = sc->omega;
    constexpr int W = Chunk<T>::W;
    CHUNK_STRIDE(c, n, W)
    {
        double rv[W], pv[W], vv[W];
        load_chunk<T>(r, c, rv);
        load_chunk<T>(p, c, pv);
        load_chunk<T>(v, c, vv);
        T o[W];
#pragma unroll
        for (int j = 0; j < W; ++j) o[j] = (T)(rv[j] + beta * (pv[j] - omega * vv[j]));
        store_chunk<T>(p, c, o);
    }
    REST_STRIDE(i, n, W) p[i] = (T)((double)r[i] + beta * ((double)p[i] - omega * (double)v[i]));
}

// The SpMV kernels are latency bound; for the FP64 layouts with blocks of
// at most 2 x 2 and rows of at most 8 blocks their launch bounds trade the
// reduction's registers for resident warps (8 and 6 blocks of 256 per SM,
// without spills); the other instantiations keep the compiler's choice.
template <int B, int KM, class T>
constexpr int spmv_min_blocks(int hot)
{
    return (B <= 2 && KM == 8 && sizeof(T) == sizeof(double)) ? hot : 1;
}

// v = A ph ; alpha = rho_new / (rhat . v)
template <int B, int KM, class T>
__global__ void __launch_bounds__(kThreads, spmv_min_blocks<B, KM, T>(8)) bicg_spmv_alpha_kernel(SellView m, const T* __restrict__ a, const T* __restrict__ ph,
                                       const T* __restrict__ rhat, T* __restrict__ v, int nb, double* partials,
                                       unsigned int* counter, KScal* sc)
{
    pdl_wait();
    if (stopped(sc)) return;
    double d[1] = {0.0};
    GRID_STRIDE(rr, nb)
    {
        const int R = (int)rr;
        double acc[B];
#pragma unroll
        for (int c = 0; c < B; ++c) acc[c] = 0.0;
        bdot<B, KM, T, T>(m, m.slice_ptr[R >> 5], R & 31, 0, m.len[R], a, ph, ph, INT_MAX, acc);
        double h[B];
        load_bvec<B, T>(rhat, R, h);
#pragma unroll
        for (int c = 0; c < B; ++c) {
            const T vi = (T)acc[c];
            v[R * B + c] = vi;
            d[0] += h[c] * (double)vi;
        }
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
    pdl_wait();
    if (stopped(sc)) return;
    const double alpha = sc->alpha;
    double d[1] = {0.0};
    constexpr int W = Chunk<T>::W;
    CHUNK_STRIDE(c, n, W)
    {
        double rv[W], vv[W];
        load_chunk<T>(r, c, rv);
        load_chunk<T>(v, c, vv);
        T o[W];
#pragma unroll
        for (int j = 0; j < W; ++j) {
            o[j] = (T)(rv[j] - alpha * vv[j]);
            d[0] += (double)o[j] * (double)o[j];
        }
        store_chunk<T>(s, c, o);
    }
    REST_STRIDE(i, n, W)
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
template <int B, int KM, class T>
__global__ void __launch_bounds__(kThreads, spmv_min_blocks<B, KM, T>(6)) bicg_spmv_omega_kernel(SellView m, const T* __restrict__ a, const T* __restrict__ sh,
                                       const T* __restrict__ s, T* __restrict__ t, int nb, double* partials,
                                       unsigned int* counter, KScal* sc)
{
    pdl_wait();
    if (stopped(sc) || sc->s_conv) return;
    double d[2] = {0.0, 0.0};
    GRID_STRIDE(rr, nb)
    {
        const int R = (int)rr;
        double acc[B];
#pragma unroll
        for (int c = 0; c < B; ++c) acc[c] = 0.0;
        bdot<B, KM, T, T>(m, m.slice_ptr[R >> 5], R & 31, 0, m.len[R], a, sh, sh, INT_MAX, acc);
        double sv[B];
        load_bvec<B, T>(s, R, sv);
#pragma unroll
        for (int c = 0; c < B; ++c) {
            const T ti = (T)acc[c];
            t[R * B + c] = ti;
            d[0] += (double)ti * sv[c];
            d[1] += (double)ti * (double)ti;
        }
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
    pdl_wait();
    if (stopped(sc)) return;
    const double alpha = sc->alpha;
    const int half = sc->s_conv;
    const double omega = half ? 0.0 : sc->omega;
    double d[2] = {0.0, 0.0};
    constexpr int W = Chunk<T>::W;
    if (half) {
        CHUNK_STRIDE(c, n, W)
        {
            double xv[W], pv[W];
            load_chunk<T>(x, c, xv);
            load_chunk<T>(ph, c, pv);
            T o[W];
#pragma unroll
            for (int j = 0; j < W; ++j) o[j] = (T)(xv[j] + alpha * pv[j]);
            store_chunk<T>(x, c, o);
        }
        REST_STRIDE(i, n, W) x[i] = (T)((double)x[i] + alpha * (double)ph[i]);
    } else {
        CHUNK_STRIDE(c, n, W)
        {
            double xv[W], pv[W], shv[W], sv[W], tv[W], hv[W];
            load_chunk<T>(x, c, xv);
            load_chunk<T>(ph, c, pv);
            load_chunk<T>(sh, c, shv);
            load_chunk<T>(s, c, sv);
            load_chunk<T>(t, c, tv);
            load_chunk<T>(rhat, c, hv);
            T xo[W], ro[W];
#pragma unroll
            for (int j = 0; j < W; ++j) {
                xo[j] = (T)(xv[j] + alpha * pv[j] + omega * shv[j]);
                ro[j] = (T)(sv[j] - omega * tv[j]);
                d[0] += (double)ro[j] * (double)ro[j];
                d[1] += hv[j] * (double)ro[j];
            }
            store_chunk<T>(x, c, xo);
            store_chunk<T>(r, c, ro);
        }
        REST_STRIDE(i, n, W)
        {
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
template <int B, int KM>
__global__ void residual_kernel(SellView m, const double* __restrict__ a, const double* __restrict__ x,
                                const double* __restrict__ b, double* __restrict__ r, float* __restrict__ r32, int nb,
                                double* partials, unsigned int* counter, double* out_rr)
{
    double d[1] = {0.0};
    GRID_STRIDE(rr, nb)
    {
        const int R = (int)rr;
        double acc[B];
#pragma unroll
        for (int c = 0; c < B; ++c) acc[c] = 0.0;
        bdot<B, KM, double, double>(m, m.slice_ptr[R >> 5], R & 31, 0, m.len[R], a, x, x, INT_MAX, acc);
#pragma unroll
        for (int c = 0; c < B; ++c) {
            const double ri = b[R * B + c] - acc[c];
            r[R * B + c] = ri;
            r32[R * B + c] = (float)ri;
            d[0] += ri * ri;
        }
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
// Coarse-level values: each entry of the coarse pattern is the sum of the
// finer level's values that aggregate onto it (Galerkin product R A R^T with
// a 0/1 aggregation R), gathered in ascending fine-entry order, and stored
// at its value position gpos[c] (the other positions, padding and entries a
// block does not have, are zeroed beforehand).
__global__ void galerkin_kernel(int64_t nnz_c, const int* __restrict__ gptr, const int* __restrict__ gidx,
                                const int* __restrict__ gpos, const double* __restrict__ fine,
                                double* __restrict__ coarse)
{
    GRID_STRIDE(c, nnz_c)
    {
        double s = 0.0;
        const int k1 = gptr[c + 1];
        for (int k = gptr[c]; k < k1; ++k) s += fine[gidx[k]];
        coarse[gpos[c]] = s;
    }
}

template <int B, int KM, class T, class M>
__global__ void mg_residual_kernel(int nb, int r_zero, SellView m, const M* __restrict__ a, const T* __restrict__ x,
                                   const T* __restrict__ b, T* __restrict__ out, const KScal* sc, int skip_if_s)
{
    pdl_wait();
    if (mg_skip(sc, skip_if_s)) return;
    THREAD_RANGE;
    residual_rows<B, KM, T, M, false, false, false>(nb, r_zero, m, a, x, b, out, tid, nth);
}

template <class T>
__global__ void mg_restrict_kernel(int nc, const int* __restrict__ mptr, const int* __restrict__ midx,
                                   const T* __restrict__ t, int t_zero, T* __restrict__ rc, const KScal* sc,
                                   int skip_if_s)
{
    pdl_wait();
    if (mg_skip(sc, skip_if_s)) return;
    THREAD_RANGE;
    restrict_rows<T, false>(nc, mptr, midx, t, t_zero, rc, tid, nth);
}

template <int B, class T>
__global__ void mg_prolong_kernel(int nb, const int* __restrict__ aggb, const T* __restrict__ zc, T* __restrict__ z,
                                  double alpha, const KScal* sc, int skip_if_s)
{
    pdl_wait();
    if (mg_skip(sc, skip_if_s)) return;
    THREAD_RANGE;
    prolong_rows<B, T, false>(nb, aggb, zc, z, alpha, tid, nth);
}

// The coarse correction of a level that stores A P (A times the
// piecewise-constant prolongation; blocks of each fine block row summed per
// coarse block column, about 4 per row against 7 in A).  With t = r - A z
// left by the down-leg:
//   t -= alpha (A P) zc   (= r - A (z + alpha P zc), by linearity; the
//                          rows below r_zero of t are zero, not stored)
//   z += alpha P zc       (as prolong_rows)
// one pass over A P instead of the prolongation and a pass over A.
template <int B, int KM, class T, class M>
__global__ void mg_correct_kernel(int nb, int r_zero, SellView ap, const M* __restrict__ apv,
                                  const int* __restrict__ aggb, const T* __restrict__ zc, T* __restrict__ z,
                                  T* __restrict__ t, double alpha, const KScal* sc, int skip_if_s)
{
    pdl_wait();
    if (mg_skip(sc, skip_if_s)) return;
    THREAD_RANGE;
    for (int R = tid; R < nb; R += nth) {
        double acc[B];
#pragma unroll
        for (int c = 0; c < B; ++c) acc[c] = 0.0;
        bdot<B, KM, T, M>(ap, ap.slice_ptr[R >> 5], R & 31, 0, ap.len[R], apv, zc, zc, INT_MAX, acc);
        double tv[B];
        if (R < r_zero) {  // zero, not stored (residual_rows without ZW)
#pragma unroll
            for (int c = 0; c < B; ++c) tv[c] = 0.0;
        } else {
            load_bvec<B, T>(t, R, tv);
        }
#pragma unroll
        for (int c = 0; c < B; ++c) tv[c] -= alpha * acc[c];
        store_bvec<B, T>(t, R, tv);
        double e[B];
        load_bvec<B, T>(zc, aggb[R], e);
#pragma unroll
        for (int c = 0; c < B; ++c) e[c] *= alpha;
        update_z<B, T, false>(z, R, e);
    }
}

// Values of A P: slot q of A P is the sum, value by value, of the A slots
// gidx[gptr[q] .. gptr[q + 1]) (ascending); padding slots get 0.
__global__ void ap_values_kernel(int64_t slots, int bb, const int* __restrict__ gptr, const int* __restrict__ gidx,
                                 const double* __restrict__ a, double* __restrict__ ap)
{
    GRID_STRIDE(i, slots * bb)
    {
        const int64_t q = i / bb;
        const int e = (int)(i - q * bb);
        double s = 0.0;
        const int g1 = gptr[q + 1];
        for (int g = gptr[q]; g < g1; ++g) s += a[(int64_t)gidx[g] * bb + e];
        ap[i] = s;
    }
}

// Inverse of the coarsest matrix (n <= kCoarsest unknowns), one thread block,
// in place in shared memory: Gauss-Jordan elimination with partial pivoting
// (Numerical Recipes, gaussj, row pivots only).  Per pivot k: a warp finds
// the largest |a_rk|, r >= k (the lowest r among equals) while every thread
// copies column k; rows k and p are swapped and row k is divided by the
// pivot; every other row r takes a_rj - a_kj f_r with f_r its entry in
// column k (column k itself becomes -f_r / pivot).  The row swaps show up
// as column swaps of the result, undone in reverse order when the inverse
// is written out.  A zero or non-finite pivot sets *status.
constexpr int kCoarsest = 128;

template <int B>
__global__ void __launch_bounds__(1024) dense_inverse_kernel(int nb, SellView m, const double* __restrict__ a,
                                                             double* __restrict__ inv, int* status)
{
    constexpr int BB = B * B;
    extern __shared__ __align__(16) double dsm[];
    const int n = nb * B;
    double* w = dsm;                  // n x n, row-major
    double* colk = dsm + n * n;       // column k before the row swap
    __shared__ int piv_row;
    __shared__ int perm[kCoarsest];   // row swapped with k at step k
    for (int i = threadIdx.x; i < n * n; i += blockDim.x) w[i] = 0.0;
    __syncthreads();
    for (int R = threadIdx.x; R < nb; R += blockDim.x) {
        const int lane = R & 31, sb = m.slice_ptr[R >> 5];
        for (int k = 0; k < m.len[R]; ++k) {
            const int J = m.col[sb + (k << 5) + lane];
            for (int i = 0; i < B; ++i)
                for (int j = 0; j < B; ++j) w[(R * B + i) * n + J * B + j] = a[(size_t)(sb + (k << 5) + lane) * BB + i * B + j];
        }
    }
    __syncthreads();
    for (int k = 0; k < n; ++k) {
        for (int r = threadIdx.x; r < n; r += blockDim.x) colk[r] = w[r * n + k];
        if (threadIdx.x < 32) {
            double best = -1.0;
            int bi = n;
            for (int r = k + (int)threadIdx.x; r < n; r += 32) {
                const double v = fabs(w[r * n + k]);
                if (v > best) {
                    best = v;
                    bi = r;
                }
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                const double ob = __shfl_xor_sync(0xffffffffu, best, o);
                const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
                if (ob > best || (ob == best && oi < bi)) {
                    best = ob;
                    bi = oi;
                }
            }
            if (threadIdx.x == 0) {
                piv_row = bi < n ? bi : k;
                perm[k] = piv_row;
                if (!(best > 0.0) || !isfinite(best)) *status = 1;
            }
        }
        __syncthreads();
        const int p = piv_row;
        const double pv = colk[p];
        for (int j = threadIdx.x; j < n; j += blockDim.x) {
            const double tk = w[k * n + j], tp = w[p * n + j];
            w[p * n + j] = tk;
            w[k * n + j] = (j == k ? 1.0 : tp) / pv;
        }
        __syncthreads();
        for (int i = threadIdx.x; i < n * n; i += blockDim.x) {
            const int r = i / n, j = i - r * n;
            if (r == k) continue;
            const double f = r == p ? colk[k] : colk[r];
            w[i] = (j == k ? 0.0 : w[i]) - w[k * n + j] * f;
        }
        __syncthreads();
    }
    // column j of the inverse is column src[j] of w: the swaps of steps
    // n-1 .. 0 applied to the columns in turn
    __shared__ int src[kCoarsest];
    if (threadIdx.x == 0) {
        for (int j = 0; j < n; ++j) src[j] = j;
        for (int k = n - 1; k >= 0; --k) {
            const int p = perm[k];
            if (p != k) {
                const int t = src[k];
                src[k] = src[p];
                src[p] = t;
            }
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < n * n; i += blockDim.x) {
        const int r = i / n, j = i - r * n;
        inv[i] = w[r * n + src[j]];
    }
}

template <class T, class M>
__global__ void dense_apply_kernel(int n, const M* __restrict__ inv, const T* __restrict__ r, T* __restrict__ z,
                                   const KScal* sc, int skip_if_s)
{
    pdl_wait();
    if (mg_skip(sc, skip_if_s)) return;
    dense_rows<T, M, false>(n, inv, r, z, (int)threadIdx.x, (int)blockDim.x);
}

// ---- the coarse end of the V-cycle in one kernel ------------------------------
// Below a size threshold a level of the V-cycle is a few microseconds of
// work spread over seven dependent launches.  mg_tail_kernel runs the whole
// cycle from one level down to the dense coarsest solve and back on a single
// thread-block cluster, with a cluster barrier (release/acquire at cluster
// scope) where the launch-per-step cycle has a kernel boundary, through the
// same row-range steps, so both give identical results.  Vectors written
// inside the kernel are read with L2-only loads.  Every thread passes every
// barrier: loop bounds are kernel parameters or device arrays that do not
// change while it runs, and so is the early-exit flag (a converged solve).
constexpr int kTailThreads = 512;
constexpr int kMaxTail = 8;
constexpr int kMaxPrefetch = 64;

// A device array the fused cycle prefetches into L2 when it starts (the
// fine level's sweeps between two visits evict the coarse levels' data).
struct PrefetchRegion {
    const void* ptr;  // 16-byte aligned
    unsigned long long bytes;
};

// Stages of a level the fused cycle takes (their bounds are kernel
// parameters).
constexpr int kTailStages = 8;

// Offsets (bytes) of a level's arrays in the shared memory of block 0, for
// the levels at the coarse end that the fused cycle keeps there.
struct TailLocal {
    int a, lu, inv, col, len, dk, aggb, mpad, r, z, t, w;
};

// One device array copied into block 0's shared memory when the kernel starts.
struct TailCopy {
    const void* src;  // 16-byte aligned
    int dst;          // shared memory offset, 16-byte aligned
    int bytes;        // a multiple of 4
};
constexpr int kMaxCopies = 32;
// Shared memory of the levels kept there (block 0; every block of the
// cluster is launched with the same size).
constexpr int kTailSmem = 200 * 1024;

template <class T, class M>
struct TailLevel {
    int nb = 0, n = 0, coarsest = 0;
    TailLocal so{};              // shared memory layout (levels >= local_first)
    SellView m{};                // slices of uniform width m.width
    const M* a = nullptr;
    const M* lu = nullptr;
    const M* inv = nullptr;      // coarsest level
    int nstages = 0;
    int sp[kTailStages + 1] = {};  // stage bounds
    const int* aggb = nullptr;   // to the next coarser level
    const int* mpad = nullptr;   // aggregate members, kMembers per coarse unknown
    T *r = nullptr, *z = nullptr, *t = nullptr, *w = nullptr;
};

template <class T, class M>
struct TailParams {
    TailLevel<T, M> lv[kMaxTail];
    int nlev = 0;
    int local_first = kMaxTail;  // first level kept in block 0's shared memory (>= 1; nlev: none)
    int nregions = 0;
    int ncopies = 0;
    PrefetchRegion reg[kMaxPrefetch];
    TailCopy copies[kMaxCopies];
    double alpha = 1.0;          // coarse-correction factor
    long long* trace = nullptr;  // SM clock after each step (linsolver_tail_trace)
};

// Thread blocks split every region into 16-byte aligned chunks and hand them
// to the TMA unit as bulk L2 prefetches.
__device__ __forceinline__ void prefetch_regions(const PrefetchRegion* reg, int nregions)
{
    if ((int)threadIdx.x >= nregions) return;
    const PrefetchRegion& g = reg[threadIdx.x];
    const unsigned long long chunk = ((g.bytes / gridDim.x) + 15ull) & ~15ull;
    const unsigned long long off = chunk * blockIdx.x;
    if (off >= g.bytes) return;
    unsigned long long len = g.bytes - off < chunk ? g.bytes - off : chunk;
    len &= ~15ull;
    if (len == 0) return;
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"((const char*)g.ptr + off), "r"((unsigned)len)
                 : "memory");
}

__device__ __forceinline__ void cluster_barrier()
{
    asm volatile("barrier.cluster.arrive.release;\n\tbarrier.cluster.wait.acquire;" ::: "memory");
}

// Entries of the step trace: the start, then one per step.
constexpr int kTraceMax = 128;

// Ends one step of the fused cycle: a cluster barrier, after which thread 0
// of block 0 records the SM clock when a trace buffer is given.
__device__ __forceinline__ void tail_step(long long* trace, int& k)
{
    cluster_barrier();
    if (trace != nullptr && blockIdx.x == 0 && threadIdx.x == 0 && k < kTraceMax) trace[k] = clock64();
    ++k;
}

// out = M^{-1} b on one level (zadd += out when given), stage by stage.
template <int B, int KM, class T, class M>
__device__ __forceinline__ void tail_ilu(const TailLevel<T, M>& L, const T* b, T* out, T* zadd, int tid, int nth,
                                         long long* trace, int& tk)
{
    constexpr bool U = KM > 0;
    const int ns = L.nstages;
    if (ns <= 0) return;
    const int r_first = L.sp[1];
    for (int s = 1; s < ns; ++s) {
        const int last = s == ns - 1;
        lower_rows<B, KM, T, M, true, U>(L.sp[s], L.sp[s + 1], r_first, last, L.m, L.lu, b, out,
                                         last ? zadd : nullptr, tid, nth);
        tail_step(trace, tk);
    }
    for (int s = ns >= 2 ? ns - 2 : 0; s >= 0; --s) {
        upper_rows<B, KM, T, M, true, U>(L.sp[s], L.sp[s + 1], s == 0, L.m, L.lu, b, out, zadd, tid, nth);
        tail_step(trace, tk);
    }
}

static_assert(sizeof(TailParams<double, double>) <= 4096, "fused cycle parameters exceed 4 KB");

// Block 0 starts the copies of the shared-memory levels' arrays (cp.async:
// global to shared without registers; waited for with cp.async.wait_all,
// which ends when this thread's copies have landed).
__device__ __forceinline__ void start_local_copies(const TailCopy* cp, int ncopies, unsigned char* sm)
{
    for (int i = 0; i < ncopies; ++i) {
        const char* src = (const char*)cp[i].src;
        const unsigned dst = (unsigned)__cvta_generic_to_shared(sm + cp[i].dst);
        const int n16 = cp[i].bytes >> 4;
        for (int j = threadIdx.x; j < n16; j += blockDim.x)
            asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst + 16 * j), "l"(src + 16 * j) : "memory");
        for (int j = (n16 << 2) + threadIdx.x; j < (cp[i].bytes >> 2); j += blockDim.x)
            asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(dst + 4 * j), "l"(src + 4 * j) : "memory");
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
}

// A level's arrays in block 0's shared memory.
template <class T, class M>
struct LocalView {
    SellView m;
    const M *a, *lu, *inv;
    const int *aggb, *mpad;
    T *r, *z, *t, *w;
};

template <class T, class M>
__device__ __forceinline__ LocalView<T, M> local_view(const TailLevel<T, M>& G, unsigned char* sm)
{
    const TailLocal& o = G.so;
    LocalView<T, M> v;
    v.m = SellView{nullptr, (const int*)(sm + o.col), (const int*)(sm + o.len), (const int*)(sm + o.dk), G.m.width};
    v.a = (const M*)(sm + o.a);
    v.lu = (const M*)(sm + o.lu);
    v.inv = (const M*)(sm + o.inv);
    v.aggb = (const int*)(sm + o.aggb);
    v.mpad = (const int*)(sm + o.mpad);
    v.r = (T*)(sm + o.r);
    v.z = (T*)(sm + o.z);
    v.t = (T*)(sm + o.t);
    v.w = (T*)(sm + o.w);
    return v;
}

// out = M^{-1} b on a shared-memory level, stage by stage (block barriers).
template <int B, int KM, class T, class M>
__device__ __forceinline__ void local_ilu(const TailLevel<T, M>& G, const LocalView<T, M>& V, const T* b, T* out,
                                          T* zadd)
{
    const int tid = (int)threadIdx.x, nth = (int)blockDim.x;
    const int ns = G.nstages;
    if (ns <= 0) return;
    for (int s = 1; s < ns; ++s) {
        const int last = s == ns - 1;
        lower_rows<B, KM, T, M, false, true>(G.sp[s], G.sp[s + 1], G.sp[1], last, V.m, V.lu, b, out,
                                             last ? zadd : nullptr, tid, nth);
        __syncthreads();
    }
    for (int s = ns >= 2 ? ns - 2 : 0; s >= 0; --s) {
        upper_rows<B, KM, T, M, false, true>(G.sp[s], G.sp[s + 1], s == 0, V.m, V.lu, b, out, zadd, tid, nth);
        __syncthreads();
    }
}

// The coarse end of the cycle on block 0 alone, from level lf (whose right
// side is restricted from the residual t of level lf - 1 in global memory)
// down to the dense solve and back; the correction of level lf is written to
// its global z.  Same steps and operations as the cluster-wide ones.
template <int B, int KM, class T, class M>
__device__ void local_cycle(const TailParams<T, M>& p, int lf, unsigned char* sm)
{
    const int tid = (int)threadIdx.x, nth = (int)blockDim.x;
    asm volatile("cp.async.wait_all;" ::: "memory");
    __syncthreads();
    {
        const TailLevel<T, M>& F = p.lv[lf - 1];
        restrict_padded_rows<T, true>(p.lv[lf].n, F.mpad, F.t, local_view(p.lv[lf], sm).r, tid, nth);
        __syncthreads();
    }
    int l = lf;
    for (;; ++l) {
        const TailLevel<T, M>& G = p.lv[l];
        const LocalView<T, M> V = local_view(G, sm);
        if (G.coarsest || l == p.nlev - 1) {
            dense_rows<T, M, false>(G.n, V.inv, V.r, V.z, tid, nth);
            __syncthreads();
            break;
        }
        local_ilu<B, KM, T, M>(G, V, V.r, V.z, nullptr);
        residual_rows<B, KM, T, M, false, true>(G.nb, G.nstages >= 1 ? G.sp[1] : 0, V.m, V.a, V.z, V.r, V.t, tid,
                                                nth);
        __syncthreads();
        restrict_padded_rows<T, false>(p.lv[l + 1].n, V.mpad, V.t, local_view(p.lv[l + 1], sm).r, tid, nth);
        __syncthreads();
    }
    for (--l; l >= lf; --l) {
        const TailLevel<T, M>& G = p.lv[l];
        const LocalView<T, M> V = local_view(G, sm);
        prolong_rows<B, T, false>(G.nb, V.aggb, local_view(p.lv[l + 1], sm).z, V.z, p.alpha, tid, nth);
        __syncthreads();
        residual_rows<B, KM, T, M, false, true>(G.nb, 0, V.m, V.a, V.z, V.r, V.t, tid, nth);
        __syncthreads();
        local_ilu<B, KM, T, M>(G, V, V.t, V.w, V.z);
    }
    const T* zs = local_view(p.lv[lf], sm).z;
    for (int i = tid; i < p.lv[lf].n; i += nth) p.lv[lf].z[i] = zs[i];
}

// z = V-cycle(r) from level lv[0] down; r and z of lv[0] are r_top, z_top.
template <int B, int KM, class T, class M>
__global__ void __launch_bounds__(kTailThreads)
    mg_tail_kernel(const __grid_constant__ TailParams<T, M> p, const T* r_top, T* z_top, const KScal* sc, int skip_if_s)
{
    constexpr bool U = KM > 0;  // slices of uniform width (unrolled rows only)
    extern __shared__ __align__(16) unsigned char tail_smem[];
    // the levels' matrices and index arrays do not change during a solve:
    // their L2 prefetches and shared-memory copies start before the wait for
    // the previous kernel
    const int lf = p.local_first < p.nlev ? p.local_first : p.nlev;
    if (lf < p.nlev && blockIdx.x == 0) start_local_copies(p.copies, p.ncopies, tail_smem);
    prefetch_regions(p.reg, p.nregions);
    pdl_wait();
    if (mg_skip(sc, skip_if_s)) {
        asm volatile("cp.async.wait_all;" ::: "memory");
        return;
    }
    long long* const trace = p.trace;
    int tk = 0;
    if (trace != nullptr && blockIdx.x == 0 && threadIdx.x == 0) trace[tk] = clock64();
    ++tk;
    // rows go to threads a warp (one slice of 32 rows) at a time, round robin
    // over the cluster's blocks, so that a step of a few slices still spreads
    // over every SM of the cluster
    const int tid = (((int)(threadIdx.x >> 5) * (int)gridDim.x + (int)blockIdx.x) << 5) | (int)(threadIdx.x & 31);
    const int nth = (int)(gridDim.x * blockDim.x);
    int l = 0;
    for (; l < lf; ++l) {
        const TailLevel<T, M>& L = p.lv[l];
        const T* r = l == 0 ? r_top : L.r;
        T* z = l == 0 ? z_top : L.z;
        if (L.coarsest || l == p.nlev - 1) {
            dense_rows<T, M, true>(L.n, L.inv, r, z, tid, nth);
            tail_step(trace, tk);
            break;
        }
        tail_ilu<B, KM, T, M>(L, r, z, nullptr, tid, nth, trace, tk);
        residual_rows<B, KM, T, M, true, U>(L.nb, L.nstages >= 1 ? L.sp[1] : 0, L.m, L.a, z, r, L.t, tid, nth);
        tail_step(trace, tk);
        if (l + 1 < lf) {
            restrict_padded_rows<T, true>(p.lv[l + 1].n, L.mpad, L.t, p.lv[l + 1].r, tid, nth);
            tail_step(trace, tk);
        }
    }
    if (l == lf) {
        // the levels kept in shared memory: block 0 alone, the other blocks
        // wait at the next cluster barrier
        if constexpr (U) {
            if (blockIdx.x == 0) local_cycle<B, KM, T, M>(p, lf, tail_smem);
        }
        tail_step(trace, tk);
    }
    for (--l; l >= 0; --l) {
        const TailLevel<T, M>& L = p.lv[l];
        const T* r = l == 0 ? r_top : L.r;
        T* z = l == 0 ? z_top : L.z;
        prolong_rows<B, T, true>(L.nb, L.aggb, p.lv[l + 1].z, z, p.alpha, tid, nth);
        tail_step(trace, tk);
        residual_rows<B, KM, T, M, true, U>(L.nb, 0, L.m, L.a, z, r, L.t, tid, nth);
        tail_step(trace, tk);
        tail_ilu<B, KM, T, M>(L, L.t, L.w, z, tid, nth, trace, tk);
    }
}

}  // namespace

// ---------------------------------------------------------------------------
// Host analysis, cached per Jacobian pattern.
//
// Multilevel preconditioner (the default when the system is laid out as
// `ncomp` blocks of one unknown per grid cell, as newtonSolve and
// newtonSolveSystem stack them): geometric aggregation of 2x2x2 cells per
// unknown block, Galerkin coarse matrices R A R^T, a V(1,1) cycle with one
// block ILU(0) sweep before and after the coarse correction on every level,
// and a dense inverse on the coarsest level (<= 128 unknowns).  Otherwise
// plain block ILU(0).
// ---------------------------------------------------------------------------
struct HostCsr {
    int n = 0;
    std::vector<int> ptr, col;
};

struct Level {
    int n = 0;                     // unknowns
    int nb = 0;                    // block rows
    int bs = 1;                    // block size
    int64_t nnz = 0;               // scalar entries of the matrix pattern
    int cx = 1, cy = 1, cz = 1;    // cells of this level's grid
    bool coarsest = false;
    std::vector<int> stage_ptr;    // stages (colours or wavefronts) of block rows, permuted order
    // blocks left and right of the diagonal in the rows of each stage
    // (algorithmic bytes of the sweeps)
    std::vector<int64_t> stage_lower, stage_upper;
    Buf perm;                      // permuted unknown position -> natural unknown
    Buf gptr, gidx, gpos;          // Galerkin gather from the finer level's values (levels > 0)
    Buf aggb;                      // coarse block row of each block row (next coarser level)
    // A P (see mg_correct_kernel), in the same sliced layout: slots, the
    // longest row, slices, coarse block columns, row lengths, and the A slots
    // summed into each slot (gptr/gidx); levels above linsolver_mg_ap_rows
    int64_t ap_slots = 0;
    int64_t ap_blocks = 0;         // coarse block columns over all rows (without padding)
    int ap_kmax = 0;
    Buf ap_sp, ap_col, ap_len, ap_gptr, ap_gidx, ap64, ap32;
    SellView ap_view() const
    {
        return SellView{ap_sp->as<int>(), ap_col->as<int>(), ap_len->as<int>(), ap_len->as<int>(), 0};
    }
    // host copies of the slices, columns and row lengths while the
    // hierarchy is built
    std::vector<int> h_sp, h_col, h_len;
    Buf mptr, midx;                // aggregate members (unknown positions) of each coarse unknown
    Buf mpad;                      // the same, kMembers per coarse unknown, -1 past the last (or none)
    int64_t sell_size = 0;         // slots of the block sliced ELL layout
    int64_t vals = 0;              // sell_size * bs^2
    int64_t blocks = 0;            // block entries of the pattern (without padding)
    int kmax = 0;                  // longest block row
    int width = 0;                 // slots per row of every slice when uniform (else 0)
    int threads = kThreads;        // threads per block of this level's launch-per-step kernels (autotuned)
    Buf sell_ptr, sell_col, sell_len, sell_dk;
    Buf as64, lus64, as32, lus32;  // matrix, block ILU(0) factors (inverted diagonal blocks)
    Buf v64, v32;                  // 4 work vectors: r, z, t, w
    SellView view() const
    {
        return SellView{sell_ptr->as<int>(), sell_col->as<int>(), sell_len->as<int>(), sell_dk->as<int>(), width};
    }
    Buf inv64, inv32;              // coarsest level
};

struct SolverAnalysis {
    int n = 0;
    int64_t nnz = 0;
    bool natural = false;
    bool ok = true;  // every row has a diagonal entry (1 x 1 blocks)
    bool multigrid = false;
    double mg_alpha = 1.0;  // coarse-grid correction factor
    std::vector<Level> levels;
    Buf vmap;        // level-0 value <- Jacobian entry (-1: zero)
    Buf vec64, vec32, scal, partials, counter, factor_status;
    // coarse levels fused into one kernel: levels[tail_first..] (-1: none),
    // their longest block row, cluster size per precision (pc_mode)
    int tail_first = -1;
    int tail_kmax = 0;
    int tail_cluster[3] = {0, 0, 0};
    // per precision: first fused level kept in block 0's shared memory
    // (index into the fused levels; their count: none)
    int tail_local[3] = {0, 0, 0};
    int last_mode = 0;  // precision of the last solve (pc_mode)
    bool tuned[3] = {false, false, false};  // launch shapes chosen, per precision (autotune)
    Buf tail_trace;  // SM clock after each step of the last fused cycle
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
    if (!v.empty()) c.copy_to_device(b->ptr, v.data(), v.size() * 4);
    return b;
}

// Sorts a short list and drops repeats; returns the new length.
inline int sort_unique(int* v, int len)
{
    std::sort(v, v + len);
    return (int)(std::unique(v, v + len) - v);
}

// Position of `key` in the sorted short list v[0..len) (len if absent).
inline int find_small(const int* v, int len, int key)
{
    int k = 0;
    while (k < len && v[k] < key) ++k;
    return (k < len && v[k] == key) ? k : len;
}

// Builds the CSR pattern whose row r is the sorted, repeat-free union of
// the columns that gather(r, buf) writes into buf (at most `cap` of them).
// Two passes over the rows, each parallel over rows.
template <class Gather>
void build_rows(int nrows, int cap, HostCsr& out, Gather gather)
{
    out.n = nrows;
    out.ptr.assign(nrows + 1, 0);
#pragma omp parallel
    {
        std::vector<int> buf(cap > 0 ? cap : 1);
#pragma omp for schedule(static)
        for (int r = 0; r < nrows; ++r) out.ptr[r + 1] = sort_unique(buf.data(), gather(r, buf.data()));
    }
    for (int r = 0; r < nrows; ++r) out.ptr[r + 1] += out.ptr[r];
    out.col.resize(out.ptr[nrows] > 0 ? out.ptr[nrows] : 1);
#pragma omp parallel
    {
        std::vector<int> buf(cap > 0 ? cap : 1);
#pragma omp for schedule(static)
        for (int r = 0; r < nrows; ++r) {
            const int len = sort_unique(buf.data(), gather(r, buf.data()));
            std::copy(buf.data(), buf.data() + len, out.col.begin() + out.ptr[r]);
        }
    }
}

inline int max_row(const HostCsr& A)
{
    int m = 0;
    for (int r = 0; r < A.n; ++r) m = std::max(m, A.ptr[r + 1] - A.ptr[r]);
    return m;
}

// Lays out the matrix with pattern `A` (natural unknown numbering, rows with
// ascending columns) in blocks of `bs` unknowns: block row of unknown u is
// u % nb and its component u / nb (nb = n / bs).  Orders the block rows by
// stage and builds the block sliced ELL pattern (each row with its diagonal
// block).  Returns the unknown permutation (position -> natural unknown),
// its inverse, and for every entry of `A` its position in the level's value
// array.  With `uniform`, every slice is as wide as the longest row.
void order_level(Core& c, const HostCsr& A, bool natural, int bs, bool uniform, Level& L, std::vector<int>& perm,
                 std::vector<int>& iperm, std::vector<int>& vpos, bool& ok)
{
    const int n = A.n;
    const int nb = n / bs;
    const int bb = bs * bs;
    const int64_t nnz = A.ptr[n];
    const auto t0 = std::chrono::steady_clock::now();
    auto ms = [&] { return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count(); };
    // block graph (natural block numbering), sorted, with the diagonal
    HostCsr G;
    build_rows(nb, bs * max_row(A) + 1, G, [&](int R, int* buf) {
        int len = 0;
        for (int cc = 0; cc < bs; ++cc) {
            const int u = cc * nb + R;
            for (int e = A.ptr[u]; e < A.ptr[u + 1]; ++e) {
                int cell = A.col[e];
                while (cell >= nb) cell -= nb;  // column mod nb, at most bs - 1 subtractions
                buf[len++] = cell;
            }
        }
        buf[len++] = R;
        return len;
    });
    if (bs == 1) {
        bool all = true;
#pragma omp parallel for reduction(&& : all) schedule(static)
        for (int u = 0; u < n; ++u) {
            bool has = false;
            for (int e = A.ptr[u]; e < A.ptr[u + 1]; ++e) has = has || A.col[e] == u;
            all = all && has;
        }
        if (!all) ok = false;
    }
    const double tg = ms();
    const std::vector<int> key = stage_keys(G, natural);
    const double tk = ms();
    const int nst = nb > 0 ? *std::max_element(key.begin(), key.end()) + 1 : 0;
    L.stage_ptr.assign(nst + 1, 0);
    for (int R = 0; R < nb; ++R) L.stage_ptr[key[R] + 1]++;
    for (int s = 0; s < nst; ++s) L.stage_ptr[s + 1] += L.stage_ptr[s];
    std::vector<int> pb(nb), ipb(nb);
    {
        std::vector<int> pos(L.stage_ptr.begin(), L.stage_ptr.end() - 1);
        for (int R = 0; R < nb; ++R) pb[pos[key[R]]++] = R;
    }
    for (int R = 0; R < nb; ++R) ipb[pb[R]] = R;
    perm.assign(n, 0);
    iperm.assign(n, 0);
#pragma omp parallel for schedule(static)
    for (int R = 0; R < nb; ++R)
        for (int cc = 0; cc < bs; ++cc) {
            perm[R * bs + cc] = cc * nb + pb[R];
            iperm[cc * nb + pb[R]] = R * bs + cc;
        }
    const double tp = ms();
    // permuted block rows: sorted permuted columns
    std::vector<int> pptr(nb + 1, 0), pcol(G.ptr[nb] > 0 ? G.ptr[nb] : 1);
    for (int R = 0; R < nb; ++R) pptr[R + 1] = pptr[R] + (G.ptr[pb[R] + 1] - G.ptr[pb[R]]);
#pragma omp parallel for schedule(static)
    for (int R = 0; R < nb; ++R) {
        const int o = pb[R];
        int w = pptr[R];
        for (int e = G.ptr[o]; e < G.ptr[o + 1]; ++e) pcol[w++] = ipb[G.col[e]];
        std::sort(pcol.begin() + pptr[R], pcol.begin() + pptr[R + 1]);
    }
    const double tc = ms();
    // block sliced ELL, 32 block rows per slice
    const int nsl = (nb + 31) / 32;
    std::vector<int> sp(nsl + 1, 0), len(nb > 0 ? nb : 1), dk(nb > 0 ? nb : 1);
    int wmax = 0;
    for (int R = 0; R < nb; ++R) wmax = std::max(wmax, pptr[R + 1] - pptr[R]);
    for (int sl = 0; sl < nsl; ++sl) {
        int w = 0;
        for (int R = sl * 32; R < std::min(nb, sl * 32 + 32); ++R) w = std::max(w, pptr[R + 1] - pptr[R]);
        sp[sl + 1] = sp[sl] + 32 * (uniform ? wmax : w);
    }
    L.width = uniform ? wmax : 0;
    const int64_t size = sp[nsl];
    if (size * bb >= (int64_t)INT_MAX) fail(EQG_ERR_UNSUPPORTED, "linear system too large for 32-bit value offsets");
    std::vector<int> scol(size > 0 ? size : 1, 0);
    int kmax = 0;
#pragma omp parallel for reduction(max : kmax) schedule(static)
    for (int R = 0; R < nb; ++R) {
        const int base = sp[R / 32] + (R % 32);
        len[R] = pptr[R + 1] - pptr[R];
        kmax = std::max(kmax, len[R]);
        const int w = (sp[R / 32 + 1] - sp[R / 32]) / 32;
        dk[R] = -1;
        for (int k = 0; k < w; ++k) {
            if (k < len[R]) {
                scol[base + 32 * k] = pcol[pptr[R] + k];
                if (pcol[pptr[R] + k] == R) dk[R] = k;
            } else {
                scol[base + 32 * k] = R;  // padding: a valid column, values 0, never read by the kernels
            }
        }
    }
    L.kmax = kmax;
    const double ts = ms();
    // value position of every scalar entry of A, block row by block row
    vpos.assign(nnz > 0 ? nnz : 1, -1);
#pragma omp parallel for schedule(static)
    for (int Rn = 0; Rn < nb; ++Rn) {
        const int R = ipb[Rn];
        const int* row = pcol.data() + pptr[R];
        const int rl = pptr[R + 1] - pptr[R];
        for (int cu = 0; cu < bs; ++cu) {
            const int u = cu * nb + Rn;
            for (int e = A.ptr[u]; e < A.ptr[u + 1]; ++e) {
                int cell = A.col[e], cv = 0;  // column = cv nb + cell, cv < bs (no division)
                while (cell >= nb) {
                    cell -= nb;
                    ++cv;
                }
                const int k = find_small(row, rl, ipb[cell]);
                const int64_t slot0 = sp[R / 32] + 32 * k;
                vpos[e] = (int)((slot0 + R % 32) * bb + cu * bs + cv);
            }
        }
    }
    const double tv = ms();
    L.n = n;
    L.nb = nb;
    L.bs = bs;
    L.nnz = nnz;
    L.sell_size = size;
    L.vals = size * bb;
    L.blocks = pptr[nb];
    L.sell_ptr = upload_ints(c, sp);
    L.sell_col = upload_ints(c, scol);
    L.h_sp = sp;
    L.h_col = scol;
    L.h_len = len;
    L.sell_len = upload_ints(c, len);
    L.sell_dk = upload_ints(c, dk);
    {
        const int nst = (int)L.stage_ptr.size() - 1;
        L.stage_lower.assign(nst > 0 ? nst : 0, 0);
        L.stage_upper.assign(nst > 0 ? nst : 0, 0);
        for (int st = 0; st < nst; ++st)
            for (int R = L.stage_ptr[st]; R < L.stage_ptr[st + 1]; ++R) {
                const int d = dk[R] >= 0 ? dk[R] : 0;
                L.stage_lower[st] += d;
                L.stage_upper[st] += std::max(0, len[R] - d - 1);
            }
    }
    const size_t nv = (size_t)(L.vals > 0 ? L.vals : 1);
    L.as64 = c.allocN<double>(nv);
    L.lus64 = c.allocN<double>(nv);
    L.perm = upload_ints(c, perm);
    L.v64 = c.allocN<double>((size_t)4 * (n > 0 ? n : 1));
    if (c.verbose > 2 && nb > 100000)
        std::printf("        ordering of %d block rows: %.1f ms (block graph %.1f, stages %.1f, permutation %.1f, "
                    "sorted columns %.1f, slices %.1f, value positions %.1f, uploads %.1f)\n",
                    nb, ms(), tg, tk - tg, tp - tk, tc - tp, ts - tc, tv - ts, ms() - tv);
}

// A P of level L (see mg_correct_kernel): for every block row, its coarse
// block columns (aggregates of its columns, ascending) in slices of 32 rows,
// and for every slot the A slots it sums.
void build_ap(Core& c, Level& L, const std::vector<int>& aggb)
{
    const int nb = L.nb;
    const int nsl = (nb + 31) / 32;
    const int W = L.kmax;  // a row has at most as many coarse columns as blocks
    if (W < 1 || W > 64) return;
    std::vector<int> alen(nb > 0 ? nb : 1, 0);
    std::unique_ptr<int[]> rowq(new int[(size_t)nb * W]);  // coarse columns of each row, ascending
    int kmax = 0;
#pragma omp parallel for reduction(max : kmax) schedule(static)
    for (int R = 0; R < nb; ++R) {
        const int base = L.h_sp[R / 32] + (R % 32);
        int q[64];
        int nq = 0;
        for (int k = 0; k < L.h_len[R]; ++k) {
            const int P = aggb[L.h_col[base + 32 * k]];
            bool seen = false;
            for (int j = 0; j < nq; ++j) seen = seen || q[j] == P;
            if (!seen && nq < 64) q[nq++] = P;
        }
        std::sort(q, q + nq);
        alen[R] = nq;
        kmax = std::max(kmax, nq);
        for (int j = 0; j < nq; ++j) rowq[(size_t)R * W + j] = q[j];
    }
    std::vector<int> asp(nsl + 1, 0);
    for (int sl = 0; sl < nsl; ++sl) {
        int w = 0;
        for (int R = sl * 32; R < std::min(nb, sl * 32 + 32); ++R) w = std::max(w, alen[R]);
        asp[sl + 1] = asp[sl] + 32 * w;
    }
    const int64_t slots = asp[nsl];
    std::vector<int> acol(slots > 0 ? slots : 1, 0), cnt(slots + 1, 0);
#pragma omp parallel for schedule(static)
    for (int R = 0; R < nb; ++R) {
        const int abase = asp[R / 32] + (R % 32);
        const int w = (asp[R / 32 + 1] - asp[R / 32]) / 32;
        const int base = L.h_sp[R / 32] + (R % 32);
        for (int j = 0; j < w; ++j) acol[abase + 32 * j] = j < alen[R] ? rowq[(size_t)R * W + j] : aggb[R];
        for (int k = 0; k < L.h_len[R]; ++k) {
            const int P = aggb[L.h_col[base + 32 * k]];
            const int j = (int)(std::lower_bound(&rowq[(size_t)R * W], &rowq[(size_t)R * W] + alen[R], P) -
                                &rowq[(size_t)R * W]);
            cnt[abase + 32 * j + 1]++;  // one writer per slot: slots belong to one row
        }
    }
    for (int64_t q = 0; q < slots; ++q) cnt[q + 1] += cnt[q];
    std::vector<int> gidx(cnt[slots] > 0 ? cnt[slots] : 1);
#pragma omp parallel for schedule(static)
    for (int R = 0; R < nb; ++R) {
        const int abase = asp[R / 32] + (R % 32);
        const int base = L.h_sp[R / 32] + (R % 32);
        int fill[64] = {0};  // per coarse column of the row (at most W <= 64)
        for (int k = 0; k < L.h_len[R]; ++k) {
            const int P = aggb[L.h_col[base + 32 * k]];
            const int j = (int)(std::lower_bound(&rowq[(size_t)R * W], &rowq[(size_t)R * W] + alen[R], P) -
                                &rowq[(size_t)R * W]);
            const int q = abase + 32 * j;
            gidx[cnt[q] + fill[j]++] = base + 32 * k;
        }
    }
    L.ap_slots = slots;
    L.ap_kmax = kmax;
    L.ap_blocks = 0;
    for (int R = 0; R < nb; ++R) L.ap_blocks += alen[R];
    L.ap_sp = upload_ints(c, asp);
    L.ap_col = upload_ints(c, acol);
    L.ap_len = upload_ints(c, alen);
    L.ap_gptr = upload_ints(c, cnt);
    L.ap_gidx = upload_ints(c, gidx);
    L.ap64 = c.allocN<double>((size_t)(slots > 0 ? slots : 1) * L.bs * L.bs);
}

std::shared_ptr<SolverAnalysis> analyse(Core& c, const Pattern& p, bool natural, bool allow_multigrid)
{
    const auto t_start = std::chrono::steady_clock::now();
    auto since = [&] {
        return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_start).count();
    };
    // host threads of the analysis (host_threads=k; default: OpenMP's), for
    // processes that drive several runtimes at once
    const int host_threads = c.param_i("host_threads", 0);
    if (host_threads > 0) omp_set_num_threads(host_threads);
    auto an = std::make_shared<SolverAnalysis>();
    const int n = p.rows;
    an->n = n;
    an->nnz = p.nnz;
    an->natural = natural;
    HostCsr A;
    A.n = n;
    A.ptr.resize(n + 1);
    A.col.resize(p.nnz > 0 ? p.nnz : 1);
    c.copy_to_host(A.ptr.data(), p.rowptr->ptr, (size_t)(n + 1) * 4);
    if (p.nnz > 0) c.copy_to_host(A.col.data(), p.colind->ptr, (size_t)p.nnz * 4);

    const std::string pre = c.param_s("linsolver_preconditioner", "multigrid");
    if (pre != "multigrid" && pre != "ilu0") fail(EQG_ERR_ARG, "linsolver_preconditioner must be multigrid or ilu0");
    // unknowns stacked as ncomp collections over all cells
    const int ncomp = (c.nc > 0 && n % c.nc == 0) ? n / c.nc : 0;
    // coarsening stops at linsolver_mg_coarsest unknowns (at most kCoarsest)
    const int coarsest = std::max(1, std::min(kCoarsest, c.param_i("linsolver_mg_coarsest", kCoarsest)));
    // (the aggregation is geometric: Cartesian grids only)
    const bool mg_wanted =
        allow_multigrid && pre == "multigrid" && c.cartesian && ncomp >= 1 && ncomp <= 8 && n > coarsest;
    // Block ILU(0) sweeps with FP32 vectors (precision "refine") converge much
    // more slowly than scalar ones on the two-phase systems; with FP64
    // vectors, FP32 matrix values ("mixed") do not change the iteration
    // count.  So "refine" keeps 1 x 1 blocks.
    const bool fp64_vectors = c.param_s("linsolver_precision", "double") != "refine";
    const int bs =
        (!natural && fp64_vectors && (ncomp == 2 || ncomp == 3) && c.param_i("linsolver_block", 1) != 0) ? ncomp
                                                                                                          : 1;

    std::vector<int> perm, iperm, vpos;
    an->levels.emplace_back();
    const double t_copy = since();
    // levels small enough for the fused coarse cycle get slices of uniform width
    const int fuse_rows = c.param_i("linsolver_mg_fuse_rows", 40000);
    const int ap_rows = c.param_i("linsolver_mg_ap_rows", 40000);
    order_level(c, A, natural, bs, n <= fuse_rows, an->levels[0], perm, iperm, vpos, an->ok);
    const double t_level0 = since();
    {
        std::vector<int> vmap(an->levels[0].vals > 0 ? an->levels[0].vals : 1, -1);
#pragma omp parallel for schedule(static)
        for (int64_t e = 0; e < p.nnz; ++e) vmap[vpos[e]] = (int)e;
        an->vmap = upload_ints(c, vmap);
    }
    an->multigrid = mg_wanted && an->ok;
    an->mg_alpha = c.param_d("linsolver_mg_alpha", c.nz > 1 ? kMgAlpha3d : kMgAlpha2d);
    an->levels[0].cx = c.nx;
    an->levels[0].cy = c.ny;
    an->levels[0].cz = c.nz;
    if (an->multigrid) {
        // the finer level in its natural ordering, with its permutation and
        // value positions (level 0: the Jacobian pattern itself)
        const HostCsr* finep = &A;
        const std::vector<int>* fpermp = &perm;
        const std::vector<int>* fvposp = &vpos;
        HostCsr owned;
        std::vector<int> owned_perm, owned_vpos;
        for (;;) {
            const double tl0 = since();
            const HostCsr& fine = *finep;
            const std::vector<int>& fperm = *fpermp;
            const std::vector<int>& fvpos = *fvposp;
            Level& F = an->levels.back();
            const int fcx = F.cx, fcy = F.cy, fcz = F.cz;
            const int fcells = fcx * fcy * fcz;
            const int ccx = (fcx + 1) / 2, ccy = (fcy + 1) / 2, ccz = fcz > 1 ? (fcz + 1) / 2 : 1;
            const int ccells = ccx * ccy * ccz;
            const int nc_unk = ncomp * ccells;
            // aggregate of every fine unknown (natural indices)
            std::vector<int> agg_nat(fine.n);
#pragma omp parallel for schedule(static)
            for (int u = 0; u < fine.n; ++u) {
                const int comp = u / fcells, cell = u - comp * fcells;
                const int i = cell % fcx, j = (cell / fcx) % fcy, k = cell / (fcx * fcy);
                agg_nat[u] = comp * ccells + (i / 2) + ccx * ((j / 2) + ccy * (fcz > 1 ? k / 2 : 0));
            }
            // members of every coarse unknown (natural indices, ascending)
            std::vector<int> nmptr(nc_unk + 1, 0), nmidx(fine.n);
            for (int u = 0; u < fine.n; ++u) nmptr[agg_nat[u] + 1]++;
            for (int U = 0; U < nc_unk; ++U) nmptr[U + 1] += nmptr[U];
            {
                std::vector<int> pos(nmptr.begin(), nmptr.end() - 1);
                for (int u = 0; u < fine.n; ++u) nmidx[pos[agg_nat[u]]++] = u;
            }
            int max_members = 0;
            for (int U = 0; U < nc_unk; ++U) max_members = std::max(max_members, nmptr[U + 1] - nmptr[U]);
            // coarse pattern (natural ordering, sorted rows)
            HostCsr C;
            build_rows(nc_unk, max_members * max_row(fine) + 1, C, [&](int U, int* buf) {
                int len = 0;
                for (int m = nmptr[U]; m < nmptr[U + 1]; ++m) {
                    const int u = nmidx[m];
                    for (int e = fine.ptr[u]; e < fine.ptr[u + 1]; ++e) buf[len++] = agg_nat[fine.col[e]];
                }
                return len;
            });
            an->levels.emplace_back();
            Level& Lc = an->levels.back();
            Level& Lf = an->levels[an->levels.size() - 2];
            Lc.cx = ccx;
            Lc.cy = ccy;
            Lc.cz = ccz;
            std::vector<int> cperm, ciperm, cvpos;
            bool cok = true;
            const double tl1 = since();
            order_level(c, C, natural, bs, nc_unk <= fuse_rows, Lc, cperm, ciperm, cvpos, cok);
            const double tl2 = since();
            if (!cok) fail(EQG_ERR_DEVICE, "coarse level without a diagonal entry");
            // aggregation in permuted positions, and aggregate members
            std::vector<int> aggp(fine.n);
#pragma omp parallel for schedule(static)
            for (int pf = 0; pf < fine.n; ++pf) aggp[pf] = ciperm[agg_nat[fperm[pf]]];
            std::vector<int> mptr(nc_unk + 1, 0), midx(fine.n);
            for (int pf = 0; pf < fine.n; ++pf) mptr[aggp[pf] + 1]++;
            for (int P = 0; P < nc_unk; ++P) mptr[P + 1] += mptr[P];
            {
                std::vector<int> pos(mptr.begin(), mptr.end() - 1);
                for (int pf = 0; pf < fine.n; ++pf) midx[pos[aggp[pf]]++] = pf;
            }
            {
                // per block row: unknown R*bs + c aggregates onto coarse R'*bs + c
                std::vector<int> aggb(Lf.nb);
                bool whole = true;
#pragma omp parallel for schedule(static) reduction(&& : whole)
                for (int R = 0; R < Lf.nb; ++R) {
                    aggb[R] = aggp[R * bs] / bs;
                    for (int cc = 0; cc < bs; ++cc) whole = whole && aggp[R * bs + cc] == aggb[R] * bs + cc;
                }
                if (!whole) fail(EQG_ERR_DEVICE, "aggregation splits a block");
                Lf.aggb = upload_ints(c, aggb);
                if (Lf.n > ap_rows) build_ap(c, Lf, aggb);
            }
            Lf.h_sp.clear();
            Lf.h_col.clear();
            Lf.h_len.clear();
            Lf.mptr = upload_ints(c, mptr);
            Lf.midx = upload_ints(c, midx);
            if (max_members <= kMembers) {
                std::vector<int> mpad((size_t)nc_unk * kMembers, -1);
#pragma omp parallel for schedule(static)
                for (int P = 0; P < nc_unk; ++P)
                    for (int k = mptr[P]; k < mptr[P + 1]; ++k) mpad[(size_t)P * kMembers + (k - mptr[P])] = midx[k];
                Lf.mpad = upload_ints(c, mpad);
            }
            const double tl3 = since();
            // Galerkin gather: for every coarse entry, the value positions of
            // the fine entries that aggregate onto it, in ascending fine-entry
            // order.  A coarse row's entries come only from its members' rows,
            // so both passes run per coarse row.
            const int64_t fnnz = fine.ptr[fine.n];
            const int cnnz = C.ptr[nc_unk];
            std::vector<int> gptr(cnnz + 1, 0), gidx(fnnz > 0 ? fnnz : 1);
#pragma omp parallel for schedule(static)
            for (int U = 0; U < nc_unk; ++U) {
                const int* row = C.col.data() + C.ptr[U];
                const int rl = C.ptr[U + 1] - C.ptr[U];
                for (int m = nmptr[U]; m < nmptr[U + 1]; ++m) {
                    const int u = nmidx[m];
                    for (int e = fine.ptr[u]; e < fine.ptr[u + 1]; ++e)
                        gptr[C.ptr[U] + find_small(row, rl, agg_nat[fine.col[e]]) + 1]++;
                }
            }
            for (int k = 0; k < cnnz; ++k) gptr[k + 1] += gptr[k];
#pragma omp parallel
            {
                std::vector<int> pos;
#pragma omp for schedule(static)
                for (int U = 0; U < nc_unk; ++U) {
                    const int* row = C.col.data() + C.ptr[U];
                    const int rl = C.ptr[U + 1] - C.ptr[U];
                    pos.assign(gptr.begin() + C.ptr[U], gptr.begin() + C.ptr[U + 1]);
                    for (int m = nmptr[U]; m < nmptr[U + 1]; ++m) {
                        const int u = nmidx[m];
                        for (int e = fine.ptr[u]; e < fine.ptr[u + 1]; ++e)
                            gidx[pos[find_small(row, rl, agg_nat[fine.col[e]])]++] = fvpos[e];
                    }
                }
            }
            Lc.gptr = upload_ints(c, gptr);
            Lc.gidx = upload_ints(c, gidx);
            Lc.gpos = upload_ints(c, cvpos);
            Lc.nnz = cnnz;
            if (c.verbose > 2)
                std::printf("        coarse level of %d unknowns: %.1f ms (pattern %.1f, ordering %.1f, aggregation "
                            "and A P %.1f, Galerkin lists %.1f)\n",
                            nc_unk, since() - tl0, tl1 - tl0, tl2 - tl1, tl3 - tl2, since() - tl3);
            if (nc_unk <= coarsest || (ccx == 1 && ccy == 1 && ccz == 1)) {
                if (nc_unk > kCoarsest) {
                    an->multigrid = false;  // cannot coarsen further and too large to invert
                    an->levels.resize(1);
                    break;
                }
                Lc.coarsest = true;
                Lc.inv64 = c.allocN<double>((size_t)nc_unk * nc_unk);
                break;
            }
            owned = std::move(C);
            owned_perm = std::move(cperm);
            owned_vpos = std::move(cvpos);
            finep = &owned;
            fpermp = &owned_perm;
            fvposp = &owned_vpos;
        }
    }
    if (an->multigrid) {
        // fuse the levels of at most linsolver_mg_fuse_rows unknowns (0: none):
        // from the first level from which on every level is that small, has
        // slices of uniform width, at most kTailStages stages and aggregates
        // of at most kMembers members (the coarsest needs none of these)
        const int nl = (int)an->levels.size();
        auto fusable = [&](const Level& L) {
            return L.coarsest || (L.n <= fuse_rows && L.width > 0 && (int)L.stage_ptr.size() - 1 <= kTailStages &&
                                  L.mpad);
        };
        for (int l = nl - 1; l >= 0 && nl - l <= kMaxTail && fusable(an->levels[l]); --l)
            if (!an->levels[l].coarsest) an->tail_first = l;
        if (an->tail_first >= 0)
            for (int l = an->tail_first; l < nl; ++l)
                if (!an->levels[l].coarsest) an->tail_kmax = std::max(an->tail_kmax, an->levels[l].kmax);
    }
    for (auto& L : an->levels) {
        L.h_sp.clear();
        L.h_col.clear();
        L.h_len.clear();
    }
    an->vec64 = c.allocN<double>((size_t)10 * vec_stride(n));
    an->scal = c.alloc(sizeof(KScal));
    an->partials = c.allocN<double>((size_t)kRedBlocks * 2);
    an->counter = c.allocN<unsigned int>(1);
    an->factor_status = c.allocN<int>(1);
    EQG_CUDA(cudaMemsetAsync(an->counter->ptr, 0, sizeof(unsigned int), c.stream));
    c.sync();
    if (c.verbose > 2) {
        std::printf("        linear solver analysis: %.1f ms (pattern copy %.1f, level 0 %.1f, coarse levels %.1f)\n",
                    since(), t_copy, t_level0 - t_copy, since() - t_level0);
        std::printf("        linear solver: %dx%d blocks%s, levels:", bs, bs, an->multigrid ? ", multigrid" : "");
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
    for (int k = 0; k < 10; ++k) q[k] = base + (size_t)k * vec_stride(n);
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
template <class T>
const T* level_ap(const Level& L);
template <>
const double* level_ap<double>(const Level& L) { return L.ap64->as<double>(); }
template <>
const float* level_ap<float>(const Level& L) { return L.ap32->as<float>(); }

// Precision of a preconditioner application: vectors T, matrix values M.
// [0] FP64, [1] FP32 (inner solve of "refine"), [2] FP64 vectors with FP32
// matrices ("mixed").
template <class T, class M>
constexpr int pc_mode()
{
    return sizeof(T) == sizeof(float) ? 1 : (sizeof(M) == sizeof(float) ? 2 : 0);
}

// Cluster size for mg_tail_kernel<B, KM, T, M>: linsolver_mg_cluster
// (default 16, at most 16), reduced until the device reports that it can
// schedule one cluster of that size.
template <int B, int KM, class T, class M>
int tail_cluster_size(Core& c)
{
    int want = std::min(16, std::max(1, c.param_i("linsolver_mg_cluster", 16)));
    auto kern = mg_tail_kernel<B, KM, T, M>;
    if (want > 8) EQG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
    EQG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, kTailSmem));
    for (; want > 1; want /= 2) {
        cudaLaunchConfig_t cfg = {};
        cudaLaunchAttribute attr[1];
        cfg.gridDim = dim3(want);
        cfg.blockDim = dim3(kTailThreads);
        cfg.dynamicSmemBytes = kTailSmem;
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = want;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        int clusters = 0;
        if (cudaOccupancyMaxActiveClusters(&clusters, kern, &cfg) == cudaSuccess && clusters > 0) break;
        (void)cudaGetLastError();
    }
    return want;
}

// The fused levels kept in block 0's shared memory: from the coarsest level
// upward while their arrays fit in kTailSmem bytes (the first fused level
// stays cluster-wide).  Only for slices of uniform width (rows of at most 16
// blocks) and with linsolver_mg_local=1 (the default).  Returns the first
// such level as an index into the fused levels (their count: none); fills
// `bytes` and, when `p` is given, the layout and the copies.
template <class T, class M>
int plan_local(Core& c, const SolverAnalysis& an, int& bytes, TailParams<T, M>* p)
{
    const int nlev = (int)an.levels.size() - an.tail_first;
    bytes = 0;
    if (an.tail_first < 0 || an.tail_kmax > 16 || !c.param_i("linsolver_mg_local", 1)) return nlev;
    auto al = [](int64_t b) { return (b + 15) & ~(int64_t)15; };
    int lf = nlev;
    int64_t total = 0;
    int copies = 0;
    for (int i = nlev - 1; i >= 1; --i) {
        const Level& L = an.levels[an.tail_first + i];
        int64_t b = 2 * al((int64_t)L.n * sizeof(T));
        int nc = 0;
        if (L.coarsest) {
            b += al((int64_t)L.n * L.n * sizeof(M));
            nc = 1;
        } else {
            const Level& C = an.levels[an.tail_first + i + 1];
            b += 2 * al(L.vals * (int64_t)sizeof(M)) + al(L.sell_size * 4) + 3 * al((int64_t)L.nb * 4) +
                 al((int64_t)C.n * kMembers * 4) + 2 * al((int64_t)L.n * sizeof(T));
            nc = 7;
        }
        if (total + b > kTailSmem || copies + nc > kMaxCopies) break;
        total += b;
        copies += nc;
        lf = i;
    }
    if (lf == nlev) return nlev;
    bytes = (int)total;
    if (p) {
        int off = 0;
        auto place = [&](int64_t b) {
            const int o = off;
            off += (int)al(b);
            return o;
        };
        auto copy = [&](const void* src, int dst, int64_t b) {
            p->copies[p->ncopies++] = TailCopy{src, dst, (int)b};
        };
        for (int i = lf; i < nlev; ++i) {
            const Level& L = an.levels[an.tail_first + i];
            TailLocal& o = p->lv[i].so;
            o = TailLocal{};
            o.r = place((int64_t)L.n * sizeof(T));
            o.z = place((int64_t)L.n * sizeof(T));
            if (L.coarsest) {
                o.inv = place((int64_t)L.n * L.n * sizeof(M));
                copy(level_inv<M>(L), o.inv, (int64_t)L.n * L.n * sizeof(M));
                continue;
            }
            const Level& C = an.levels[an.tail_first + i + 1];
            o.t = place((int64_t)L.n * sizeof(T));
            o.w = place((int64_t)L.n * sizeof(T));
            o.a = place(L.vals * (int64_t)sizeof(M));
            o.lu = place(L.vals * (int64_t)sizeof(M));
            o.col = place(L.sell_size * 4);
            o.len = place((int64_t)L.nb * 4);
            o.dk = place((int64_t)L.nb * 4);
            o.aggb = place((int64_t)L.nb * 4);
            o.mpad = place((int64_t)C.n * kMembers * 4);
            copy(level_a<M>(L), o.a, L.vals * (int64_t)sizeof(M));
            copy(level_lu<M>(L), o.lu, L.vals * (int64_t)sizeof(M));
            copy(L.sell_col->ptr, o.col, L.sell_size * 4);
            copy(L.sell_len->ptr, o.len, (int64_t)L.nb * 4);
            copy(L.sell_dk->ptr, o.dk, (int64_t)L.nb * 4);
            copy(L.aggb->ptr, o.aggb, (int64_t)L.nb * 4);
            copy(L.mpad->ptr, o.mpad, (int64_t)C.n * kMembers * 4);
        }
        if (off != bytes) fail(EQG_ERR_DEVICE, "fused coarse cycle: shared memory layout mismatch");
        p->local_first = lf;
    }
    return lf;
}

// Algorithmic bytes of the solver launches (reported with kernel timings):
// every matrix block the step needs read once (its B^2 values and 4-byte
// column), 4 bytes of row data per block row read (its length or diagonal
// position), every vector element the step needs read or written once.
template <class M>
double block_bytes(const Level& L, int64_t blocks)
{
    return (double)blocks * (double)(sizeof(M) * L.bs * L.bs + 4);
}

// Launches kernel k on the runtime stream.  With c.pdl_launch it is a
// programmatic dependent launch: its blocks may be scheduled while the
// kernel before it on the stream finishes, which hides the launch latency
// between the dependent kernels of a BiCGStab iteration; k starts with
// pdl_wait(), so it reads nothing before that kernel has completed.
template <class... KArgs, class... Args>
void launch_k(Core& c, void (*k)(KArgs...), int grid, int block, Args... args)
{
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.stream = c.stream;
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = c.pdl_launch ? 1 : 0;
    EQG_CUDA(cudaLaunchKernelEx(&cfg, k, args...));
}

// Chooses the cluster size of the fused coarse cycle for one precision;
// called before any stream capture.
template <class T, class M>
void prepare_tail(Core& c, SolverAnalysis& an)
{
    if (an.tail_first < 0) return;
    if (c.param_i("linsolver_tail_trace", 0) && !an.tail_trace) {
        an.tail_trace = c.allocN<long long>(kTraceMax);
        EQG_CUDA(cudaMemsetAsync(an.tail_trace->ptr, 0, kTraceMax * sizeof(long long), c.stream));
    }
    const int mode = pc_mode<T, M>();
    int& cl = an.tail_cluster[mode];
    const int bs = an.levels[an.tail_first].bs;
    if (!cl) WITH_BS(bs, WITH_KMAX(an.tail_kmax, cl = tail_cluster_size<BS, KK, T, M>(c)));
    int bytes = 0;
    an.tail_local[mode] = plan_local<T, M>(c, an, bytes, nullptr);
    an.last_mode = mode;
}

// z = V-cycle(r) from level tail_first down, as one mg_tail_kernel launch.
template <class T, class M>
void launch_tail(Core& c, const SolverAnalysis& an, const T* r, T* z, const KScal* sc, int skip_if_s)
{
    TailParams<T, M> p;
    auto region = [&](const void* ptr, int64_t bytes) {
        if (p.nregions < kMaxPrefetch && bytes >= 16) p.reg[p.nregions++] = PrefetchRegion{ptr, (unsigned long long)bytes};
    };
    for (size_t l = an.tail_first; l < an.levels.size(); ++l) {
        const Level& L = an.levels[l];
        region(L.sell_ptr->ptr, ((L.nb + 31) / 32 + 1) * 4);
        region(L.sell_col->ptr, L.sell_size * 4);
        region(L.sell_len->ptr, (int64_t)L.nb * 4);
        region(L.sell_dk->ptr, (int64_t)L.nb * 4);
        region(level_a<M>(L), L.vals * (int64_t)sizeof(M));
        if (L.coarsest) {
            region(level_inv<M>(L), (int64_t)L.n * L.n * (int64_t)sizeof(M));
        } else {
            region(level_lu<M>(L), L.vals * (int64_t)sizeof(M));
            region(L.aggb->ptr, (int64_t)L.nb * 4);
            region(L.mpad->ptr, (int64_t)an.levels[l + 1].n * kMembers * 4);
        }
        TailLevel<T, M>& t = p.lv[p.nlev++];
        t.nb = L.nb;
        t.n = L.n;
        t.coarsest = L.coarsest ? 1 : 0;
        t.m = L.view();
        t.a = level_a<M>(L);
        t.nstages = (int)L.stage_ptr.size() - 1;
        for (int s = 0; s <= t.nstages && s <= kTailStages; ++s) t.sp[s] = L.stage_ptr[s];
        if (L.coarsest) {
            t.inv = level_inv<M>(L);
        } else {
            t.lu = level_lu<M>(L);
            t.aggb = L.aggb->as<int>();
            t.mpad = L.mpad->as<int>();
        }
        t.r = level_vec<T>(L, 0);
        t.z = level_vec<T>(L, 1);
        t.t = level_vec<T>(L, 2);
        t.w = level_vec<T>(L, 3);
    }
    if (an.tail_trace) p.trace = an.tail_trace->as<long long>();
    p.alpha = an.mg_alpha;
    p.local_first = p.nlev;
    int smem = 0;
    if (an.tail_local[pc_mode<T, M>()] < p.nlev) plan_local<T, M>(c, an, smem, &p);
    const int cl = an.tail_cluster[pc_mode<T, M>()];
    if (cl <= 0) fail(EQG_ERR_DEVICE, "fused coarse cycle launched before its cluster size was chosen");
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[2];
    cfg.gridDim = dim3(cl);
    cfg.blockDim = dim3(kTailThreads);
    cfg.dynamicSmemBytes = (size_t)smem;
    cfg.stream = c.stream;
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = cl;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    attr[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[1].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = c.pdl_launch ? 2 : 1;
    // algorithmic bytes: every fused level's matrix, factors and index
    // arrays once (the data the bulk prefetch fetches) and its four vectors
    double tail_bytes = 0.0;
    for (size_t l = an.tail_first; l < an.levels.size(); ++l) {
        const Level& L = an.levels[l];
        tail_bytes += (L.coarsest ? (double)L.n * L.n : 2.0 * L.vals) * sizeof(M) + 4.0 * L.sell_size +
                      8.0 * L.nb + 4.0 * L.n * sizeof(T);
    }
    WITH_BS(an.levels[an.tail_first].bs, WITH_KMAX(an.tail_kmax, launch(c, "mg_tail", [&] {
                EQG_CUDA(cudaLaunchKernelEx(&cfg, mg_tail_kernel<BS, KK, T, M>, p, r, z, sc, skip_if_s));
            }, tail_bytes)));
}

// Prints the steps of the last fused coarse cycle (linsolver_tail_trace=1):
// SM clock cycles from the end of one step to the end of the next, named in
// the kernel's order.
void report_tail_trace(Core& c, const SolverAnalysis& an)
{
    if (!an.tail_trace || an.tail_first < 0) return;
    std::vector<long long> t(kTraceMax);
    c.sync();
    EQG_CUDA(cudaMemcpy(t.data(), an.tail_trace->ptr, kTraceMax * sizeof(long long), cudaMemcpyDeviceToHost));
    std::vector<std::string> names;
    const int last = (int)an.levels.size() - 1;
    auto ilu = [&](int l) {
        const int ns = (int)an.levels[l].stage_ptr.size() - 1;
        for (int s = 1; s < ns; ++s) names.push_back("L" + std::to_string(l) + ".lower" + std::to_string(s));
        for (int s = ns >= 2 ? ns - 2 : 0; s >= 0 && ns > 0; --s)
            names.push_back("L" + std::to_string(l) + ".upper" + std::to_string(s));
    };
    const int lf = an.tail_first + an.tail_local[an.last_mode];  // first shared-memory level (last + 1: none)
    int l = an.tail_first;
    for (; l < lf; ++l) {
        if (an.levels[l].coarsest || l == last) {
            names.push_back("L" + std::to_string(l) + ".dense");
            break;
        }
        ilu(l);
        names.push_back("L" + std::to_string(l) + ".residual");
        if (l + 1 < lf) names.push_back("L" + std::to_string(l) + ".restrict");
    }
    if (l == lf && lf <= last)
        names.push_back("L" + std::to_string(lf - 1) + ".restrict+L" + std::to_string(lf) + "-L" +
                        std::to_string(last) + ".shared");
    for (--l; l >= an.tail_first; --l) {
        names.push_back("L" + std::to_string(l) + ".prolong");
        names.push_back("L" + std::to_string(l) + ".residual");
        ilu(l);
    }
    const int nsteps = std::min((int)names.size(), kTraceMax - 1);
    int khz = 0;
    cudaDeviceGetAttribute(&khz, cudaDevAttrClockRate, c.device);
    std::printf("        fused coarse cycle: %lld SM cycles (%.1f us at %.0f MHz), per step:",
                t[nsteps] - t[0], khz > 0 ? (t[nsteps] - t[0]) / (khz * 1e-3) : 0.0, khz * 1e-3);
    for (int i = 0; i < nsteps; ++i) std::printf(" %s=%lld", names[i].c_str(), t[i + 1] - t[i]);
    std::printf("\n");
}

// out = M^{-1} b for the block ILU(0) factors of one level; with zadd,
// zadd += out as rows finish.  One kernel per stage: forward sweeps of
// stages 1 .. S-1 (the last one finishing its rows), then backward sweeps
// of stages S-2 .. 0.
template <class T, class M>
void ilu_apply(Core& c, const Level& L, const T* b, T* out, T* zadd, const KScal* sc, int skip_if_s)
{
    const M* lu = level_lu<M>(L);
    const int ns = (int)L.stage_ptr.size() - 1;
    if (ns <= 0) return;
    const int r_first = L.stage_ptr[1];
    // algorithmic bytes of a stage: its off-diagonal blocks on the swept
    // side, its inverted diagonal blocks where rows finish, 4 bytes per row
    // (diagonal position), its rows of b or y read and of out written, the
    // other stages' values it gathers (counted as one vector of the stage's
    // size) and zadd read and written where rows finish
    const double vrow = (double)L.bs * sizeof(T);
    for (int s = 1; s < ns; ++s) {
        const int r0 = L.stage_ptr[s], r1 = L.stage_ptr[s + 1];
        const int last = s == ns - 1;
        const double bytes = block_bytes<M>(L, L.stage_lower[s]) +
                             (last ? (double)(r1 - r0) * L.bs * L.bs * sizeof(M) : 0.0) +
                             (r1 - r0) * (4.0 + vrow * ((last && zadd) ? 5.0 : 3.0));
        WITH_BS(L.bs, WITH_KMAX(L.kmax, launch(c, "bilu_lower", [&] {
                    launch_k(c, bilu_lower_kernel<BS, KK, T, M>, blocksFor(r1 - r0, L.threads), L.threads, r0, r1,
                             r_first, last,
                             L.view(), lu, b, out, last ? zadd : nullptr, sc, skip_if_s);
                }, bytes)));
    }
    for (int s = ns >= 2 ? ns - 2 : 0; s >= 0; --s) {
        const int r0 = L.stage_ptr[s], r1 = L.stage_ptr[s + 1];
        const double bytes = block_bytes<M>(L, L.stage_upper[s]) + (double)(r1 - r0) * L.bs * L.bs * sizeof(M) +
                             (r1 - r0) * (8.0 + vrow * (zadd ? 5.0 : 3.0));
        WITH_BS(L.bs, WITH_KMAX(L.kmax, launch(c, "bilu_upper", [&] {
                    launch_k(c, bilu_upper_kernel<BS, KK, T, M>, blocksFor(r1 - r0, L.threads), L.threads, r0, r1,
                             (int)(s == 0),
                             L.view(), lu, b, out, zadd, sc, skip_if_s);
                }, bytes)));
    }
}

// out = b - A x (block rows below r_zero: 0)
template <class T, class M>
void level_residual(Core& c, const Level& L, const T* x, const T* b, T* out, int r_zero, const KScal* sc,
                    int skip_if_s)
{
    // rows from r_zero: their blocks and lengths, b read and out written;
    // x read once
    const int64_t skipped = r_zero > 0 && !L.stage_lower.empty()
                                ? L.stage_lower[0] + L.stage_upper[0] + (L.stage_ptr[1] - L.stage_ptr[0])
                                : 0;
    const double bytes = block_bytes<M>(L, L.blocks - skipped) +
                         (L.nb - r_zero) * (4.0 + 2.0 * L.bs * sizeof(T)) + (double)L.n * sizeof(T);
    WITH_BS(L.bs, WITH_KMAX(L.kmax, launch(c, "mg_residual", [&] {
                launch_k(c, mg_residual_kernel<BS, KK, T, M>, blocksFor(L.nb, L.threads), L.threads, L.nb, r_zero,
                         L.view(),
                         level_a<M>(L), x, b, out, sc, skip_if_s);
            }, bytes)));
}

// z = V-cycle(r) on level l.
template <class T, class M>
void vcycle(Core& c, const SolverAnalysis& an, size_t l, const T* r, T* z, const KScal* sc, int skip)
{
    if ((int)l == an.tail_first) {
        launch_tail<T, M>(c, an, r, z, sc, skip);
        return;
    }
    const Level& L = an.levels[l];
    if (L.coarsest) {
        launch(c, "mg_dense_apply", [&] {
            launch_k(c, dense_apply_kernel<T, M>, 1, kThreads, L.n, level_inv<M>(L), r, z, sc, skip);
        }, (double)L.n * L.n * sizeof(M) + 2.0 * L.n * sizeof(T));
        return;
    }
    const Level& C = an.levels[l + 1];
    T* t = level_vec<T>(L, 2);
    T* w = level_vec<T>(L, 3);
    T* rc = level_vec<T>(C, 0);
    T* zc = level_vec<T>(C, 1);
    // pre-smoothing z = M^{-1} r.  The first stage's block rows have no
    // lower part and were solved last, against the final z of every other
    // stage, with their rows of A unchanged by the factorization
    // (D_R^{-1} = A_RR^{-1}, U_RJ = A_RJ): their residual r - A z is zero.
    // Those rows of t are not stored: the restriction skips them and the
    // A P up-leg takes them as zero.
    const int r_zero = L.stage_ptr.size() > 1 ? L.stage_ptr[1] : 0;
    ilu_apply<T, M>(c, L, r, z, nullptr, sc, skip);
    level_residual<T, M>(c, L, z, r, t, r_zero, sc, skip);
    launch(c, "mg_restrict", [&] {
        launch_k(c, mg_restrict_kernel<T>, blocksFor(C.n, L.threads), L.threads, C.n, (const int*)L.mptr->as<int>(),
                 (const int*)L.midx->as<int>(), (const T*)t, r_zero * L.bs, rc, sc, skip);
    }, (double)(L.n - r_zero * L.bs) * sizeof(T) + (double)C.n * sizeof(T) + 4.0 * (C.n + 1) + 4.0 * L.n);
    vcycle<T, M>(c, an, l + 1, rc, zc, sc, skip);
    // coarse correction z += alpha P zc and its residual t = r - A z, then
    // post-smoothing z += M^{-1} t.  Through A P with FP64 vectors only: with
    // the FP32 vectors of "refine" the updated residual drifts from r - A z
    // and the iterations per time step rose from 203 to 254 (128x128x64)
    if (L.ap_slots > 0 && sizeof(T) == sizeof(double)) {
        // A P blocks and row lengths, aggregates, zc once, z and t (rows
        // from r_zero) read and written
        const double bytes = block_bytes<M>(L, L.ap_blocks) + 8.0 * L.nb + (double)C.n * sizeof(T) +
                             2.0 * L.n * sizeof(T) + 2.0 * (L.n - r_zero * L.bs) * sizeof(T);
        WITH_BS(L.bs, WITH_KMAX(L.ap_kmax, launch(c, "mg_correct", [&] {
                    launch_k(c, mg_correct_kernel<BS, KK, T, M>, blocksFor(L.nb, L.threads), L.threads, L.nb, r_zero,
                             L.ap_view(),
                             level_ap<M>(L), (const int*)L.aggb->as<int>(), (const T*)zc, z, t, an.mg_alpha, sc, skip);
                }, bytes)));
    } else {
        WITH_BS(L.bs, launch(c, "mg_prolong", [&] {
                    launch_k(c, mg_prolong_kernel<BS, T>, blocksFor(L.nb, L.threads), L.threads, L.nb,
                             (const int*)L.aggb->as<int>(), (const T*)zc, z, an.mg_alpha, sc, skip);
                }, 4.0 * L.nb + (double)C.n * sizeof(T) + 2.0 * L.n * sizeof(T)));
        level_residual<T, M>(c, L, z, r, t, 0, sc, skip);
    }
    ilu_apply<T, M>(c, L, t, w, z, sc, skip);
}

template <class T, class M>
void precondition(Core& c, const SolverAnalysis& an, const T* in, T* out, const KScal* sc, int skip_if_s)
{
    if (an.multigrid) vcycle<T, M>(c, an, 0, in, out, sc, skip_if_s);
    else ilu_apply<T, M>(c, an.levels[0], in, out, nullptr, sc, skip_if_s);
}

// out = M^{-1} in; with pc32 (FP64 vectors only) from the FP32 copies of the
// preconditioner's matrices.
template <class T>
void apply_pc(Core& c, const SolverAnalysis& an, const T* in, T* out, const KScal* sc, int skip_if_s, bool pc32)
{
    if constexpr (sizeof(T) == sizeof(double)) {
        if (pc32) {
            precondition<double, float>(c, an, in, out, sc, skip_if_s);
            return;
        }
    }
    precondition<T, T>(c, an, in, out, sc, skip_if_s);
}

// ---- autotuning of launch shapes ---------------------------------------------
// Per Jacobian pattern and precision, the threads per block of every
// launch-per-step V-cycle level's kernels (128, 256 or 512) and the cluster
// size of the fused coarse cycle (the largest the device schedules, half or
// a quarter of it) are chosen by timing preconditioner applications on the
// solve's right-hand side (CUDA events on the runtime stream), before the
// first BiCGStab iteration and its graph capture; one level at a time, then
// the cluster.  A row's operations do not depend on the launch shape, so the
// results are the same for every choice.  Choices are kept for the process,
// keyed by device, system and hierarchy sizes and precision, and read from
// and written to the JSON file linsolver_tune_file (or $EQG_TUNE_FILE) when
// one is named.  linsolver_autotune=0 keeps 256 threads and the largest
// cluster.
struct TuneChoice {
    std::vector<int> threads;
    int cluster = 0;
};
std::mutex g_tune_mutex;
std::map<std::string, TuneChoice> g_tune_cache;
std::map<std::string, bool> g_tune_files_read;

// The file holds one entry per line:
//   "<key>": {"threads": [t0, t1, ...], "cluster": c},
void tune_file_read(const std::string& path)
{
    std::ifstream f(path.c_str());
    std::string line;
    while (std::getline(f, line)) {
        const size_t k0 = line.find('"'), k1 = line.find('"', k0 + 1);
        const size_t a0 = line.find('['), a1 = line.find(']');
        const size_t c0 = line.find("\"cluster\":");
        if (k0 == std::string::npos || k1 == std::string::npos || a0 == std::string::npos ||
            a1 == std::string::npos || c0 == std::string::npos)
            continue;
        TuneChoice t;
        std::string nums = line.substr(a0 + 1, a1 - a0 - 1);
        for (char& ch : nums)
            if (ch == ',') ch = ' ';
        std::istringstream in(nums);
        int v = 0;
        while (in >> v) t.threads.push_back(v);
        t.cluster = std::atoi(line.c_str() + c0 + 10);
        g_tune_cache.emplace(line.substr(k0 + 1, k1 - k0 - 1), t);
    }
}

void tune_file_write(const std::string& path)
{
    const std::string tmp = path + ".tmp";
    {
        std::ofstream f(tmp.c_str());
        f << "{\n";
        size_t i = 0;
        for (auto& kv : g_tune_cache) {
            f << "\"" << kv.first << "\": {\"threads\": [";
            for (size_t j = 0; j < kv.second.threads.size(); ++j) f << (j ? ", " : "") << kv.second.threads[j];
            f << "], \"cluster\": " << kv.second.cluster << "}" << (++i < g_tune_cache.size() ? "," : "") << "\n";
        }
        f << "}\n";
    }
    std::rename(tmp.c_str(), path.c_str());
}

template <class T, class M>
void autotune(Core& c, SolverAnalysis& an, const T* b, T* out, const KScal* sc)
{
    const int mode = pc_mode<T, M>();
    if (an.tuned[mode]) return;
    an.tuned[mode] = true;
    if (c.param_i("linsolver_autotune", 1) == 0) return;
    // levels with launch-per-step kernels: all but the fused ones and a
    // dense coarsest level
    std::vector<int> lv;
    for (size_t l = 0; l < an.levels.size(); ++l) {
        if (an.multigrid && an.tail_first >= 0 && (int)l >= an.tail_first) break;
        if (an.levels[l].coarsest) break;
        lv.push_back((int)l);
        if (!an.multigrid) break;
    }
    cudaDeviceProp prop;
    EQG_CUDA(cudaGetDeviceProperties(&prop, c.device));
    std::ostringstream key;
    key << prop.name << "; n " << an.n << "; nnz " << an.nnz << "; bs " << an.levels[0].bs << "; levels";
    for (auto& L : an.levels) key << " " << L.n;
    key << "; fused from " << an.tail_first << "; precision " << mode;
    std::string file = c.param_s("linsolver_tune_file", "");
    if (file.empty() && std::getenv("EQG_TUNE_FILE")) file = std::getenv("EQG_TUNE_FILE");
    {
        std::lock_guard<std::mutex> lock(g_tune_mutex);
        if (!file.empty() && !g_tune_files_read[file]) {
            tune_file_read(file);
            g_tune_files_read[file] = true;
        }
        auto it = g_tune_cache.find(key.str());
        if (it != g_tune_cache.end() && it->second.threads.size() == lv.size()) {
            for (size_t i = 0; i < lv.size(); ++i) an.levels[lv[i]].threads = it->second.threads[i];
            if (an.tail_first >= 0 && it->second.cluster > 0 && it->second.cluster <= an.tail_cluster[mode])
                an.tail_cluster[mode] = it->second.cluster;
            return;
        }
    }
    // tuning launches are not part of a kernel profile
    const std::string timed = c.timed_kernel;
    c.timed_kernel.clear();
    cudaEvent_t e0, e1;
    EQG_CUDA(cudaEventCreate(&e0));
    EQG_CUDA(cudaEventCreate(&e1));
    auto measure = [&] {
        precondition<T, M>(c, an, b, out, sc, 0);
        float best = 1e30f;
        for (int rep = 0; rep < 2; ++rep) {
            EQG_CUDA(cudaEventRecord(e0, c.stream));
            for (int k = 0; k < 4; ++k) precondition<T, M>(c, an, b, out, sc, 0);
            EQG_CUDA(cudaEventRecord(e1, c.stream));
            EQG_CUDA(cudaEventSynchronize(e1));
            float ms = 0.f;
            EQG_CUDA(cudaEventElapsedTime(&ms, e0, e1));
            best = std::min(best, ms);
        }
        return best;
    };
    float cur = measure();
    const float first = cur;
    for (int l : lv) {
        Level& L = an.levels[l];
        int best_t = L.threads;
        for (int t : {128, 256, 512}) {
            if (t == best_t) continue;
            L.threads = t;
            const float ms = measure();
            if (ms < cur) {
                cur = ms;
                best_t = t;
            }
        }
        L.threads = best_t;
    }
    int& cl = an.tail_cluster[mode];
    if (an.tail_first >= 0 && cl > 1) {
        const int top = cl;
        int best_c = cl;
        for (int cand : {top / 2, top / 4}) {
            if (cand < 2) continue;
            cl = cand;
            const float ms = measure();
            if (ms < cur) {
                cur = ms;
                best_c = cand;
            }
        }
        cl = best_c;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    c.timed_kernel = timed;
    TuneChoice t;
    for (int l : lv) t.threads.push_back(an.levels[l].threads);
    t.cluster = an.tail_first >= 0 ? cl : 0;
    if (c.verbose > 2) {
        std::printf("        autotune: %.3f -> %.3f ms per V-cycle; threads per level:", first / 4, cur / 4);
        for (int v : t.threads) std::printf(" %d", v);
        std::printf("; cluster %d\n", t.cluster);
    }
    std::lock_guard<std::mutex> lock(g_tune_mutex);
    g_tune_cache[key.str()] = t;
    if (!file.empty()) tune_file_write(file);
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
    const int nbr = blocksFor(L0.nb, kThreads, kRedBlocks);
    const double vb = (double)n * sizeof(T);  // one vector
    const double spmv_bytes = block_bytes<T>(L0, L0.blocks) + 4.0 * L0.nb + 3.0 * vb;
    launch(c, "bicg_init", [&] {
        bicg_init_kernel<T><<<nb, kThreads, 0, c.stream>>>(v.b, v.r, v.rhat, v.p, v.v, v.x, n, part, cnt, sc, tol * tol);
    }, 6.0 * vb);
    auto iteration = [&] {
        launch(c, "bicg_p", [&] {
            launch_k(c, bicg_p_kernel<T>, blocksFor(n), kThreads, (const T*)v.r, (const T*)v.v, v.p, n,
                     (const KScal*)sc);
        }, 4.0 * vb);
        apply_pc<T>(c, an, v.p, v.ph, sc, 0, pc32);
        WITH_BS(L0.bs, WITH_KMAX(L0.kmax, launch(c, "bicg_spmv_alpha", [&] {
                    launch_k(c, bicg_spmv_alpha_kernel<BS, KK, T>, nbr, kThreads, L0.view(), a, (const T*)v.ph,
                             (const T*)v.rhat, v.v, L0.nb, part, cnt, sc);
                }, spmv_bytes)));
        launch(c, "bicg_s", [&] {
            launch_k(c, bicg_s_kernel<T>, nb, kThreads, (const T*)v.r, (const T*)v.v, v.s, n, part, cnt, sc);
        }, 3.0 * vb);
        apply_pc<T>(c, an, v.s, v.sh, sc, 1, pc32);
        WITH_BS(L0.bs, WITH_KMAX(L0.kmax, launch(c, "bicg_spmv_omega", [&] {
                    launch_k(c, bicg_spmv_omega_kernel<BS, KK, T>, nbr, kThreads, L0.view(), a, (const T*)v.sh,
                             (const T*)v.s, v.t, L0.nb, part, cnt, sc);
                }, spmv_bytes)));
        launch(c, "bicg_xr", [&] {
            launch_k(c, bicg_xr_kernel<T>, nb, kThreads, (const T*)v.ph, (const T*)v.sh, (const T*)v.s,
                     (const T*)v.t, (const T*)v.rhat, v.x, v.r, n, part, cnt, sc);
        }, 8.0 * vb);
    };
    // launch shapes of the preconditioner, once per analysis and precision
    // (before the graph capture below)
    if (an.multigrid || an.levels[0].n > 0) {
        if constexpr (sizeof(T) == sizeof(double)) {
            if (pc32) autotune<double, float>(c, an, v.b, v.ph, sc);
            else autotune<double, double>(c, an, v.b, v.ph, sc);
        } else {
            autotune<float, float>(c, an, v.b, v.ph, sc);
        }
    }
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
        // diverged: the residual 1e8 times the right-hand side's norm
        // (BiCGStab's excursions on systems it solves stay far below)
        const double bb = tol > 0 ? h.thr / (tol * tol) : 0.0;
        if (bb > 0 && h.rr > 1e16 * bb) break;
    }
    res.converged = h.status == ST_CONV;
    res.iterations = h.iterations;
    const double b2 = tol > 0 ? h.thr / (tol * tol) : 0.0;
    res.rel_residual = b2 > 0 ? std::sqrt(h.rr / b2) : 0.0;
    return res;
}

void factor_level(Core& c, const Level& L, int* status)
{
    EQG_CUDA(cudaMemcpyAsync(L.lus64->ptr, L.as64->ptr, (size_t)L.vals * 8, cudaMemcpyDeviceToDevice, c.stream));
    const int ns = (int)L.stage_ptr.size() - 1;
    for (int s = 0; s < ns; ++s) {
        const int r0 = L.stage_ptr[s], r1 = L.stage_ptr[s + 1];
        // the stage's blocks read and written, the upper blocks of the rows
        // they eliminate read once (counted as the stage's own upper blocks)
        const int64_t stage_blocks = L.stage_lower[s] + L.stage_upper[s] + (r1 - r0);
        const double bytes = block_bytes<double>(L, stage_blocks) + 8.0 * L.bs * L.bs * stage_blocks +
                             block_bytes<double>(L, L.stage_upper[s]) + 8.0 * (r1 - r0);
        WITH_BS(L.bs, launch(c, "bilu_factor", [&] {
                    bilu_factor_stage_kernel<BS><<<blocksFor(r1 - r0), kThreads, 0, c.stream>>>(
                        r0, r1, L.view(), L.lus64->as<double>(), status);
                }, bytes));
    }
}

void to_float(Core& c, const Buf& src, Buf& dst, int64_t n)
{
    if (!dst) dst = c.allocN<float>((size_t)(n > 0 ? n : 1));
    launch(c, "to_float",
           [&] { to_float_kernel<<<blocksFor(n), kThreads, 0, c.stream>>>(src->as<double>(), dst->as<float>(), n); },
           12.0 * n);
}

}  // namespace

namespace {

// One solve with the analysis in `slot` (built on first use; without
// multigrid when allow_multigrid is false).
SolveResult solve_with(Core& c, const PatternP& p, std::shared_ptr<SolverAnalysis>& slot, bool allow_multigrid,
                       const double* jval, const double* rhs, double* xout)
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
    // iterations per graph launch between host convergence checks: after
    // convergence the rest of a chunk still launches (its kernels return at
    // once); on 128x128x64, 4 beat 8 and 16 (72.7, 73.3, 74.2 ms of Krylov
    // time per step)
    const int check_every = std::max(1, c.param_i("linsolver_check_every", 4));

    if (!slot || slot->natural != natural) slot = analyse(c, *p, natural, allow_multigrid);
    c.pdl_launch = c.param_i("linsolver_pdl", 1) != 0;
    SolverAnalysis& an = *slot;
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
        // gather_rows=1: one block row per thread (measured slower on the
        // 128x128x64 Jacobian: 0.74 against 0.64 ms per gather)
        if (c.param_i("gather_rows", 0) != 0) {
            const int* sp = L0.sell_ptr->as<int>();
            if (L0.bs == 1)
                gather_rows_kernel<1><<<blocksFor(L0.nb + 32), kThreads, 0, c.stream>>>(L0.nb, sp, jval, an.vmap->as<int>(),
                                                                                  L0.as64->as<double>());
            else if (L0.bs == 2)
                gather_rows_kernel<4><<<blocksFor(L0.nb + 32), kThreads, 0, c.stream>>>(L0.nb, sp, jval, an.vmap->as<int>(),
                                                                                  L0.as64->as<double>());
            else
                gather_rows_kernel<9><<<blocksFor(L0.nb + 32), kThreads, 0, c.stream>>>(L0.nb, sp, jval, an.vmap->as<int>(),
                                                                                  L0.as64->as<double>());
        } else {
            gather_values_kernel<<<blocksFor(L0.vals), kThreads, 0, c.stream>>>(jval, an.vmap->as<int>(),
                                                                                L0.as64->as<double>(), L0.vals);
        }
    }, 12.0 * L0.vals + 8.0 * an.nnz);
    for (size_t l = 1; l < an.levels.size(); ++l) {
        const Level& F = an.levels[l - 1];
        const Level& C = an.levels[l];
        EQG_CUDA(cudaMemsetAsync(C.as64->ptr, 0, (size_t)C.vals * sizeof(double), c.stream));
        // the finer level's entries and their gather indices once, the
        // coarse entries (list bounds, position, value) once
        launch(c, "mg_galerkin", [&] {
            galerkin_kernel<<<blocksFor(C.nnz), kThreads, 0, c.stream>>>(C.nnz, C.gptr->as<int>(), C.gidx->as<int>(),
                                                                         C.gpos->as<int>(), F.as64->as<double>(),
                                                                         C.as64->as<double>());
        }, 12.0 * F.nnz + 16.0 * C.nnz);
    }
    for (auto& L : an.levels)
        if (L.ap_slots > 0) {
            launch(c, "mg_ap_values", [&] {
                ap_values_kernel<<<blocksFor(L.ap_slots * L.bs * L.bs), kThreads, 0, c.stream>>>(
                    L.ap_slots, L.bs * L.bs, L.ap_gptr->as<int>(), L.ap_gidx->as<int>(), L.as64->as<double>(),
                    L.ap64->as<double>());
            }, block_bytes<double>(L, L.blocks) + 8.0 * L.ap_slots + 8.0 * L.bs * L.bs * L.ap_slots);
        }
    EQG_CUDA(cudaMemsetAsync(an.factor_status->ptr, 0, sizeof(int), c.stream));
    for (auto& L : an.levels) {
        if (L.coarsest) {
            WITH_BS(L.bs, launch(c, "mg_dense_inverse", [&] {
                const size_t smem = ((size_t)L.n * L.n + L.n) * sizeof(double);
                // one value for every call: runtimes on other host threads set
                // the same attribute of the same kernel, and a smaller value
                // set between this call's set and its launch would fail it
                const size_t most = ((size_t)kCoarsest * kCoarsest + kCoarsest) * sizeof(double);
                EQG_CUDA(cudaFuncSetAttribute(dense_inverse_kernel<BS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              (int)std::max(smem, most)));
                dense_inverse_kernel<BS><<<1, 1024, smem, c.stream>>>(L.nb, L.view(), L.as64->as<double>(),
                                                                     L.inv64->as<double>(), an.factor_status->as<int>());
            }, 16.0 * L.n * L.n));
        } else {
            factor_level(c, L, an.factor_status->as<int>());
        }
    }
    Vecs<double> v = vecs<double>(an.vec64->as<double>(), n);
    launch(c, "permute",
           [&] { permute_kernel<<<blocksFor(n), kThreads, 0, c.stream>>>(rhs, L0.perm->as<int>(), v.b, n); },
           20.0 * n);
    if (mixed || refine) {
        for (auto& L : an.levels) {
            to_float(c, L.as64, L.as32, L.vals);
            if (L.ap_slots > 0) to_float(c, L.ap64, L.ap32, L.ap_slots * L.bs * L.bs);
            if (L.coarsest) to_float(c, L.inv64, L.inv32, (int64_t)L.n * L.n);
            else to_float(c, L.lus64, L.lus32, L.vals);
            if (refine && !L.v32) L.v32 = c.allocN<float>((size_t)4 * (L.n > 0 ? L.n : 1));
        }
        if (refine && !an.vec32) an.vec32 = c.allocN<float>((size_t)10 * vec_stride(n));
        if (refine) prepare_tail<float, float>(c, an);
        else prepare_tail<double, float>(c, an);
    } else {
        prepare_tail<double, double>(c, an);
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
        const int nbr = blocksFor(L0.nb, kThreads, kRedBlocks);
        k_fill(c, v.x, 0.0, n);
        Buf rr_dev = c.allocN<double>(2);
        launch(c, "sumsq",
               [&] { sumsq_kernel<<<nb, kThreads, 0, c.stream>>>(v.b, n, part, cnt, rr_dev->as<double>()); },
               8.0 * n);
        auto residual = [&] {
            WITH_BS(L0.bs, WITH_KMAX(L0.kmax, launch(c, "residual", [&] {
                        residual_kernel<BS, KK><<<nbr, kThreads, 0, c.stream>>>(
                            L0.view(), L0.as64->as<double>(), v.x, v.b, v.r, w.b, L0.nb, part, cnt,
                            rr_dev->as<double>() + 1);
                    }, block_bytes<double>(L0, L0.blocks) + 4.0 * L0.nb + 28.0 * n)));
        };
        residual();
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
                   [&] { add_float_kernel<<<blocksFor(n), kThreads, 0, c.stream>>>(v.x, w.x, n); }, 20.0 * n);
            residual();
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
    report_tail_trace(c, an);
    launch(c, "unpermute",
           [&] { unpermute_kernel<<<blocksFor(n), kThreads, 0, c.stream>>>(v.x, L0.perm->as<int>(), xout, n); },
           20.0 * n);
    res.block_size = L0.bs;
    res.blocks = L0.blocks;
    return res;
}

}  // namespace

// A solve that the multigrid-preconditioned BiCGStab does not converge (a
// breakdown, a zero pivot, or the iteration limit) is repeated once with
// block ILU(0) alone (linsolver_fallback=1, the default): on systems that
// are singular on both sides, such as the conservation form of the
// two-phase equations, the V-cycle's coarse corrections can keep the
// iteration from converging where the single-level preconditioner does.
SolveResult linear_solve(Core& c, const PatternP& p, const double* jval, const double* rhs, double* xout)
{
    SolveResult res = solve_with(c, p, p->analysis, true, jval, rhs, xout);
    res.multigrid = p->analysis && p->analysis->multigrid;
    if (res.converged || !res.multigrid || c.param_i("linsolver_fallback", 1) == 0) return res;
    if (c.verbose > 0)
        std::printf("        linear solve: multigrid did not converge after %d iterations; block ILU(0) alone\n",
                    res.iterations);
    SolveResult again = solve_with(c, p, p->analysis_fallback, false, jval, rhs, xout);
    again.iterations += res.iterations;
    again.fallbacks = 1;
    return again;
}

}  // namespace eqg

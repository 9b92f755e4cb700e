// Forward-mode AD on the device: Jacobian sparsity patterns and values.
//
// Semantics follow Opm::AutoDiffBlock over Eigen sparse matrices, as used by
// the reference serial backend (equelleTypes.hpp:67-84; rules restated in
// backends/cuda/src/collOfScalar.cu:273-401):
//   - sum/difference: union pattern, explicit zeros kept;
//   - product/quotient/sqrt/sign: row scaling diag(w) J, pattern unchanged,
//     then the union for two operands;
//   - operator matrix times ADB (gradient, divergence, On, Extend, ESpan
//     subset/superset): conservative sparse product M J, entry (i,j)
//     accumulated over M's row entries in ascending source order.
// Output patterns are computed once, symbolically, and cached by the ids of
// the input patterns (and operator), so each Newton iteration after the
// first only runs the numeric kernels.
#include "eqg_internal.cuh"

#include <cub/cub.cuh>

#include <climits>
#include <cstring>

namespace eqg {

namespace {

#define GRID_STRIDE(i, n) \
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < (n); i += (int64_t)gridDim.x * blockDim.x)

// ---------------------------------------------------------------------------
// Elementwise Jacobian rules.
// ---------------------------------------------------------------------------
struct Rule {
    int rule;
    const double* va;
    const double* vb;
    const double* vout;
    const uint8_t* mask;
    double s;
};

__device__ __forceinline__ void rule_weights(const Rule& r, int64_t i, double& wa, double& wb, double& post)
{
    wa = 1.0;
    wb = 1.0;
    post = 1.0;
    switch (r.rule) {
    case JR_ADD: break;
    case JR_SUB: wb = -1.0; break;
    case JR_MUL: {
        // D2*Ja + D1*Jb with D1 = diag(a), D2 = diag(b)
        const double a = r.va ? r.va[i] : r.s;
        const double b = r.vb ? r.vb[i] : r.s;
        wa = b;
        wb = a;
        break;
    }
    case JR_DIV: {
        // D3*(D2*Ja - D1*Jb), D3 = diag(1/(b*b))
        const double a = r.va ? r.va[i] : r.s;
        const double b = r.vb ? r.vb[i] : r.s;
        wa = b;
        wb = -a;
        post = 1.0 / (b * b);
        break;
    }
    case JR_SCALE_CONST: wa = r.s; break;
    case JR_DIV_BY_CONST:
        wa = r.s;
        post = 1.0 / (r.s * r.s);
        break;
    case JR_SQRT: wa = 0.5 / r.vout[i]; break;
    case JR_SIGN: wa = r.va[i] >= 0.0 ? 1.0 : -1.0; break;
    case JR_NEG: wa = -1.0; break;
    case JR_SELECT: {
        const bool m = r.mask[i] != 0;
        wa = m ? 1.0 : 0.0;
        wb = m ? 0.0 : 1.0;
        break;
    }
    }
}


// The deferred rules of an operand applied to one of its stored values in
// row `row`, in order, each with the eager kernel's arithmetic.
__device__ __forceinline__ double apply_deferred(const Deferred& d, int64_t row, double x)
{
    for (int k = 0; k < d.n; ++k) {
        const DeferredRule& q = d.r[k];
        const Rule r{q.rule, q.va, q.vb, q.vout, q.mask, q.s};
        double wa, wb, post;
        rule_weights(r, row, wa, wb, post);
        double acc = 0.0;
        acc += (q.side == 0 ? wa : wb) * x;
        x = post * acc;
    }
    return x;
}


// ---------------------------------------------------------------------------
// Conservative product M*J by K-way merge of the selected rows of J.
// ---------------------------------------------------------------------------
template <int KMAX>
struct Streams {
    int pos[KMAX], end[KMAX];
    double w[KMAX];

    __device__ __forceinline__ void load(int i, const int* mptr, const int* msrc, const double* mw, const int* jptr)
    {
        const int m0 = mptr[i];
        const int k = mptr[i + 1] - m0;
#pragma unroll
        for (int t = 0; t < KMAX; ++t) {
            if (t < k) {
                const int r = msrc[m0 + t];
                pos[t] = jptr[r];
                end[t] = jptr[r + 1];
                w[t] = mw ? mw[m0 + t] : 1.0;
            } else {
                pos[t] = 0;
                end[t] = 0;
                w[t] = 0.0;
            }
        }
    }

    __device__ __forceinline__ int next_col(const int* jcol) const
    {
        int c = INT_MAX;
#pragma unroll
        for (int t = 0; t < KMAX; ++t)
            if (pos[t] < end[t]) c = min(c, jcol[pos[t]]);
        return c;
    }

    __device__ __forceinline__ void advance(const int* jcol, int c)
    {
#pragma unroll
        for (int t = 0; t < KMAX; ++t)
            if (pos[t] < end[t] && jcol[pos[t]] == c) ++pos[t];
    }
};

template <int KMAX>
__global__ void spgemm_count_kernel(int n_out, const int* mptr, const int* msrc, const int* jptr, const int* jcol,
                                    int64_t* cnt)
{
    GRID_STRIDE(i, n_out)
    {
        Streams<KMAX> s;
        s.load((int)i, mptr, msrc, nullptr, jptr);
        int64_t count = 0;
        for (;;) {
            const int c = s.next_col(jcol);
            if (c == INT_MAX) break;
            ++count;
            s.advance(jcol, c);
        }
        cnt[i] = count;
    }
}

template <int KMAX>
__global__ void spgemm_fill_kernel(int n_out, const int* mptr, const int* msrc, const int* jptr, const int* jcol,
                                   const int* optr, int* ocol)
{
    GRID_STRIDE(i, n_out)
    {
        Streams<KMAX> s;
        s.load((int)i, mptr, msrc, nullptr, jptr);
        int o = optr[i];
        for (;;) {
            const int c = s.next_col(jcol);
            if (c == INT_MAX) break;
            ocol[o++] = c;
            s.advance(jcol, c);
        }
    }
}

template <int KMAX>
__global__ void spgemm_numeric_kernel(int n_out, const int* __restrict__ mptr, const int* __restrict__ msrc,
                                      const double* __restrict__ mw, const int* __restrict__ jptr,
                                      const int* __restrict__ jcol, const double* __restrict__ jval,
                                      const int* __restrict__ optr, const int* __restrict__ ocol,
                                      double* __restrict__ oval)
{
    GRID_STRIDE(i, n_out)
    {
        Streams<KMAX> s;
        s.load((int)i, mptr, msrc, mw, jptr);
        const int p1 = optr[i + 1];
        for (int p = optr[i]; p < p1; ++p) {
            const int c = ocol[p];
            double acc = 0.0;
#pragma unroll
            for (int t = 0; t < KMAX; ++t) {
                if (s.pos[t] < s.end[t] && jcol[s.pos[t]] == c) {
                    acc += s.w[t] * jval[s.pos[t]];
                    ++s.pos[t];
                }
            }
            oval[p] = acc;
        }
    }
}

// Position plan of M*J for one output pattern: for every output entry, the
// entries of J that the K-way merge adds into it, in the merge's order
// (stream t of M's row ascending), packed as t << kPlanShift | position in
// J.  Built once with the output pattern; the numeric product then runs one
// thread per output entry, with the same operations in the same order as
// spgemm_numeric_kernel.
constexpr int kPlanShift = 27;
constexpr int kPlanMask = (1 << kPlanShift) - 1;

template <int KMAX, bool COUNT>
__global__ void spgemm_plan_kernel(int n_out, const int* __restrict__ mptr, const int* __restrict__ msrc,
                                   const int* __restrict__ jptr, const int* __restrict__ jcol,
                                   const int* __restrict__ optr, const int* __restrict__ ocol,
                                   int64_t* __restrict__ cnt, const int* __restrict__ start,
                                   int* __restrict__ contrib)
{
    GRID_STRIDE(i, n_out)
    {
        Streams<KMAX> s;
        s.load((int)i, mptr, msrc, nullptr, jptr);
        const int p1 = optr[i + 1];
        for (int p = optr[i]; p < p1; ++p) {
            const int c = ocol[p];
            int n = 0;
            const int o = COUNT ? 0 : start[p];
#pragma unroll
            for (int t = 0; t < KMAX; ++t) {
                if (s.pos[t] < s.end[t] && jcol[s.pos[t]] == c) {
                    if (!COUNT) contrib[o + n] = (t << kPlanShift) | s.pos[t];
                    ++n;
                    ++s.pos[t];
                }
            }
            if (COUNT) cnt[p] = n;
        }
    }
}

__global__ void spgemm_planned_kernel(int64_t nnz, const int* __restrict__ rowidx, const int* __restrict__ mptr,
                                      const double* __restrict__ mw, const int* __restrict__ start,
                                      const int* __restrict__ contrib, const double* __restrict__ jval,
                                      double* __restrict__ oval, const int* __restrict__ msrc, const Deferred dj)
{
    GRID_STRIDE(e, nnz)
    {
        const int m0 = mptr[rowidx[e]];
        const int k1 = start[e + 1];
        double acc = 0.0;
        for (int k = start[e]; k < k1; ++k) {
            const int q = contrib[k];
            const int t = q >> kPlanShift;
            // J's value with its deferred rules, in J's row (M's source)
            const double jv = dj.n ? apply_deferred(dj, msrc[m0 + t], jval[q & kPlanMask]) : jval[q & kPlanMask];
            acc += mw[m0 + t] * jv;
        }
        oval[e] = acc;
    }
}

// y = M x, each row accumulated from 0.0 over ascending source entries.
__global__ void opmat_apply_kernel(int n_out, const int* __restrict__ mptr, const int* __restrict__ msrc,
                                   const double* __restrict__ mw, const double* __restrict__ x,
                                   double* __restrict__ y)
{
    GRID_STRIDE(i, n_out)
    {
        double acc = 0.0;
        const int e1 = mptr[i + 1];
        for (int e = mptr[i]; e < e1; ++e) acc += mw[e] * x[msrc[e]];
        y[i] = acc;
    }
}

__global__ void map_count_kernel(const int32_t* map, int64_t n, int64_t* cnt, int n_src, int32_t* err)
{
    GRID_STRIDE(i, n)
    {
        const int32_t m = map[i];
        if (m >= n_src) *err = 1;
        cnt[i] = m >= 0 ? 1 : 0;
    }
}

__global__ void map_fill_kernel(const int32_t* map, int64_t n, const int* ptr, int* src, double* w)
{
    GRID_STRIDE(i, n)
    {
        const int32_t m = map[i];
        if (m >= 0) {
            src[ptr[i]] = m;
            w[ptr[i]] = 1.0;
        }
    }
}

__global__ void identity_pattern_kernel(int n, int* rowptr, int* colind, double* ones)
{
    GRID_STRIDE(i, (int64_t)n + 1)
    {
        rowptr[i] = (int)i;
        if (i < n) {
            colind[i] = (int)i;
            if (ones) ones[i] = 1.0;
        }
    }
}

__global__ void ones_kernel(double* o, int64_t n)
{
    GRID_STRIDE(i, n) o[i] = 1.0;
}

__global__ void rowidx_kernel(int rows, const int* rowptr, int* rowidx)
{
    GRID_STRIDE(i, rows)
    {
        for (int e = rowptr[i]; e < rowptr[i + 1]; ++e) rowidx[e] = (int)i;
    }
}

__global__ void i64_to_rowptr_kernel(const int64_t* incl, int n, int* rowptr)
{
    GRID_STRIDE(i, (int64_t)n + 1) rowptr[i] = i == 0 ? 0 : (int)incl[i - 1];
}

// ---------------------------------------------------------------------------
// Elementwise Jacobian rules over patterns (operands read through their
// deferred rules da, db).
// ---------------------------------------------------------------------------
// Operands share the output pattern: one thread per nonzero.
__global__ void ew_flat_kernel(Rule r, const int* __restrict__ rowidx, const double* __restrict__ ja,
                               const double* __restrict__ jb, double* __restrict__ out, int64_t nnz,
                               const Deferred da, const Deferred db)
{
    GRID_STRIDE(e, nnz)
    {
        const int i = rowidx[e];
        double wa, wb, post;
        rule_weights(r, i, wa, wb, post);
        double acc = 0.0;
        if (ja) acc += wa * apply_deferred(da, i, ja[e]);
        if (jb) acc += wb * apply_deferred(db, i, jb[e]);
        out[e] = post * acc;
    }
}

// out = the stored values with their deferred rules applied.
__global__ void apply_deferred_kernel(const Deferred d, const int* __restrict__ rowidx, const double* __restrict__ j,
                                      double* __restrict__ out, int64_t nnz)
{
    GRID_STRIDE(e, nnz) out[e] = apply_deferred(d, rowidx[e], j[e]);
}

// Operands on different patterns: merge each row into the union pattern.
__global__ void ew_merge_kernel(Rule r, int rows, const int* __restrict__ aptr, const int* __restrict__ acol,
                                const double* __restrict__ ja, const int* __restrict__ bptr,
                                const int* __restrict__ bcol, const double* __restrict__ jb,
                                const int* __restrict__ optr, const int* __restrict__ ocol,
                                double* __restrict__ out, const Deferred da, const Deferred db)
{
    GRID_STRIDE(i, rows)
    {
        double wa, wb, post;
        rule_weights(r, i, wa, wb, post);
        int pa = ja ? aptr[i] : 0, ea = ja ? aptr[i + 1] : 0;
        int pb = jb ? bptr[i] : 0, eb = jb ? bptr[i + 1] : 0;
        const int p1 = optr[i + 1];
        for (int p = optr[i]; p < p1; ++p) {
            const int c = ocol[p];
            double acc = 0.0;
            if (pa < ea && acol[pa] == c) acc += wa * apply_deferred(da, i, ja[pa++]);
            if (pb < eb && bcol[pb] == c) acc += wb * apply_deferred(db, i, jb[pb++]);
            out[p] = post * acc;
        }
    }
}

// out = [x (n1 values), y (n2 values)]: the sum of two Jacobians whose
// entries lie in disjoint row ranges (each entry 1.0 * its one operand).
__global__ void concat_kernel(const double* __restrict__ x, int64_t n1, const double* __restrict__ y, int64_t n2,
                              double* __restrict__ out, const int* __restrict__ rowidx, const Deferred dx,
                              const Deferred dy)
{
    if (dx.n == 0 && dy.n == 0) {
        GRID_STRIDE(e, n1 + n2) out[e] = e < n1 ? x[e] : y[e - n1];
    } else {
        GRID_STRIDE(e, n1 + n2) out[e] = e < n1 ? apply_deferred(dx, rowidx[e], x[e])
                                                : apply_deferred(dy, rowidx[e], y[e - n1]);
    }
}

// Position in each operand of every entry of the union pattern (-1: absent),
// built once per operand pattern pair.
__global__ void merge_map_kernel(int rows, const int* __restrict__ aptr, const int* __restrict__ acol,
                                 const int* __restrict__ bptr, const int* __restrict__ bcol,
                                 const int* __restrict__ optr, const int* __restrict__ ocol, int* __restrict__ ia,
                                 int* __restrict__ ib)
{
    GRID_STRIDE(i, rows)
    {
        int pa = aptr ? aptr[i] : 0, ea = aptr ? aptr[i + 1] : 0;
        int pb = bptr ? bptr[i] : 0, eb = bptr ? bptr[i + 1] : 0;
        const int p1 = optr[i + 1];
        for (int p = optr[i]; p < p1; ++p) {
            const int c = ocol[p];
            ia[p] = (pa < ea && acol[pa] == c) ? pa++ : -1;
            ib[p] = (pb < eb && bcol[pb] == c) ? pb++ : -1;
        }
    }
}

// ew_merge_kernel through the position maps: one thread per nonzero, the
// same operations in the same order.
__global__ void ew_mapped_kernel(Rule r, const int* __restrict__ rowidx, const int* __restrict__ ia,
                                 const int* __restrict__ ib, const double* __restrict__ ja,
                                 const double* __restrict__ jb, double* __restrict__ out, int64_t nnz,
                                 const Deferred da, const Deferred db)
{
    GRID_STRIDE(e, nnz)
    {
        const int i = rowidx[e];
        double wa, wb, post;
        rule_weights(r, i, wa, wb, post);
        const int xa = ia[e], xb = ib[e];
        double acc = 0.0;
        if (xa >= 0) acc += wa * apply_deferred(da, i, ja[xa]);
        if (xb >= 0) acc += wb * apply_deferred(db, i, jb[xb]);
        out[e] = post * acc;
    }
}

// Union pattern of two patterns with the same shape.
template <bool FILL>
__global__ void union_kernel(int rows, const int* aptr, const int* acol, const int* bptr, const int* bcol,
                             int64_t* cnt, const int* optr, int* ocol)
{
    GRID_STRIDE(i, rows)
    {
        int pa = aptr[i], ea = aptr[i + 1], pb = bptr[i], eb = bptr[i + 1];
        int64_t count = 0;
        int o = FILL ? optr[i] : 0;
        while (pa < ea || pb < eb) {
            int c;
            if (pb >= eb || (pa < ea && acol[pa] < bcol[pb])) c = acol[pa++];
            else if (pa >= ea || bcol[pb] < acol[pa]) c = bcol[pb++];
            else {
                c = acol[pa++];
                ++pb;
            }
            if (FILL) ocol[o++] = c;
            else ++count;
        }
        if (!FILL) cnt[i] = count;
    }
}

}  // namespace

// Inclusive scan of per-row counts into an int32 rowptr; returns nnz.
int64_t counts_to_rowptr(Core& c, Buf& counts, int rows, Buf& rowptr)
{
    Buf incl = c.allocN<int64_t>(rows > 0 ? rows : 1);
    if (rows > 0) {
        size_t tmp_bytes = 0;
        EQG_CUDA(cub::DeviceScan::InclusiveSum(nullptr, tmp_bytes, counts->as<int64_t>(), incl->as<int64_t>(), rows,
                                               c.stream));
        Buf tmp = c.alloc(tmp_bytes > 0 ? tmp_bytes : 16);
        EQG_CUDA(cub::DeviceScan::InclusiveSum(tmp->ptr, tmp_bytes, counts->as<int64_t>(), incl->as<int64_t>(), rows,
                                               c.stream));
        c.launches++;
    }
    int64_t total = 0;
    if (rows > 0) {
        EQG_CUDA(cudaMemcpyAsync(&c.pinned[0], incl->as<int64_t>() + rows - 1, sizeof(int64_t),
                                 cudaMemcpyDeviceToHost, c.stream));
        c.sync();
        std::memcpy(&total, &c.pinned[0], sizeof(int64_t));
    }
    if (total > (int64_t)INT_MAX) fail(EQG_ERR_UNSUPPORTED, "sparsity pattern with more than 2^31-1 entries");
    rowptr = c.allocN<int>((size_t)rows + 1);
    launch(c, "rowptr", [&] { i64_to_rowptr_kernel<<<blocksFor((int64_t)rows + 1), kThreads, 0, c.stream>>>(incl->as<int64_t>(), rows,
                                                                                  rowptr->as<int>()); });
    return total;
}

namespace {

template <int KMAX>
void spgemm_symbolic(Core& c, const OpMatrix& m, const Pattern& j, Pattern& out)
{
    Buf cnt = c.allocN<int64_t>(m.n_out > 0 ? m.n_out : 1);
    const int nb = blocksFor(m.n_out);
    if (m.n_out > 0) {
        launch(c, "spgemm_count", [&] { spgemm_count_kernel<KMAX><<<nb, kThreads, 0, c.stream>>>(m.n_out, m.ptr->as<int>(), m.src->as<int>(),
                                                                j.rowptr->as<int>(), j.colind->as<int>(),
                                                                cnt->as<int64_t>()); });
    }
    out.nnz = counts_to_rowptr(c, cnt, m.n_out, out.rowptr);
    out.colind = c.allocN<int>(out.nnz > 0 ? out.nnz : 1);
    if (m.n_out > 0) {
        launch(c, "spgemm_fill", [&] { spgemm_fill_kernel<KMAX><<<nb, kThreads, 0, c.stream>>>(m.n_out, m.ptr->as<int>(), m.src->as<int>(),
                                                               j.rowptr->as<int>(), j.colind->as<int>(),
                                                               out.rowptr->as<int>(), out.colind->as<int>()); });
    }
}

template <int KMAX>
void spgemm_build_plan(Core& c, const OpMatrix& m, const Pattern& j, Pattern& out)
{
    if (m.n_out <= 0 || out.nnz <= 0) return;
    Buf cnt = c.allocN<int64_t>((size_t)out.nnz);
    const int nb = blocksFor(m.n_out);
    launch(c, "spgemm_plan_count", [&] {
        spgemm_plan_kernel<KMAX, true><<<nb, kThreads, 0, c.stream>>>(
            m.n_out, m.ptr->as<int>(), m.src->as<int>(), j.rowptr->as<int>(), j.colind->as<int>(),
            out.rowptr->as<int>(), out.colind->as<int>(), cnt->as<int64_t>(), nullptr, nullptr);
    });
    const int64_t total = counts_to_rowptr(c, cnt, (int)out.nnz, out.plan_start);
    out.plan_entries = total;
    out.plan_contrib = c.allocN<int>(total > 0 ? total : 1);
    launch(c, "spgemm_plan_fill", [&] {
        spgemm_plan_kernel<KMAX, false><<<nb, kThreads, 0, c.stream>>>(
            m.n_out, m.ptr->as<int>(), m.src->as<int>(), j.rowptr->as<int>(), j.colind->as<int>(),
            out.rowptr->as<int>(), out.colind->as<int>(), nullptr, out.plan_start->as<int>(),
            out.plan_contrib->as<int>());
    });
    pattern_build_rowidx(c, out);
}

template <int KMAX>
void spgemm_numeric(Core& c, const OpMatrix& m, const Pattern& jp, const double* jv, const Pattern& op, double* ov,
                    const Deferred& jd)
{
    if (m.n_out <= 0) return;
    if (jd.n && !op.plan_start) fail(EQG_ERR_DEVICE, "operator product of deferred Jacobian values without a plan");
    if (op.plan_start) {
        // algorithmic bytes: the output's row indices and plan, the
        // contributing Jacobian values and M's row pointers and weights, the
        // output values
        const double bytes = 16.0 * op.nnz + 12.0 * op.plan_entries + 4.0 * (m.n_out + 1) + 8.0 * m.nnz;
        launch(c, "spgemm_planned", [&] {
            spgemm_planned_kernel<<<blocksFor(op.nnz), kThreads, 0, c.stream>>>(
                op.nnz, op.rowidx->as<int>(), m.ptr->as<int>(), m.w->as<double>(), op.plan_start->as<int>(),
                op.plan_contrib->as<int>(), jv, ov, m.src->as<int>(), jd);
        }, bytes + 16.0 * jd.n * jp.rows);
        return;
    }
    // algorithmic bytes: M (row pointers, sources, weights), the Jacobian
    // operand and the output pattern (row pointers, columns, values) once
    const double bytes = 4.0 * (m.n_out + 1) + 12.0 * m.nnz + 4.0 * (jp.rows + 1) + 12.0 * jp.nnz +
                         4.0 * (op.rows + 1) + 12.0 * op.nnz;
    launch(c, "spgemm_numeric", [&] { spgemm_numeric_kernel<KMAX><<<blocksFor(m.n_out), kThreads, 0, c.stream>>>(
        m.n_out, m.ptr->as<int>(), m.src->as<int>(), m.w->as<double>(), jp.rowptr->as<int>(), jp.colind->as<int>(),
        jv, op.rowptr->as<int>(), op.colind->as<int>(), ov); }, bytes);
}

int kmax_for(int max_row)
{
    if (max_row <= 1) return 1;
    if (max_row <= 2) return 2;
    if (max_row <= 4) return 4;
    if (max_row <= 6) return 6;
    if (max_row <= 8) return 8;
    if (max_row <= 16) return 16;
    fail(EQG_ERR_UNSUPPORTED, "operator rows longer than 16 entries");
}

}  // namespace

OpMatrixP opmat_from_host(Core& c, int n_out, int n_src, const std::vector<int32_t>& ptr,
                          const std::vector<int32_t>& src, const std::vector<double>& w)
{
    auto m = std::make_shared<OpMatrix>();
    m->id = c.newId();
    m->n_out = n_out;
    m->n_src = n_src;
    for (int i = 0; i < n_out; ++i) m->max_row = std::max(m->max_row, ptr[i + 1] - ptr[i]);
    m->nnz = (int64_t)src.size();
    m->ptr = c.allocN<int32_t>(ptr.size());
    m->src = c.allocN<int32_t>(src.empty() ? 1 : src.size());
    m->w = c.allocN<double>(w.empty() ? 1 : w.size());
    EQG_CUDA(cudaMemcpyAsync(m->ptr->ptr, ptr.data(), ptr.size() * 4, cudaMemcpyHostToDevice, c.stream));
    if (!src.empty()) {
        EQG_CUDA(cudaMemcpyAsync(m->src->ptr, src.data(), src.size() * 4, cudaMemcpyHostToDevice, c.stream));
        EQG_CUDA(cudaMemcpyAsync(m->w->ptr, w.data(), w.size() * 8, cudaMemcpyHostToDevice, c.stream));
    }
    c.sync();
    return m;
}

OpMatrixP opmat_from_map(Core& c, const int32_t* map_dev, int n_out, int n_src, bool allow_missing)
{
    auto m = std::make_shared<OpMatrix>();
    m->id = c.newId();
    m->n_out = n_out;
    m->n_src = n_src;
    m->max_row = 1;
    Buf cnt = c.allocN<int64_t>(n_out > 0 ? n_out : 1);
    Buf err = c.allocN<int32_t>(1);
    EQG_CUDA(cudaMemsetAsync(err->ptr, 0, 4, c.stream));
    if (n_out > 0) {
        launch(c, "map_count", [&] { map_count_kernel<<<blocksFor(n_out), kThreads, 0, c.stream>>>(map_dev, n_out, cnt->as<int64_t>(), n_src,
                                                                      err->as<int32_t>()); });
    }
    const int64_t nnz = counts_to_rowptr(c, cnt, n_out, m->ptr);
    int32_t herr = 0;
    EQG_CUDA(cudaMemcpyAsync(c.pinned, err->ptr, 4, cudaMemcpyDeviceToHost, c.stream));
    c.sync();
    std::memcpy(&herr, c.pinned, 4);
    if (herr) fail(EQG_ERR_ARG, "index map points outside its source collection");
    if (!allow_missing && nnz != n_out) fail(EQG_ERR_ARG, "index map has unmatched entries");
    m->nnz = nnz;
    m->src = c.allocN<int32_t>(nnz > 0 ? nnz : 1);
    m->w = c.allocN<double>(nnz > 0 ? nnz : 1);
    if (n_out > 0) {
        launch(c, "map_fill", [&] { map_fill_kernel<<<blocksFor(n_out), kThreads, 0, c.stream>>>(map_dev, n_out, m->ptr->as<int>(),
                                                                    m->src->as<int>(), m->w->as<double>()); });
    }
    return m;
}

void opmat_apply_values(Core& c, const OpMatrix& m, const double* x, double* y)
{
    if (m.n_out <= 0) return;
    if (m.stencil && c.stencil_ops && stencil_apply_values(c, m.stencil, x, y)) return;
    launch(c, "opmat_apply", [&] { opmat_apply_kernel<<<blocksFor(m.n_out), kThreads, 0, c.stream>>>(m.n_out, m.ptr->as<int>(), m.src->as<int>(),
                                                                     m.w->as<double>(), x, y); },
           4.0 * (m.n_out + 1) + 12.0 * m.nnz + 8.0 * m.n_src + 8.0 * m.n_out);
}

PatternP pattern_identity(Core& c, int n)
{
    auto it = c.identity_patterns.find(n);
    if (it != c.identity_patterns.end()) return it->second;
    auto p = std::make_shared<Pattern>();
    p->id = c.newId();
    p->rows = p->cols = n;
    p->nnz = n;
    p->max_row = n > 0 ? 1 : 0;
    p->rowptr = c.allocN<int>((size_t)n + 1);
    p->colind = c.allocN<int>(n > 0 ? n : 1);
    launch(c, "identity_pattern", [&] { identity_pattern_kernel<<<blocksFor((int64_t)n + 1), kThreads, 0, c.stream>>>(n, p->rowptr->as<int>(),
                                                                                 p->colind->as<int>(), nullptr); });
    c.identity_patterns[n] = p;
    return p;
}

Buf ones(Core& c, int64_t n)
{
    auto it = c.ones_cache.find(n);
    if (it != c.ones_cache.end()) return it->second;
    Buf b = c.allocN<double>(n > 0 ? n : 1);
    if (n > 0) {
        launch(c, "ones", [&] { ones_kernel<<<blocksFor(n), kThreads, 0, c.stream>>>(b->as<double>(), n); });
    }
    c.ones_cache[n] = b;
    return b;
}

PatternP pattern_spgemm(Core& c, const OpMatrix& m, const PatternP& j, bool with_plan)
{
    if (m.n_src != j->rows) fail(EQG_ERR_ARG, "operator/Jacobian shape mismatch");
    const auto key = std::make_tuple(1, m.id, j->id, (int64_t)0);
    auto it = c.pattern_cache.find(key);
    if (it != c.pattern_cache.end()) {
        c.pattern_hits++;
        return it->second;
    }
    auto p = std::make_shared<Pattern>();
    p->id = c.newId();
    p->rows = m.n_out;
    p->cols = j->cols;
    switch (kmax_for(m.max_row)) {
    case 1: spgemm_symbolic<1>(c, m, *j, *p); break;
    case 2: spgemm_symbolic<2>(c, m, *j, *p); break;
    case 4: spgemm_symbolic<4>(c, m, *j, *p); break;
    case 6: spgemm_symbolic<6>(c, m, *j, *p); break;
    case 8: spgemm_symbolic<8>(c, m, *j, *p); break;
    default: spgemm_symbolic<16>(c, m, *j, *p); break;
    }
    // the position plan, when positions and streams fit its packing
    if (with_plan && c.param_i("spgemm_plan", 1) != 0 && j->nnz <= kPlanMask && p->nnz < (int64_t)INT_MAX / 2) {
        switch (kmax_for(m.max_row)) {
        case 1: spgemm_build_plan<1>(c, m, *j, *p); break;
        case 2: spgemm_build_plan<2>(c, m, *j, *p); break;
        case 4: spgemm_build_plan<4>(c, m, *j, *p); break;
        case 6: spgemm_build_plan<6>(c, m, *j, *p); break;
        case 8: spgemm_build_plan<8>(c, m, *j, *p); break;
        default: spgemm_build_plan<16>(c, m, *j, *p); break;
        }
    }
    c.patterns_built++;
    c.pattern_cache[key] = p;
    return p;
}

void spgemm_values(Core& c, const OpMatrix& m, const Pattern& jp, const double* jv, const Pattern& op, double* ov,
                   const Deferred* jd)
{
    const Deferred none;
    const Deferred& d = jd ? *jd : none;
    switch (kmax_for(m.max_row)) {
    case 1: spgemm_numeric<1>(c, m, jp, jv, op, ov, d); break;
    case 2: spgemm_numeric<2>(c, m, jp, jv, op, ov, d); break;
    case 4: spgemm_numeric<4>(c, m, jp, jv, op, ov, d); break;
    case 6: spgemm_numeric<6>(c, m, jp, jv, op, ov, d); break;
    case 8: spgemm_numeric<8>(c, m, jp, jv, op, ov, d); break;
    default: spgemm_numeric<16>(c, m, jp, jv, op, ov, d); break;
    }
}

void jacobian_apply_deferred(Core& c, const Deferred& d, Pattern& p, const double* j, double* out)
{
    if (p.nnz <= 0) return;
    pattern_build_rowidx(c, p);
    launch(c, "jac_deferred", [&] {
        apply_deferred_kernel<<<blocksFor(p.nnz), kThreads, 0, c.stream>>>(d, p.rowidx->as<int>(), j, out, p.nnz);
    }, 20.0 * p.nnz + 4.0 * p.nnz + 16.0 * d.n * p.rows);
}

PatternP pattern_union(Core& c, const PatternP& a, const PatternP& b)
{
    if (a->id == b->id) return a;
    if (a->rows != b->rows || a->cols != b->cols) fail(EQG_ERR_ARG, "Jacobian shape mismatch in sum");
    const uint64_t lo = std::min(a->id, b->id), hi = std::max(a->id, b->id);
    const auto key = std::make_tuple(2, lo, hi, (int64_t)0);
    auto it = c.pattern_cache.find(key);
    if (it != c.pattern_cache.end()) {
        c.pattern_hits++;
        return it->second;
    }
    auto p = std::make_shared<Pattern>();
    p->id = c.newId();
    p->rows = a->rows;
    p->cols = a->cols;
    Buf cnt = c.allocN<int64_t>(p->rows > 0 ? p->rows : 1);
    const int nb = blocksFor(p->rows);
    if (p->rows > 0) {
        launch(c, "union_count", [&] { union_kernel<false><<<nb, kThreads, 0, c.stream>>>(p->rows, a->rowptr->as<int>(), a->colind->as<int>(),
                                                          b->rowptr->as<int>(), b->colind->as<int>(),
                                                          cnt->as<int64_t>(), nullptr, nullptr); });
    }
    p->nnz = counts_to_rowptr(c, cnt, p->rows, p->rowptr);
    p->colind = c.allocN<int>(p->nnz > 0 ? p->nnz : 1);
    if (p->rows > 0) {
        launch(c, "union_fill", [&] { union_kernel<true><<<nb, kThreads, 0, c.stream>>>(p->rows, a->rowptr->as<int>(), a->colind->as<int>(),
                                                         b->rowptr->as<int>(), b->colind->as<int>(), nullptr,
                                                         p->rowptr->as<int>(), p->colind->as<int>()); });
        // operands with entries in disjoint row ranges (the stacked
        // residuals of a system): the union lists one operand's entries, then
        // the other's
        std::vector<int> ra(p->rows + 1), rb(p->rows + 1);
        EQG_CUDA(cudaMemcpyAsync(ra.data(), a->rowptr->ptr, ra.size() * 4, cudaMemcpyDeviceToHost, c.stream));
        EQG_CUDA(cudaMemcpyAsync(rb.data(), b->rowptr->ptr, rb.size() * 4, cudaMemcpyDeviceToHost, c.stream));
        c.sync();
        auto first_row = [&](const std::vector<int>& r) {
            for (int i = 0; i < p->rows; ++i)
                if (r[i + 1] > r[i]) return i;
            return p->rows;
        };
        auto last_row = [&](const std::vector<int>& r) {
            for (int i = p->rows - 1; i >= 0; --i)
                if (r[i + 1] > r[i]) return i;
            return -1;
        };
        if (a->nnz > 0 && b->nnz > 0) {
            if (last_row(ra) < first_row(rb)) {
                p->concat_first = a->id;
                p->concat_second = b->id;
            } else if (last_row(rb) < first_row(ra)) {
                p->concat_first = b->id;
                p->concat_second = a->id;
            }
        }
    }
    c.patterns_built++;
    c.pattern_cache[key] = p;
    return p;
}

void pattern_build_rowidx(Core& c, Pattern& p)
{
    if (p.rowidx) return;
    p.rowidx = c.allocN<int>(p.nnz > 0 ? p.nnz : 1);
    if (p.rows > 0) {
        launch(c, "rowidx", [&] { rowidx_kernel<<<blocksFor(p.rows), kThreads, 0, c.stream>>>(p.rows, p.rowptr->as<int>(), p.rowidx->as<int>()); });
    }
}

void jacobian_elementwise(Core& c, const JacArgs& a, const Pattern& out, double* jout)
{
    Rule r{a.rule, a.va, a.vb, a.vout, a.mask, a.s};
    const bool flat = (!a.pa || a.pa->id == out.id) && (!a.pb || a.pb->id == out.id);
    if (out.nnz <= 0) return;
    // algorithmic bytes: the operand Jacobians' values and the output's once,
    // the output's row pointers, the per-row operand values the rule uses;
    // operands on other patterns add their column indices and the output's
    const int64_t na = a.pa ? a.pa->nnz : 0, nbv = a.pb ? a.pb->nnz : 0;
    const double per_row = 8.0 * ((a.va ? 1 : 0) + (a.vb ? 1 : 0) + (a.vout ? 1 : 0)) + (a.mask ? 1.0 : 0.0);
    const double bytes = 8.0 * (na + nbv + out.nnz) + 4.0 * (out.rows + 1) + per_row * out.rows +
                         (flat ? 0.0 : 4.0 * (na + nbv + out.nnz)) + 16.0 * (a.da.n + a.db.n) * out.rows;
    if (a.rule == JR_ADD && a.pa && a.pb && out.concat_first && c.jac_concat &&
        ((a.pa->id == out.concat_first && a.pb->id == out.concat_second) ||
         (a.pb->id == out.concat_first && a.pa->id == out.concat_second))) {
        const bool a_first = a.pa->id == out.concat_first;
        const double* x = a_first ? a.ja : a.jb;
        const double* y = a_first ? a.jb : a.ja;
        const int64_t n1 = a_first ? a.pa->nnz : a.pb->nnz, n2 = out.nnz - n1;
        const Deferred& dx = a_first ? a.da : a.db;
        const Deferred& dy = a_first ? a.db : a.da;
        if (dx.n || dy.n) pattern_build_rowidx(c, const_cast<Pattern&>(out));
        launch(c, "jac_concat", [&] {
            concat_kernel<<<blocksFor(out.nnz), kThreads, 0, c.stream>>>(
                x, n1, y, n2, jout, (dx.n || dy.n) ? out.rowidx->as<int>() : nullptr, dx, dy);
        }, 16.0 * out.nnz);
        return;
    }
    if (flat) {
        pattern_build_rowidx(c, const_cast<Pattern&>(out));
        launch(c, "jac_flat", [&] {
            ew_flat_kernel<<<blocksFor(out.nnz), kThreads, 0, c.stream>>>(
                r, out.rowidx->as<int>(), a.pa ? a.ja : nullptr, a.pb ? a.jb : nullptr, jout, out.nnz, a.da, a.db);
        }, bytes);
    } else if (out.nnz < (int64_t)INT_MAX / 2) {
        // through position maps kept with the output pattern
        Pattern& o = const_cast<Pattern&>(out);
        pattern_build_rowidx(c, o);
        const auto key = std::make_pair(a.pa ? a.pa->id : 0, a.pb ? a.pb->id : 0);
        Buf& maps = o.merge_maps[key];
        if (!maps) {
            maps = c.allocN<int>((size_t)2 * out.nnz);
            launch(c, "merge_map", [&] {
                merge_map_kernel<<<blocksFor(out.rows), kThreads, 0, c.stream>>>(
                    out.rows, a.pa ? a.pa->rowptr->as<int>() : nullptr, a.pa ? a.pa->colind->as<int>() : nullptr,
                    a.pb ? a.pb->rowptr->as<int>() : nullptr, a.pb ? a.pb->colind->as<int>() : nullptr,
                    out.rowptr->as<int>(), out.colind->as<int>(), maps->as<int>(), maps->as<int>() + out.nnz);
            });
        }
        launch(c, "jac_merge", [&] {
            ew_mapped_kernel<<<blocksFor(out.nnz), kThreads, 0, c.stream>>>(
                r, out.rowidx->as<int>(), maps->as<int>(), maps->as<int>() + out.nnz, a.pa ? a.ja : nullptr,
                a.pb ? a.jb : nullptr, jout, out.nnz, a.da, a.db);
        }, bytes);
    } else {
        launch(c, "jac_merge", [&] { ew_merge_kernel<<<blocksFor(out.rows), kThreads, 0, c.stream>>>(
            r, out.rows, a.pa ? a.pa->rowptr->as<int>() : nullptr, a.pa ? a.pa->colind->as<int>() : nullptr,
            a.pa ? a.ja : nullptr, a.pb ? a.pb->rowptr->as<int>() : nullptr, a.pb ? a.pb->colind->as<int>() : nullptr,
            a.pb ? a.jb : nullptr, out.rowptr->as<int>(), out.colind->as<int>(), jout, a.da, a.db); }, bytes);
    }
}

}  // namespace eqg

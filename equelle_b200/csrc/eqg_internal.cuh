// Internal types of the device runtime behind include/eqg.h.
//
// Data layout in HBM (one runtime = one grid = one CUDA stream):
//   - every collection value array is a dense double[n];
//   - a Jacobian is a CSR pattern (int32 rowptr[n+1], int32 colind[nnz],
//     ascending columns) shared through the pattern cache, plus a double[nnz]
//     value array owned by the collection;
//   - entity sets are int32[n] (-1 = outside), masks uint8[n];
//   - the grid's helper operators (gradient, divergence, On/Extend
//     selections) are small-row CSR "operator matrices" with double weights.
// All buffers are immutable once written, so handles share them freely.
#pragma once

#include "eqg.h"

#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <map>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <tuple>
#include <unordered_map>
#include <unordered_set>
#include <vector>

struct eqg_coll;
struct eqg_mask;

namespace eqg {

struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

[[noreturn]] inline void fail(int code, const std::string& msg) { throw Error(code, msg); }

#define EQG_CUDA(call)                                                                              \
    do {                                                                                            \
        cudaError_t e_ = (call);                                                                    \
        if (e_ != cudaSuccess)                                                                      \
            ::eqg::fail(EQG_ERR_DEVICE, std::string(#call " failed: ") + cudaGetErrorString(e_));    \
    } while (0)

struct Core;

// Device allocation from the runtime's stream-ordered pool.
struct DevBuf {
    Core* core = nullptr;
    void* ptr = nullptr;
    size_t bytes = 0;
    ~DevBuf();
    template <class T>
    T* as() const { return static_cast<T*>(ptr); }
};
using Buf = std::shared_ptr<DevBuf>;

// CSR sparsity pattern on the device.
struct SolverAnalysis;
struct Pattern {
    uint64_t id = 0;
    int rows = 0, cols = 0;
    int64_t nnz = 0;
    int max_row = 0;            // longest row
    Buf rowptr;                 // int32[rows+1]
    Buf colind;                 // int32[nnz]
    Buf rowidx;                 // int32[nnz], built on demand (row of each entry)
    // for a union pattern: per pair of operand patterns (ids), the position
    // of each entry in either operand (-1: absent), int32[2 nnz]
    std::map<std::pair<uint64_t, uint64_t>, Buf> merge_maps;
    // for a pattern made as M J (gradient, divergence, On, Extend, spans):
    // per entry, the positions of J's entries that add into it (see
    // spgemm_plan_kernel), int32[nnz+1] bounds and int32 packed positions
    Buf plan_start, plan_contrib;
    int64_t plan_entries = 0;
    // for a union pattern whose operands have entries in disjoint row
    // ranges, the one with the lower rows first: the union's entries are
    // those of concat_first, then those of concat_second (ids; 0: not such
    // a union)
    uint64_t concat_first = 0, concat_second = 0;
    std::shared_ptr<SolverAnalysis> analysis;  // linear-solver analysis, built on demand
    // the analysis without multigrid, for a solve that the multigrid
    // preconditioner did not converge (linsolver_fallback)
    std::shared_ptr<SolverAnalysis> analysis_fallback;
};
using PatternP = std::shared_ptr<Pattern>;

// A small-row operator matrix M (n_out x n_src): out = M x and out_J = M J.
struct OpMatrix {
    uint64_t id = 0;
    int n_out = 0, n_src = 0;
    int max_row = 0;
    int64_t nnz = 0;
    // a helper operator of the Cartesian grid that the stencil kernels apply
    // to values by face and cell index arithmetic (STENCIL_*; 0: none)
    int stencil = 0;
    Buf ptr;   // int32[n_out+1]
    Buf src;   // int32[nnz], ascending within a row
    Buf w;     // double[nnz]
};
using OpMatrixP = std::shared_ptr<OpMatrix>;

struct SolverStats {
    int64_t linear_solves = 0, krylov_iterations = 0, refinement_sweeps = 0;
    double last_residual = 0.0;
    int64_t last_rows = 0, last_nnz = 0;
    int64_t last_block_size = 0, last_blocks = 0;
};

struct Mark {
    cudaEvent_t ev;
};

// Accumulated device time of one phase (pairs of events on the stream).
struct PhaseClock {
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> pairs;
    cudaEvent_t open = nullptr;
    int64_t count = 0;
    void start(cudaStream_t s)
    {
        cudaEventCreate(&open);
        cudaEventRecord(open, s);
    }
    void stop(cudaStream_t s)
    {
        cudaEvent_t e;
        cudaEventCreate(&e);
        cudaEventRecord(e, s);
        pairs.emplace_back(open, e);
        open = nullptr;
        ++count;
    }
    double total_ms() const { return ms_from(0); }
    // time of the intervals first .. end
    double ms_from(size_t first) const
    {
        double ms = 0.0;
        for (size_t i = first; i < pairs.size(); ++i) {
            float f = 0.f;
            cudaEventSynchronize(pairs[i].second);
            cudaEventElapsedTime(&f, pairs[i].first, pairs[i].second);
            ms += f;
        }
        return ms;
    }
    void clear()
    {
        for (auto& p : pairs) {
            cudaEventDestroy(p.first);
            cudaEventDestroy(p.second);
        }
        pairs.clear();
        if (open) cudaEventDestroy(open);
        open = nullptr;
        count = 0;
    }
};

// Runtime state shared by every handle (a handle keeps the core alive).
struct Core {
    cudaStream_t stream = nullptr;
    int device = 0;
    cudaMemPool_t pool = nullptr;
    std::map<std::string, std::string> params;

    // grid
    int dim = 2, nx = 6, ny = 1, nz = 1;
    double dx = 1, dy = 1, dz = 1;
    int nc = 0, nf = 0, nif = 0;
    bool cartesian = true;  // false: read from a grid file (grid_filename); nx = ny = nz = 0
    Buf face_cells;      // int32[2*nf]
    Buf face_normals;    // double[dim*nf], area-scaled (component-major); grids read from a file only
    Buf face_areas;      // double[nf]
    Buf face_centroids;  // double[dim*nf] (component-major: d*nf + f)
    Buf cell_volumes;    // double[nc]
    Buf cell_centroids;  // double[dim*nc] (component-major)
    OpMatrixP grad, ngrad, div_interior, div_full;

    // settings
    int verbose = 0, max_iter = 10;
    double abs_res_tol = 1e-6;
    // assembly fast paths (parameters of the same names, read once)
    bool jac_concat = true, jac_defer = true, stencil_ops = true, span_share = true;

    // accounting
    std::atomic<int64_t> launches{0};
    int64_t bytes_in_use = 0, bytes_peak = 0;
    int64_t patterns_built = 0, pattern_hits = 0;
    int64_t newton_solves = 0, newton_iterations = 0;
    SolverStats solver;

    // caches
    uint64_t next_id = 1;
    std::map<std::tuple<int, uint64_t, uint64_t, int64_t>, PatternP> pattern_cache;
    std::map<std::tuple<int, uint64_t, uint64_t, int64_t>, OpMatrixP> opmat_cache;
    std::map<int64_t, PatternP> identity_patterns;
    std::map<int64_t, Buf> ones_cache;
    std::map<std::tuple<int, uint64_t>, struct eqg_set*> derived_sets;  // owned references

    // scratch for reductions
    Buf red_partials;   // double[kRedBlocks * 4]
    Buf red_counter;    // unsigned int
    double* pinned = nullptr;  // small pinned host buffer
    // pinned staging for large copies between device memory and pageable
    // host memory (copy_to_device / copy_to_host), allocated on first use
    char* stage[2] = {nullptr, nullptr};
    cudaEvent_t stage_done[2] = {nullptr, nullptr};
    std::vector<Mark> marks;
    std::vector<eqg_solve_info> solves;
    // device timing of one named kernel (parameter time_kernel)
    std::string timed_kernel;  // a kernel name, or "*" for all of them
    bool pdl_launch = false;   // BiCGStab iteration kernels as programmatic dependent launches (linsolver_pdl)
    struct TimedLaunch {
        const char* name;
        cudaEvent_t a, b;
        double bytes;  // algorithmic bytes of the launch (< 0: not stated)
    };
    std::vector<TimedLaunch> timer_pairs;
    PhaseClock residual_clock, factor_clock, krylov_clock;
    // deferred value expressions: recording on (`lazy`), evaluated by the
    // expression kernel (`lazy_vm`, parameter lazy=1) or, when recorded for
    // fusion (parameter fuse), by a fused step that matches the recorded
    // DAG (fused.cu) or one kernel per node; handles with pending values,
    // evaluation passes run, fused evaluations run
    bool lazy = false;
    bool lazy_vm = false;
    bool fuse = false;
    std::unordered_set<eqg_coll*> lazy_colls;
    std::unordered_set<eqg_mask*> lazy_masks;
    int64_t lazy_passes = 0;
    int64_t fused_evaluations = 0;
    std::shared_ptr<struct FuseState> fuse_state;  // fused.cu: verified operators and arrays, cached maxima
    Buf flush_buf;  // written before each Newton solve under flush_l2
    // asynchronous output copies (eqg_output_*): device -> pinned host on
    // their own stream.  The ticket table and the pinned pool are shared with
    // the thread that waits for copies (mutex); device buffers of finished
    // copies are dropped on the runtime's own thread (reap_outputs).
    struct OutputCopy {
        Buf values;              // kept alive until the copy has finished
        double* host = nullptr;  // pinned
        size_t bytes = 0;
        int64_t n = 0;
        cudaEvent_t done = nullptr;
    };
    cudaStream_t copy_stream = nullptr;
    std::mutex output_mutex;
    std::map<int64_t, OutputCopy> output_copies;
    std::vector<OutputCopy> output_released;
    std::multimap<size_t, double*> pinned_pool;
    int64_t next_ticket = 1;
    void reap_outputs();

    Core();
    ~Core();

    // caching allocator (see core.cu)
    std::unordered_map<size_t, std::vector<void*>> free_blocks;
    int64_t cached_bytes = 0;
    bool releasing = false;
    static size_t size_class(size_t bytes);
    void release_cached();

    uint64_t newId() { return next_id++; }
    Buf alloc(size_t bytes);
    template <class T>
    Buf allocN(size_t n) { return alloc(n * sizeof(T)); }
    void free(void* p, size_t bytes);
    void sync();
    void checkLaunch(const char* what);
    // bytes between pageable host memory and device memory through the
    // pinned staging buffers, in chunks, DMA of one chunk overlapping the
    // host copy of the other; both return with the copy finished
    void copy_to_device(void* dst, const void* src, size_t bytes);
    void copy_to_host(void* dst, const void* src, size_t bytes);
    double param_d(const std::string& k, double d) const;
    int param_i(const std::string& k, int d) const;
    std::string param_s(const std::string& k, const std::string& d) const;
};

using CoreP = std::shared_ptr<Core>;

// ---- deferred value expressions (lazy.cu, fused.cu) ----------------------
// Value-only operations (arithmetic, with a scalar, unary, comparisons,
// trinaryIf, mask logic, constant collections and, when recorded for
// fusion, On/Extend/gradient/divergence) are recorded as nodes of a DAG
// over materialized arrays instead of being launched.  The first operation
// that needs values (any other operation, a reduction, a host copy, an
// output) evaluates them.  Two evaluators, both with the same
// floating-point operations, in the same order, as the
// one-kernel-per-operation path:
//   - lazy=1: every pending node of that length in one pass of an
//     expression kernel (intermediates in shared memory; about as costly as
//     the launches it replaces, so off by default);
//   - fuse=1 (the default on two-dimensional Cartesian grids, outside Newton
//     solves): a fused step when the DAG matches one (fused.cu), else one
//     kernel per node, the kernel the operation launches when not deferred.
enum LazyOp { LZ_LEAF, LZ_CONST, LZ_BIN, LZ_BINS, LZ_UNARY, LZ_CMP, LZ_CMPS, LZ_SEL, LZ_LOGIC, LZ_OPMAT };

struct LazyNode {
    int op = LZ_LEAF;
    int sub = 0;           // the operator of LZ_BIN/BINS/UNARY/CMP/CMPS/LOGIC
    double s = 0.0;        // scalar operand (LZ_BINS, LZ_CMPS) or value (LZ_CONST)
    int scalar_left = 0;
    bool mask = false;     // a mask (uint8) rather than doubles
    int64_t n = 0;
    double cost = 1;       // nodes below (an upper bound; shared nodes counted twice)
    std::shared_ptr<LazyNode> a, b, c;
    Buf leaf;              // LZ_LEAF: the values
    OpMatrixP m;           // LZ_OPMAT: the helper operator applied to `a`
};
using LazyP = std::shared_ptr<LazyNode>;

// Values of a collection or mask, evaluating its pending expression first.
const double* coll_values(Core& c, const eqg_coll* x);
const uint8_t* mask_values(Core& c, const eqg_mask* m);
void settle(Core& c, const eqg_coll* x);
void settle(Core& c, const eqg_mask* m);
// True when `x` may be an operand of a deferred operation (lazy mode, no
// Jacobian).
bool lazy_ok(const Core& c, const eqg_coll* x);
LazyP lazy_node(const eqg_coll* x);
LazyP lazy_node(const eqg_mask* m);
LazyP lazy_make(int op, int sub, int64_t n, bool mask, LazyP a, LazyP b = nullptr, LazyP c = nullptr,
                double s = 0.0, int scalar_left = 0);
LazyP lazy_opmat(const OpMatrixP& m, LazyP a);
eqg_coll* lazy_coll(const CoreP& core, int64_t n, LazyP node);
eqg_mask* lazy_mask(const CoreP& core, int64_t n, LazyP node);
void lazy_forget(eqg_coll* x);
void lazy_forget(eqg_mask* m);
// Evaluates every pending handle (before a Newton solve).
void settle_all(Core& c);
// Evaluates a pending node (a fused step when one matches, else one kernel
// per node); it becomes a leaf.
void lazy_evaluate(Core& c, LazyNode* v);
// The node becomes a leaf over `values` (its operands are released).
void lazy_make_leaf(LazyNode* v, Buf values);

// ---- fused steps (fused.cu) -------------------------------------------------
// The pending expression under `root`, or its reduction, when it matches a
// fused step and the grid and operands meet that step's conditions: the
// values are computed and every matched handle settled (true); false leaves
// everything as it was.
bool fused_materialize(Core& c, LazyNode* root);
bool fused_reduce(Core& c, int op, LazyNode* root, double* out);

// Launches a kernel through `f`, checks the launch, and brackets it with
// CUDA events on the runtime stream when `name` is the timed kernel.
// `bytes`: the launch's algorithmic bytes (the data its operation must read
// and write at least once), reported with the timings (< 0: not stated).
template <class F>
inline void launch(Core& c, const char* name, F&& f, double bytes = -1.0)
{
    const bool timed = !c.timed_kernel.empty() && (c.timed_kernel == name || c.timed_kernel == "*");
    cudaEvent_t a = nullptr, b = nullptr;
    if (timed) {
        cudaEventCreate(&a);
        cudaEventCreate(&b);
        cudaEventRecord(a, c.stream);
    }
    f();
    c.checkLaunch(name);
    if (timed) {
        cudaEventRecord(b, c.stream);
        c.timer_pairs.push_back({name, a, b, bytes});
    }
}

constexpr int kThreads = 256;
constexpr int kRedBlocks = 2368;  // 16 x 148 SMs: grid cap of kernels that reduce through block partials

inline int blocksFor(int64_t n, int threads = kThreads, int cap = 148 * 32)
{
    int64_t b = (n + threads - 1) / threads;
    if (b < 1) b = 1;
    if (b > cap) b = cap;
    return (int)b;
}

// ---- kernels exposed to the C-ABI layer (ops.cu, jacobian.cu, solver.cu) ----
enum EwOp { EW_ADD = 0, EW_SUB, EW_MUL, EW_DIV };

void k_fill(Core& c, double* out, double v, int64_t n);
void k_fill_i32(Core& c, int32_t* out, int32_t v, int64_t n);
void k_binary(Core& c, int op, const double* a, const double* b, double* out, int64_t n);
void k_binary_scalar(Core& c, int op, const double* a, double s, int scalar_left, double* out, int64_t n);
void k_unary_value(Core& c, int op, const double* a, double* out, int64_t n);
void k_compare(Core& c, int op, const double* a, const double* b, uint8_t* out, int64_t n);
void k_compare_scalar(Core& c, int op, const double* a, double s, int scalar_left, uint8_t* out, int64_t n);
void k_select_value(Core& c, const uint8_t* m, const double* a, const double* b, double* out, int64_t n);
void k_mask_logic(Core& c, int op, const uint8_t* a, const uint8_t* b, uint8_t* out, int64_t n);
void k_set_select(Core& c, const uint8_t* m, const int32_t* a, const int32_t* b, int32_t* out, int64_t n);
void k_is_empty(Core& c, const int32_t* s, uint8_t* out, int64_t n);
void k_face_neighbour(Core& c, const int32_t* faces, int side, int32_t* out, int64_t n, int32_t* err);
void k_gather_i32(Core& c, const int32_t* data, const int32_t* map, int32_t* out, int64_t n, int32_t fill);
void k_gather_f64(Core& c, const double* data, const int32_t* idx, int stride, int comp, double* out, int64_t n,
                  int32_t* err);
void k_normal(Core& c, const int32_t* faces, double* out, int comp, int64_t n, int32_t* err);
void k_locate(Core& c, const int32_t* sorted, int64_t n_sorted, const int32_t* keys, int32_t* pos, int64_t n_keys,
              int identity_n, int32_t* err);
void k_scatter_inverse(Core& c, const int32_t* pos, int64_t n, int32_t* inv, int32_t* err);
void k_is_strictly_sorted(Core& c, const int32_t* a, int64_t n, int32_t* flag);
double k_reduce(Core& c, int op, const double* a, int64_t n);
double k_two_norm(Core& c, const double* a, int64_t n);

// An elementwise rule with one Jacobian operand (a row scaling: product or
// quotient by a collection without Jacobian, by a constant, negation, sqrt,
// sign, trinaryIf with one differentiable branch), kept on the result
// instead of applied: the result shares the operand's pattern and stored
// values, and every reader applies the deferred rules in order, row by row,
// with the arithmetic of the eager kernel (post_i * (0 + w_i x), w_i the
// rule's weight of the operand's side).  A chain of such rules then costs no
// pass over the Jacobian of its own.
struct DeferredRule {
    int rule = 0;  // a JacRule
    int side = 0;  // 0: the operand is a (weight wa), 1: b (weight wb)
    const double* va = nullptr;
    const double* vb = nullptr;
    const double* vout = nullptr;
    const uint8_t* mask = nullptr;
    double s = 0.0;
};
constexpr int kMaxDeferred = 4;
struct Deferred {
    int n = 0;
    DeferredRule r[kMaxDeferred];
};

// Operator matrices and Jacobians (jacobian.cu)
OpMatrixP opmat_from_map(Core& c, const int32_t* map_dev, int n_out, int n_src, bool allow_missing);
OpMatrixP opmat_from_host(Core& c, int n_out, int n_src, const std::vector<int32_t>& ptr,
                          const std::vector<int32_t>& src, const std::vector<double>& w);
void opmat_apply_values(Core& c, const OpMatrix& m, const double* x, double* y);
// Helper operators of Cartesian grids applied to values without their CSR
// arrays (core.cu); false when `kind` is not one of them.
enum StencilKind { STENCIL_NONE = 0, STENCIL_GRAD, STENCIL_NGRAD, STENCIL_DIV_FULL, STENCIL_DIV_INTERIOR };
bool stencil_apply_values(Core& c, int kind, const double* x, double* y);
PatternP pattern_identity(Core& c, int n);
Buf ones(Core& c, int64_t n);
// with_plan: also build the output's position plan (spgemm_plan_kernel)
PatternP pattern_spgemm(Core& c, const OpMatrix& m, const PatternP& j, bool with_plan = true);
// ov = M jv; with deferred rules on jv only through the output's position
// plan (spgemm_has_plan), whose kernel applies them per source row.
void spgemm_values(Core& c, const OpMatrix& m, const Pattern& jp, const double* jv, const Pattern& op,
                   double* ov, const Deferred* jd = nullptr);
inline bool spgemm_has_plan(const Pattern& op) { return (bool)op.plan_start; }
PatternP pattern_union(Core& c, const PatternP& a, const PatternP& b);
// Elementwise Jacobian rule: out_row(i) = post_i * (wa_i * A_row(i) (+) wb_i * B_row(i)).
// Weights come from the operand values per op (see jacobian.cu).
enum JacRule {
    JR_ADD = 0, JR_SUB, JR_MUL, JR_DIV,  // two operands, either may be absent
    JR_SCALE_CONST,                        // out = s * A
    JR_DIV_BY_CONST,                       // (1/(s*s)) * (s * A)
    JR_SQRT,                               // (0.5/sqrt(x)) * A
    JR_SIGN,                               // sign(x) * A
    JR_NEG,                                // -A
    JR_SELECT                              // m*A (+) (1-m)*B
};
struct JacArgs {
    int rule = JR_ADD;
    const double* va = nullptr;   // value of operand a
    const double* vb = nullptr;   // value of operand b
    const double* vout = nullptr; // value of the result (sqrt uses it)
    const uint8_t* mask = nullptr;
    double s = 0.0;
    const Pattern* pa = nullptr;
    const double* ja = nullptr;
    const Pattern* pb = nullptr;
    const double* jb = nullptr;
    Deferred da, db;  // rules deferred on the operands' stored values
};
void jacobian_elementwise(Core& c, const JacArgs& args, const Pattern& out, double* jout);
// Stored values with the deferred rules applied (one pass), into out.
void jacobian_apply_deferred(Core& c, const Deferred& d, Pattern& p, const double* j, double* out);
void pattern_build_rowidx(Core& c, Pattern& p);
// Inclusive scan of int64 per-row counts into an int32 rowptr; returns nnz.
int64_t counts_to_rowptr(Core& c, Buf& counts, int rows, Buf& rowptr);
// Ascending indices i in [0, n) with flags[i] != 0.
Buf compact_indices(Core& c, const uint8_t* flags, int64_t n, int64_t& count);

// Linear solver (solver.cu)
struct SolveResult {
    bool converged = false;
    int iterations = 0;
    int sweeps = 0;
    double rel_residual = 0.0;
    int block_size = 1;   // layout of the system in the preconditioner
    int64_t blocks = 0;   // block entries of the matrix pattern
    bool multigrid = false;  // the preconditioner was the multigrid V-cycle
    int fallbacks = 0;       // solves repeated with block ILU(0) alone
};
SolveResult linear_solve(Core& c, const PatternP& p, const double* jval, const double* rhs, double* x);

}  // namespace eqg

// ---- handle structs (global namespace, named in eqg.h) -------------------
struct eqg_set {
    std::atomic<int> refs{1};
    eqg::CoreP core;
    uint64_t id = 0;
    int entity = EQG_CELLS;
    int64_t n = 0;
    eqg::Buf idx;          // int32[n]
    bool identity = false; // idx[i] == i for all i (all cells / all faces)
    int sorted = -1;       // strictly ascending: -1 unknown, 0 no, 1 yes
};

struct eqg_mask {
    std::atomic<int> refs{1};
    eqg::CoreP core;
    int64_t n = 0;
    eqg::Buf v;  // uint8[n]; null while `lazy` is pending
    eqg::LazyP lazy;
};

struct eqg_coll {
    std::atomic<int> refs{1};
    eqg::CoreP core;
    int64_t n = 0;
    eqg::Buf val;           // double[n]; null while `lazy` is pending
    eqg::PatternP pat;      // null: no Jacobian
    eqg::Buf jval;          // double[nnz], before the rules in jdef
    eqg::Deferred jdef;     // row rules deferred on jval (see DeferredRule)
    std::vector<eqg::Buf> jkeep;  // value arrays those rules read
    eqg::LazyP lazy;        // deferred value-only expression
};

struct eqg_runtime {
    eqg::CoreP core;
    eqg_set* builtin[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
};

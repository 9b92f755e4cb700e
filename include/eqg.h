/*
 * eqg.h -- C ABI of the Equelle runtime (libeqg).
 *
 * The C++ surface that Equelle-generated simulators compile against
 * (equelle/EquelleRuntimeCPU.hpp in this tree) is a header-only layer over
 * these functions.  Two libraries export exactly this ABI:
 *   - libeqg.so        : the product, device code for sm_100a (B200);
 *   - the CPU oracle   : a restatement of the reference serial backend, used
 *                        only by tests and the CPU baseline.
 *
 * Conventions
 *   - Every function that can fail returns int: EQG_OK (0) or an EQG_ERR_*
 *     code; the message is in eqg_last_error() (thread-local).
 *   - Handles are reference counted.  A function that returns a handle in an
 *     out-parameter hands over one reference; release it with *_release.
 *   - One runtime owns one grid and one device stream; it is not thread safe,
 *     mirroring the single-threaded reference (EquelleRuntimeCPU keeps mutable
 *     output counters, backends/serial/include/equelle/EquelleRuntimeCPU.hpp:157).
 *   - No function returns before its result is valid for the next eqg_* call
 *     on the same runtime; host-visible results (reductions, *_to_host) are
 *     complete when the call returns.
 *
 * Citations name the reference interface each entry point replaces, as
 * path:line inside sintefmath/equelle.
 */
#ifndef EQG_H
#define EQG_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes --------------------------------------------------- */
#define EQG_OK 0
#define EQG_ERR_ARG 1        /* bad argument: sizes, kinds, null handles   */
#define EQG_ERR_DEVICE 2     /* CUDA error or device-side check failure     */
#define EQG_ERR_SOLVER 3     /* linear solver did not converge              */
#define EQG_ERR_UNSUPPORTED 4
#define EQG_ERR_CALLBACK 5   /* a residual callback reported failure        */
#define EQG_ERR_MEMORY 6

typedef struct eqg_runtime eqg_runtime;
typedef struct eqg_set eqg_set;   /* CollOfCell / CollOfFace               */
typedef struct eqg_mask eqg_mask; /* CollOfBool                            */
typedef struct eqg_coll eqg_coll; /* CollOfScalar: value + optional Jacobian */

enum eqg_entity { EQG_CELLS = 0, EQG_FACES = 1 };

enum eqg_builtin_set {
    EQG_ALL_CELLS = 0,
    EQG_BOUNDARY_CELLS = 1,
    EQG_INTERIOR_CELLS = 2,
    EQG_ALL_FACES = 3,
    EQG_BOUNDARY_FACES = 4,
    EQG_INTERIOR_FACES = 5
};

enum eqg_binary_op { EQG_ADD = 0, EQG_SUB = 1, EQG_MUL = 2, EQG_DIV = 3 };
enum eqg_unary_op { EQG_NEG = 0, EQG_SQRT = 1, EQG_ABS = 2 };
enum eqg_compare_op { EQG_LT = 0, EQG_LE = 1, EQG_GT = 2, EQG_GE = 3, EQG_EQ = 4, EQG_NE = 5 };
enum eqg_reduce_op { EQG_MIN = 0, EQG_MAX = 1, EQG_SUM = 2, EQG_PROD = 3 };
enum eqg_mask_op { EQG_AND = 0, EQG_OR = 1, EQG_NOT = 2 };

typedef struct eqg_grid_info {
    int dimensions;
    int nx, ny, nz;
    double dx, dy, dz;
    int64_t number_of_cells;
    int64_t number_of_faces;
    int64_t number_of_interior_faces;
} eqg_grid_info;

typedef struct eqg_stats {
    int64_t kernel_launches;    /* device kernels this runtime launched      */
    int64_t newton_solves;
    int64_t newton_iterations;
    int64_t linear_solves;
    int64_t krylov_iterations;  /* inner (precision of the inner solve)      */
    int64_t refinement_sweeps;  /* outer FP64 iterative-refinement sweeps    */
    int64_t patterns_built;     /* sparsity patterns computed symbolically   */
    int64_t pattern_cache_hits;
    int64_t device_bytes_in_use;
    int64_t device_bytes_peak;
    double last_linear_residual; /* relative residual of the last solve      */
    int64_t last_matrix_rows;    /* size of the last linear system           */
    int64_t last_matrix_nnz;
    /* Device time of the kernel named by the runtime parameter time_kernel
     * (CUDA events around each of its launches; 0 when unset). */
    int64_t timed_kernel_launches;
    double timed_kernel_ms;
    /* Time in the Newton phases (device clock for the product, host clock
     * for the oracle): residual callbacks, preconditioner set-up (value
     * gather + ILU(0) factorization), Krylov iterations. */
    int64_t residual_evaluations;
    double residual_ms;
    double factor_ms;
    double krylov_ms;
    /* Layout of the last linear system in the preconditioner: block size
     * (unknowns per block row) and stored blocks (1 and the nonzeros for a
     * scalar layout; the oracle always reports a scalar layout). */
    int64_t last_block_size;
    int64_t last_matrix_blocks;
    /* Deferred expressions evaluated by a fused step (parameter fuse). */
    int64_t fused_evaluations;
} eqg_stats;

/* ---- errors and identity -------------------------------------------- */
const char* eqg_last_error(void);
/* "cuda-sm100a" for the product, "cpu-oracle" for the oracle. */
const char* eqg_backend_name(void);

/* ---- runtime -------------------------------------------------------- */
/* Builds the grid and the helper operators from key=value parameters.
 * Keys read: grid_dim (2), nx (6), ny (1), nz (1), dx, dy, dz (1.0),
 * verbose (0), max_iter (10), abs_res_tol (1e-6),
 * linsolver_residual_tolerance (1e-8), linsolver_max_iterations (1000).
 * The device library also reads linsolver_preconditioner (multigrid |
 * ilu0), linsolver_ordering (multicolor | natural),
 * linsolver_precision (double | mixed: FP32 preconditioner | refine: FP32
 * BiCGStab inside FP64 refinement), linsolver_inner_tolerance (1e-4) and
 * linsolver_max_sweeps (60) for refine, linsolver_check_every (4),
 * linsolver_block (1: ncomp x ncomp block ILU(0) for 2 or 3 unknowns per
 * cell; 0: scalar ILU(0)), linsolver_mg_fuse_rows (40000: the V-cycle
 * levels up to this size run as one kernel; 0: none), linsolver_mg_cluster
 * (16: thread blocks of that kernel's cluster, at most 16),
 * linsolver_mg_alpha (factor of the coarse-grid correction z += alpha P zc;
 * 1.4 on 3D grids, 1.9 on 2D grids), linsolver_mg_ap_rows (40000: levels
 * with more unknowns correct their residual through A P instead of
 * recomputing r - A z), linsolver_mg_coarsest (128: coarsening stops at
 * this many unknowns, at most 128; that level is solved with a dense
 * inverse), linsolver_pdl (1: the BiCGStab iteration's kernels
 * as programmatic dependent launches; 0: plain launches), linsolver_mg_local (1: that kernel keeps its coarsest levels in one thread
 * block's shared memory while they fit in 200 KB; 0: off),
 * linsolver_tail_trace (0; 1: print the SM clock cycles of every step of the
 * last fused cycle after each linear solve), lazy (0; 1:
 * defer value-only elementwise operations and evaluate them in batches),
 * fuse (1 on two-dimensional Cartesian grids, else 0: outside Newton solves,
 * defer value-only operations, On/Extend/gradient/divergence included, and
 * evaluate them as a fused explicit step where the deferred expressions are
 * one, else one kernel per operation; results are the same bits either way),
 * host_threads (0: OpenMP's default for the solver analysis),
 * linsolver_fallback (1: a solve that the multigrid preconditioner does not
 * converge is repeated once with block ILU(0) alone; 0: reported as a
 * failure), linsolver_autotune (1: choose threads per block of the launch-per-step
 * V-cycle levels and the fused cycle's cluster size by timing, once per
 * Jacobian pattern and precision; 0: 256 and the largest cluster),
 * linsolver_tune_file (a JSON file caching those choices; default
 * $EQG_TUNE_FILE, else none), spgemm_plan / span_share / jac_concat /
 * jac_defer / stencil_ops (1; 0 switches off an assembly fast path, for
 * comparisons),
 * gather_rows (0), flush_l2 (0; n: n MB written before each Newton solve's
 * start mark, so that a solve timed between its marks starts with a cold L2),
 * time_kernel
 * (a kernel name, or "*", to time with CUDA events) and device (CUDA device
 * index; default: the calling thread's current device).  grid_filename
 * (instead of grid_dim, nx, ...) reads the grid from a file: the arrays of an
 * UnstructuredGrid (face_cells, cell_facepos, cell_faces, face areas,
 * centroids and area-scaled normals, cell volumes and centroids) as text
 * after the header "eqg-grid 1" (layout: equelle_b200/grids.py, which writes
 * it); such a grid reports nx = ny = nz = 0, and its linear solves use block
 * ILU(0) (the multigrid preconditioner coarsens Cartesian grids only).
 * Replaces EquelleRuntimeCPU::EquelleRuntimeCPU(const ParameterGroup&)
 * and createGridManager (backends/serial/src/EquelleRuntimeCPU.cpp:20-65). */
int eqg_runtime_create(int nparams, const char* const* keys, const char* const* values,
                       eqg_runtime** out);
void eqg_runtime_destroy(eqg_runtime* rt);
int eqg_runtime_grid_info(const eqg_runtime* rt, eqg_grid_info* out);
int eqg_runtime_synchronize(eqg_runtime* rt);
int eqg_runtime_stats(const eqg_runtime* rt, eqg_stats* out);
int eqg_runtime_reset_stats(eqg_runtime* rt);
/* Device time per kernel name, as JSON
 * {"name": [launches, ms, bytes, launches_with_bytes], ...}, of the
 * launches timed under the parameter time_kernel (a name, or "*" for every
 * kernel); bytes sums the algorithmic bytes (data the launch's operation
 * must read and write at least once) of the launches that state them.
 * Writes at most len bytes (NUL terminated) and the size needed to
 * *needed. */
int eqg_runtime_kernel_profile(const eqg_runtime* rt, char* buf, int64_t len, int64_t* needed);
/* Timing marks: records an event on the runtime's stream (device clock for
 * the product, host steady clock for the oracle) and returns its id. */
int eqg_runtime_mark(eqg_runtime* rt, int* mark_id);
int eqg_runtime_elapsed_ms(eqg_runtime* rt, int mark_a, int mark_b, double* ms);
/* Newton-solve boundaries recorded automatically (one pair per solve):
 * start/end mark ids of solve k, or EQG_ERR_ARG if k is out of range. */
int eqg_runtime_solve_marks(const eqg_runtime* rt, int64_t k, int* start_mark, int* end_mark);

/* What solve k did. */
typedef struct eqg_solve_info {
    int start_mark, end_mark;
    int newton_iterations;
    int converged;              /* residual norm <= abs_res_tol at return   */
    int64_t krylov_iterations;
    int64_t kernel_launches;    /* device kernels launched during the solve */
    double residual_ms;         /* time in the solve's phases (as in          */
    double factor_ms;           /* eqg_stats: device clock for the product,  */
    double krylov_ms;           /* host clock for the oracle)                 */
} eqg_solve_info;
int eqg_runtime_solve_info(const eqg_runtime* rt, int64_t k, eqg_solve_info* out);

/* ---- entity collections (CollOfCell / CollOfFace) -------------------- */
/* allCells .. interiorFaces: EquelleRuntimeCPU.cpp:80-183.  The reference
 * rebuilds these vectors on every call; here they are built once and the
 * same handle is returned (retained) each time. */
int eqg_set_builtin(eqg_runtime* rt, int which, eqg_set** out);
int eqg_set_from_host(eqg_runtime* rt, int entity, const int32_t* idx, int64_t n, eqg_set** out);
int eqg_set_size(const eqg_set* s, int64_t* n);
int eqg_set_entity(const eqg_set* s, int* entity);
int eqg_set_to_host(const eqg_set* s, int32_t* out);
void eqg_set_retain(eqg_set* s);
void eqg_set_release(eqg_set* s);
/* firstCell / secondCell (EquelleRuntimeCPU.cpp:186-205). -1 = outside. */
int eqg_first_cell(eqg_runtime* rt, const eqg_set* faces, eqg_set** out);
int eqg_second_cell(eqg_runtime* rt, const eqg_set* faces, eqg_set** out);
/* isEmpty (EquelleRuntimeCPU.cpp:368-391). */
int eqg_set_is_empty(eqg_runtime* rt, const eqg_set* s, eqg_mask** out);
/* operatorOn / operatorExtend on entity collections
 * (EquelleRuntimeCPU_impl.hpp:113-141, index subset/superset :85-110).
 * Extend fills unmatched slots with -1 (a default-constructed entity). */
int eqg_set_on(eqg_runtime* rt, const eqg_set* data, const eqg_set* from, const eqg_set* to,
               eqg_set** out);
int eqg_set_extend(eqg_runtime* rt, const eqg_set* data, const eqg_set* from, const eqg_set* to,
                   eqg_set** out);
/* trinaryIf on entity collections (EquelleRuntimeCPU_impl.hpp:145-160). */
int eqg_set_select(eqg_runtime* rt, const eqg_mask* pred, const eqg_set* a, const eqg_set* b,
                   eqg_set** out);
/* The checks inputDomainSubsetOf makes (EquelleRuntimeCPU.cpp:506-511):
 * sub sorted ascending, and sub included in super. */
int eqg_set_check_subset(eqg_runtime* rt, const eqg_set* sub, const eqg_set* super,
                         int* is_sorted, int* is_included);

/* ---- boolean collections (CollOfBool, equelleTypes.hpp:43) ----------- */
int eqg_mask_from_host(eqg_runtime* rt, const uint8_t* v, int64_t n, eqg_mask** out);
int eqg_mask_size(const eqg_mask* m, int64_t* n);
int eqg_mask_to_host(const eqg_mask* m, uint8_t* out);
void eqg_mask_retain(eqg_mask* m);
void eqg_mask_release(eqg_mask* m);
/* b is ignored for EQG_NOT. */
int eqg_mask_logic(eqg_runtime* rt, int op, const eqg_mask* a, const eqg_mask* b, eqg_mask** out);

/* ---- scalar collections (CollOfScalar = AutoDiffBlock<double>,
 *      equelleTypes.hpp:67-84) ---------------------------------------- */
int eqg_coll_from_host(eqg_runtime* rt, const double* v, int64_t n, eqg_coll** out);
/* operatorExtend(Scalar, set) (EquelleRuntimeCPU_impl.hpp:15-20). */
int eqg_coll_constant(eqg_runtime* rt, double v, int64_t n, eqg_coll** out);
int eqg_coll_size(const eqg_coll* c, int64_t* n);
int eqg_coll_to_host(const eqg_coll* c, double* out);
/* Computes a collection's values now if the runtime has deferred them (the
 * fuse and lazy parameters); no effect otherwise.  The header's output()
 * calls it before its timing marks. */
int eqg_coll_evaluate(eqg_runtime* rt, const eqg_coll* c);
/* Asynchronous output (the copies behind EquelleRuntimeCPU::output,
 * EquelleRuntimeCPU_impl.hpp:342-365): eqg_output_begin starts copying the
 * values to library-owned host memory after the work already enqueued and
 * returns at once with a ticket; eqg_output_wait blocks until that copy is
 * done and gives its values, valid until eqg_output_release.  Wait and
 * release may be called from another thread than the runtime's. */
int eqg_output_begin(eqg_runtime* rt, const eqg_coll* c, int64_t* ticket);
int eqg_output_wait(eqg_runtime* rt, int64_t ticket, const double** values, int64_t* n);
int eqg_output_release(eqg_runtime* rt, int64_t ticket);
/* nnz = -1 when the collection carries no Jacobian (an ADB constant). */
int eqg_coll_jacobian_info(const eqg_coll* c, int64_t* rows, int64_t* cols, int64_t* nnz);
/* CSR with ascending column indices; explicit zeros of the symbolic
 * pattern are kept (AutoDiffBlock/Eigen semantics). */
int eqg_coll_jacobian_to_host(const eqg_coll* c, int64_t* rowptr, int32_t* colind, double* vals);
void eqg_coll_retain(eqg_coll* c);
void eqg_coll_release(eqg_coll* c);

/* singlePrimaryVariable: identity Jacobian, one block
 * (EquelleRuntimeCPU.cpp:565-571). */
int eqg_variable(eqg_runtime* rt, const eqg_coll* init, eqg_coll** out);
/* Drops the Jacobian (u.value() in EquelleRuntimeCPU_impl.hpp:278). */
int eqg_value_of(eqg_runtime* rt, const eqg_coll* c, eqg_coll** out);

/* a op b with the AutoDiffBlock sum, product and quotient rules
 * (restated by SINTEF in backends/cuda/src/collOfScalar.cu:273-401). */
int eqg_binary(eqg_runtime* rt, int op, const eqg_coll* a, const eqg_coll* b, eqg_coll** out);
/* a op s (scalar_left = 0) or s op a (scalar_left = 1):
 * equelleTypes.hpp:93-102 and the ADB scalar operators. */
int eqg_binary_scalar(eqg_runtime* rt, int op, const eqg_coll* a, double s, int scalar_left,
                      eqg_coll** out);
/* -x (equelleTypes.hpp:87-90), sqrt (:195-211),
 * abs = norm(CollOfScalar) (EquelleRuntimeCPU.cpp:241-254). */
int eqg_unary(eqg_runtime* rt, int op, const eqg_coll* a, eqg_coll** out);
/* Comparisons -> CollOfBool on values (equelleTypes.hpp:105-192). */
int eqg_compare(eqg_runtime* rt, int op, const eqg_coll* a, const eqg_coll* b, eqg_mask** out);
int eqg_compare_scalar(eqg_runtime* rt, int op, const eqg_coll* a, double s, int scalar_left,
                       eqg_mask** out);

/* gradient / negGradient / divergence / interiorDivergence
 * (EquelleRuntimeCPU.cpp:339-365; HelperOps as restated in
 * backends/cuda/src/deviceHelperOps.cpp:84-148).  divergence of a
 * collection on interior faces switches to interiorDivergence, as the
 * reference does (EquelleRuntimeCPU.cpp:353-357). */
int eqg_gradient(eqg_runtime* rt, const eqg_coll* cells, eqg_coll** out);
int eqg_neg_gradient(eqg_runtime* rt, const eqg_coll* cells, eqg_coll** out);
int eqg_divergence(eqg_runtime* rt, const eqg_coll* faces, eqg_coll** out);
int eqg_interior_divergence(eqg_runtime* rt, const eqg_coll* faces, eqg_coll** out);

/* operatorOn / operatorExtend (EquelleRuntimeCPU_impl.hpp:113-141). */
int eqg_on(eqg_runtime* rt, const eqg_coll* data, const eqg_set* from, const eqg_set* to,
           eqg_coll** out);
int eqg_extend(eqg_runtime* rt, const eqg_coll* data, const eqg_set* from, const eqg_set* to,
               eqg_coll** out);
/* trinaryIf on CollOfScalar: iftrue*mask + iffalse*(1-mask), Jacobian
 * pattern = union of both branches (EquelleRuntimeCPU_impl.hpp:163-180). */
int eqg_select(eqg_runtime* rt, const eqg_mask* pred, const eqg_coll* a, const eqg_coll* b,
               eqg_coll** out);
/* Opm::subset / Opm::superset with ESpan(num, 1, start), as used by
 * newtonSolveSystem (EquelleRuntimeCPU_impl.hpp:306-337). */
int eqg_span_subset(eqg_runtime* rt, const eqg_coll* a, int64_t start, int64_t num,
                    eqg_coll** out);
int eqg_span_superset(eqg_runtime* rt, const eqg_coll* a, int64_t start, int64_t total,
                      eqg_coll** out);

/* min/max/sum/prodReduce (EquelleRuntimeCPU.cpp:393-411). */
int eqg_reduce(eqg_runtime* rt, int op, const eqg_coll* a, double* out);
/* twoNorm (EquelleRuntimeCPU.cpp:443-446). */
int eqg_two_norm(eqg_runtime* rt, const eqg_coll* a, double* out);

/* ---- geometry -------------------------------------------------------- */
/* norm(faces) = areas, norm(cells) = volumes (EquelleRuntimeCPU.cpp:208-227). */
int eqg_measure(eqg_runtime* rt, const eqg_set* s, eqg_coll** out);
/* Column `component` of centroid(...) (EquelleRuntimeCPU.cpp:257-292). */
int eqg_centroid(eqg_runtime* rt, const eqg_set* s, int component, eqg_coll** out);
/* Column `component` of the UNIT face normal (EquelleRuntimeCPU.cpp:295-314). */
int eqg_normal(eqg_runtime* rt, const eqg_set* faces, int component, eqg_coll** out);

/* ---- Newton solver --------------------------------------------------- */
/* The residual callback receives u (with Jacobian) and must return the
 * residual in *residual (one reference), or a nonzero status. */
typedef int (*eqg_residual_fn)(void* user, const eqg_coll* u, eqg_coll** residual);
/* newtonSolve (EquelleRuntimeCPU_impl.hpp:210-279): stops when
 * twoNorm(residual) <= abs_res_tol or after max_iter updates; returns u
 * without Jacobian.  Non-convergence of Newton is not an error (the
 * reference only prints); a failed linear solve is EQG_ERR_SOLVER
 * ("Linear solver convergence failure.", EquelleRuntimeCPU.cpp:436-438). */
int eqg_newton_solve(eqg_runtime* rt, eqg_residual_fn fn, void* user, const eqg_coll* u0,
                     eqg_coll** out);
/* solveForUpdate (EquelleRuntimeCPU.cpp:413-440): du with J du = F,
 * J = residual's Jacobian. */
int eqg_solve_for_update(eqg_runtime* rt, const eqg_coll* residual, eqg_coll** du);

#ifdef __cplusplus
}
#endif

#endif /* EQG_H */

"""ctypes declarations of the C ABI in include/eqg.h.

`bind(cdll)` sets argument and result types on any library exporting the
ABI; `SYMBOLS` lists every function the header declares (tests check that
both libraries export all of them).
"""
import ctypes as C

c_int_p = C.POINTER(C.c_int)
c_i64_p = C.POINTER(C.c_int64)
c_i32_p = C.POINTER(C.c_int32)
c_u8_p = C.POINTER(C.c_uint8)
c_dbl_p = C.POINTER(C.c_double)
vp = C.c_void_p
vpp = C.POINTER(C.c_void_p)

EQG_OK = 0
EQG_ERR_ARG = 1
EQG_ERR_DEVICE = 2
EQG_ERR_SOLVER = 3
EQG_ERR_UNSUPPORTED = 4
EQG_ERR_CALLBACK = 5
EQG_ERR_MEMORY = 6

CELLS, FACES = 0, 1
ALL_CELLS, BOUNDARY_CELLS, INTERIOR_CELLS, ALL_FACES, BOUNDARY_FACES, INTERIOR_FACES = range(6)
ADD, SUB, MUL, DIV = range(4)
NEG, SQRT, ABS = range(3)
LT, LE, GT, GE, EQ, NE = range(6)
MIN, MAX, SUM, PROD = range(4)
AND, OR, NOT = range(3)


class GridInfo(C.Structure):
    _fields_ = [
        ("dimensions", C.c_int), ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
        ("dx", C.c_double), ("dy", C.c_double), ("dz", C.c_double),
        ("number_of_cells", C.c_int64), ("number_of_faces", C.c_int64),
        ("number_of_interior_faces", C.c_int64),
    ]


class Stats(C.Structure):
    _fields_ = [
        ("kernel_launches", C.c_int64), ("newton_solves", C.c_int64),
        ("newton_iterations", C.c_int64), ("linear_solves", C.c_int64),
        ("krylov_iterations", C.c_int64), ("refinement_sweeps", C.c_int64),
        ("patterns_built", C.c_int64), ("pattern_cache_hits", C.c_int64),
        ("device_bytes_in_use", C.c_int64), ("device_bytes_peak", C.c_int64),
        ("last_linear_residual", C.c_double),
        ("last_matrix_rows", C.c_int64), ("last_matrix_nnz", C.c_int64),
        ("timed_kernel_launches", C.c_int64), ("timed_kernel_ms", C.c_double),
        ("residual_evaluations", C.c_int64), ("residual_ms", C.c_double),
        ("factor_ms", C.c_double), ("krylov_ms", C.c_double),
        ("last_block_size", C.c_int64), ("last_matrix_blocks", C.c_int64),
        ("fused_evaluations", C.c_int64),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class SolveInfo(C.Structure):
    _fields_ = [
        ("start_mark", C.c_int), ("end_mark", C.c_int), ("newton_iterations", C.c_int),
        ("converged", C.c_int), ("krylov_iterations", C.c_int64), ("kernel_launches", C.c_int64),
        ("residual_ms", C.c_double), ("factor_ms", C.c_double), ("krylov_ms", C.c_double),
    ]


RESIDUAL_FN = C.CFUNCTYPE(C.c_int, vp, vp, vpp)

# name -> (restype, argtypes)
SIGNATURES = {
    "eqg_last_error": (C.c_char_p, []),
    "eqg_backend_name": (C.c_char_p, []),
    "eqg_runtime_create": (C.c_int, [C.c_int, C.POINTER(C.c_char_p), C.POINTER(C.c_char_p), vpp]),
    "eqg_runtime_destroy": (None, [vp]),
    "eqg_runtime_grid_info": (C.c_int, [vp, C.POINTER(GridInfo)]),
    "eqg_runtime_synchronize": (C.c_int, [vp]),
    "eqg_runtime_stats": (C.c_int, [vp, C.POINTER(Stats)]),
    "eqg_runtime_reset_stats": (C.c_int, [vp]),
    "eqg_runtime_kernel_profile": (C.c_int, [vp, C.c_char_p, C.c_int64, c_i64_p]),
    "eqg_runtime_mark": (C.c_int, [vp, c_int_p]),
    "eqg_runtime_elapsed_ms": (C.c_int, [vp, C.c_int, C.c_int, c_dbl_p]),
    "eqg_runtime_solve_marks": (C.c_int, [vp, C.c_int64, c_int_p, c_int_p]),
    "eqg_runtime_solve_info": (C.c_int, [vp, C.c_int64, C.POINTER(SolveInfo)]),
    "eqg_set_builtin": (C.c_int, [vp, C.c_int, vpp]),
    "eqg_set_from_host": (C.c_int, [vp, C.c_int, c_i32_p, C.c_int64, vpp]),
    "eqg_set_size": (C.c_int, [vp, c_i64_p]),
    "eqg_set_entity": (C.c_int, [vp, c_int_p]),
    "eqg_set_to_host": (C.c_int, [vp, c_i32_p]),
    "eqg_set_retain": (None, [vp]),
    "eqg_set_release": (None, [vp]),
    "eqg_first_cell": (C.c_int, [vp, vp, vpp]),
    "eqg_second_cell": (C.c_int, [vp, vp, vpp]),
    "eqg_set_is_empty": (C.c_int, [vp, vp, vpp]),
    "eqg_set_on": (C.c_int, [vp, vp, vp, vp, vpp]),
    "eqg_set_extend": (C.c_int, [vp, vp, vp, vp, vpp]),
    "eqg_set_select": (C.c_int, [vp, vp, vp, vp, vpp]),
    "eqg_set_check_subset": (C.c_int, [vp, vp, vp, c_int_p, c_int_p]),
    "eqg_mask_from_host": (C.c_int, [vp, c_u8_p, C.c_int64, vpp]),
    "eqg_mask_size": (C.c_int, [vp, c_i64_p]),
    "eqg_mask_to_host": (C.c_int, [vp, c_u8_p]),
    "eqg_mask_retain": (None, [vp]),
    "eqg_mask_release": (None, [vp]),
    "eqg_mask_logic": (C.c_int, [vp, C.c_int, vp, vp, vpp]),
    "eqg_coll_from_host": (C.c_int, [vp, c_dbl_p, C.c_int64, vpp]),
    "eqg_coll_constant": (C.c_int, [vp, C.c_double, C.c_int64, vpp]),
    "eqg_coll_size": (C.c_int, [vp, c_i64_p]),
    "eqg_coll_to_host": (C.c_int, [vp, c_dbl_p]),
    "eqg_coll_evaluate": (C.c_int, [vp, vp]),
    "eqg_output_begin": (C.c_int, [vp, vp, c_i64_p]),
    "eqg_output_wait": (C.c_int, [vp, C.c_int64, C.POINTER(c_dbl_p), c_i64_p]),
    "eqg_output_release": (C.c_int, [vp, C.c_int64]),
    "eqg_coll_jacobian_info": (C.c_int, [vp, c_i64_p, c_i64_p, c_i64_p]),
    "eqg_coll_jacobian_to_host": (C.c_int, [vp, c_i64_p, c_i32_p, c_dbl_p]),
    "eqg_coll_retain": (None, [vp]),
    "eqg_coll_release": (None, [vp]),
    "eqg_variable": (C.c_int, [vp, vp, vpp]),
    "eqg_value_of": (C.c_int, [vp, vp, vpp]),
    "eqg_binary": (C.c_int, [vp, C.c_int, vp, vp, vpp]),
    "eqg_binary_scalar": (C.c_int, [vp, C.c_int, vp, C.c_double, C.c_int, vpp]),
    "eqg_unary": (C.c_int, [vp, C.c_int, vp, vpp]),
    "eqg_compare": (C.c_int, [vp, C.c_int, vp, vp, vpp]),
    "eqg_compare_scalar": (C.c_int, [vp, C.c_int, vp, C.c_double, C.c_int, vpp]),
    "eqg_gradient": (C.c_int, [vp, vp, vpp]),
    "eqg_neg_gradient": (C.c_int, [vp, vp, vpp]),
    "eqg_divergence": (C.c_int, [vp, vp, vpp]),
    "eqg_interior_divergence": (C.c_int, [vp, vp, vpp]),
    "eqg_on": (C.c_int, [vp, vp, vp, vp, vpp]),
    "eqg_extend": (C.c_int, [vp, vp, vp, vp, vpp]),
    "eqg_select": (C.c_int, [vp, vp, vp, vp, vpp]),
    "eqg_span_subset": (C.c_int, [vp, vp, C.c_int64, C.c_int64, vpp]),
    "eqg_span_superset": (C.c_int, [vp, vp, C.c_int64, C.c_int64, vpp]),
    "eqg_reduce": (C.c_int, [vp, C.c_int, vp, c_dbl_p]),
    "eqg_two_norm": (C.c_int, [vp, vp, c_dbl_p]),
    "eqg_measure": (C.c_int, [vp, vp, vpp]),
    "eqg_centroid": (C.c_int, [vp, vp, C.c_int, vpp]),
    "eqg_normal": (C.c_int, [vp, vp, C.c_int, vpp]),
    "eqg_newton_solve": (C.c_int, [vp, RESIDUAL_FN, vp, vp, vpp]),
    "eqg_solve_for_update": (C.c_int, [vp, vp, vpp]),
}

SYMBOLS = tuple(SIGNATURES)


class EqgError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(msg)
        self.code = code


def bind(lib):
    """Declare every ABI function on `lib` (a ctypes.CDLL); returns lib."""
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


def check(lib, status):
    if status != EQG_OK:
        raise EqgError(status, lib.eqg_last_error().decode())

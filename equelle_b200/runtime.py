"""Python mirror of equelle::EquelleRuntimeCPU over the C ABI.

Same method names and argument meaning as the C++ class generated
simulators use (sintefmath/equelle backends/serial/include/equelle/
EquelleRuntimeCPU.hpp:35-134), so simulators and tests can be written in
the generated style from Python.  Works with any library that exports the
ABI of include/eqg.h: the device runtime (equelle_b200.load_library()) or
the CPU oracle used by the tests.
"""
import ctypes as C

import numpy as np

from . import capi


class _Handle:
    _release = None

    def __init__(self, rt, h):
        self.rt = rt
        self.h = h

    def __del__(self):
        h, self.h = getattr(self, "h", None), None
        if h:
            getattr(self.rt.lib, self._release)(h)


class EntitySet(_Handle):
    """CollOfCell / CollOfFace."""
    _release = "eqg_set_release"

    def __len__(self):
        n = C.c_int64()
        self.rt._ok(self.rt.lib.eqg_set_size(self.h, C.byref(n)))
        return n.value

    def size(self):
        return len(self)

    @property
    def entity(self):
        e = C.c_int()
        self.rt._ok(self.rt.lib.eqg_set_entity(self.h, C.byref(e)))
        return e.value

    def indices(self):
        out = np.empty(len(self), dtype=np.int32)
        if out.size:
            self.rt._ok(self.rt.lib.eqg_set_to_host(self.h, out.ctypes.data_as(capi.c_i32_p)))
        return out


class CollOfBool(_Handle):
    _release = "eqg_mask_release"

    def __len__(self):
        n = C.c_int64()
        self.rt._ok(self.rt.lib.eqg_mask_size(self.h, C.byref(n)))
        return n.value

    def values(self):
        out = np.empty(len(self), dtype=np.uint8)
        if out.size:
            self.rt._ok(self.rt.lib.eqg_mask_to_host(self.h, out.ctypes.data_as(capi.c_u8_p)))
        return out.astype(bool)

    def _logic(self, op, other):
        return self.rt._mask(self.rt.lib.eqg_mask_logic, op, self.h, other.h if other is not None else None)

    def __and__(self, o):
        return self._logic(capi.AND, o)

    def __or__(self, o):
        return self._logic(capi.OR, o)

    def __invert__(self):
        return self._logic(capi.NOT, None)


class CollOfScalar(_Handle):
    """Value plus optional Jacobian (AutoDiffBlock<double>)."""
    _release = "eqg_coll_release"

    def __len__(self):
        n = C.c_int64()
        self.rt._ok(self.rt.lib.eqg_coll_size(self.h, C.byref(n)))
        return n.value

    def size(self):
        return len(self)

    def value(self):
        out = np.empty(len(self), dtype=np.float64)
        if out.size:
            self.rt._ok(self.rt.lib.eqg_coll_to_host(self.h, out.ctypes.data_as(capi.c_dbl_p)))
        return out

    def jacobian(self):
        """(rows, cols, rowptr, colind, vals) or None for a constant."""
        r, c, nnz = C.c_int64(), C.c_int64(), C.c_int64()
        self.rt._ok(self.rt.lib.eqg_coll_jacobian_info(self.h, C.byref(r), C.byref(c), C.byref(nnz)))
        if nnz.value < 0:
            return None
        ptr = np.empty(r.value + 1, dtype=np.int64)
        col = np.empty(max(nnz.value, 1), dtype=np.int32)
        val = np.empty(max(nnz.value, 1), dtype=np.float64)
        self.rt._ok(self.rt.lib.eqg_coll_jacobian_to_host(
            self.h, ptr.ctypes.data_as(capi.c_i64_p), col.ctypes.data_as(capi.c_i32_p),
            val.ctypes.data_as(capi.c_dbl_p)))
        return r.value, c.value, ptr, col[:nnz.value], val[:nnz.value]

    # arithmetic (equelleTypes.hpp:86-211)
    def _bin(self, op, other, reflected=False):
        rt = self.rt
        if isinstance(other, CollOfScalar):
            a, b = (other, self) if reflected else (self, other)
            return rt._coll(rt.lib.eqg_binary, op, a.h, b.h)
        return rt._coll(rt.lib.eqg_binary_scalar, op, self.h, float(other), 1 if reflected else 0)

    def __add__(self, o):
        return self._bin(capi.ADD, o)

    def __radd__(self, o):
        return self._bin(capi.ADD, o, True)

    def __sub__(self, o):
        return self._bin(capi.SUB, o)

    def __rsub__(self, o):
        return self._bin(capi.SUB, o, True)

    def __mul__(self, o):
        return self._bin(capi.MUL, o)

    def __rmul__(self, o):
        return self._bin(capi.MUL, o, True)

    def __truediv__(self, o):
        return self._bin(capi.DIV, o)

    def __rtruediv__(self, o):
        return self._bin(capi.DIV, o, True)

    def __neg__(self):
        return self.rt._coll(self.rt.lib.eqg_unary, capi.NEG, self.h)

    def _cmp(self, op, other):
        rt = self.rt
        if isinstance(other, CollOfScalar):
            return rt._mask(rt.lib.eqg_compare, op, self.h, other.h)
        return rt._mask(rt.lib.eqg_compare_scalar, op, self.h, float(other), 0)

    def __lt__(self, o):
        return self._cmp(capi.LT, o)

    def __le__(self, o):
        return self._cmp(capi.LE, o)

    def __gt__(self, o):
        return self._cmp(capi.GT, o)

    def __ge__(self, o):
        return self._cmp(capi.GE, o)

    def eq(self, o):
        return self._cmp(capi.EQ, o)

    def ne(self, o):
        return self._cmp(capi.NE, o)


class CollOfVector:
    def __init__(self, cols):
        self.cols = list(cols)

    def col(self, i):
        return self.cols[i]

    def numCols(self):
        return len(self.cols)

    def __getitem__(self, i):
        return self.cols[i]

    def __add__(self, o):
        return CollOfVector(a + b for a, b in zip(self.cols, o.cols))

    def __sub__(self, o):
        return CollOfVector(a - b for a, b in zip(self.cols, o.cols))

    def __neg__(self):
        return CollOfVector(-a for a in self.cols)

    def __mul__(self, s):
        return CollOfVector(a * s for a in self.cols)

    __rmul__ = __mul__

    def __truediv__(self, s):
        return CollOfVector(a / s for a in self.cols)


class Runtime:
    """equelle::EquelleRuntimeCPU over a library exporting include/eqg.h."""

    def __init__(self, lib, params):
        self.lib = lib
        keys = [str(k).encode() for k in params]
        vals = [str(v).lower() if isinstance(v, bool) else str(v) for v in params.values()]
        vals = [v.encode() for v in vals]
        karr = (C.c_char_p * len(keys))(*keys)
        varr = (C.c_char_p * len(vals))(*vals)
        h = C.c_void_p()
        self._ok(lib.eqg_runtime_create(len(keys), karr, varr, C.byref(h)))
        self.h = h.value
        info = capi.GridInfo()
        self._ok(lib.eqg_runtime_grid_info(self.h, C.byref(info)))
        self.info = info
        self.dimensions = info.dimensions

    def __del__(self):
        h, self.h = getattr(self, "h", None), None
        if h:
            self.lib.eqg_runtime_destroy(h)

    # -- plumbing --------------------------------------------------------
    def _ok(self, status):
        capi.check(self.lib, status)

    def _out(self, fn, cls, *args):
        out = C.c_void_p()
        self._ok(fn(self.h, *args, C.byref(out)))
        return cls(self, out.value)

    def _coll(self, fn, *args):
        return self._out(fn, CollOfScalar, *args)

    def _mask(self, fn, *args):
        return self._out(fn, CollOfBool, *args)

    def _set(self, fn, *args):
        return self._out(fn, EntitySet, *args)

    # -- data in/out -----------------------------------------------------
    def collection(self, values):
        v = np.ascontiguousarray(values, dtype=np.float64)
        return self._coll(self.lib.eqg_coll_from_host, v.ctypes.data_as(capi.c_dbl_p), v.size)

    def constant(self, value, n):
        return self._coll(self.lib.eqg_coll_constant, float(value), int(n))

    def entity_set(self, entity, indices):
        idx = np.ascontiguousarray(indices, dtype=np.int32)
        return self._set(self.lib.eqg_set_from_host, entity, idx.ctypes.data_as(capi.c_i32_p), idx.size)

    def mask(self, values):
        v = np.ascontiguousarray(values, dtype=np.uint8)
        return self._mask(self.lib.eqg_mask_from_host, v.ctypes.data_as(capi.c_u8_p), v.size)

    def variable(self, init):
        return self._coll(self.lib.eqg_variable, init.h)

    # -- topology --------------------------------------------------------
    def allCells(self):
        return self._set(self.lib.eqg_set_builtin, capi.ALL_CELLS)

    def boundaryCells(self):
        return self._set(self.lib.eqg_set_builtin, capi.BOUNDARY_CELLS)

    def interiorCells(self):
        return self._set(self.lib.eqg_set_builtin, capi.INTERIOR_CELLS)

    def allFaces(self):
        return self._set(self.lib.eqg_set_builtin, capi.ALL_FACES)

    def boundaryFaces(self):
        return self._set(self.lib.eqg_set_builtin, capi.BOUNDARY_FACES)

    def interiorFaces(self):
        return self._set(self.lib.eqg_set_builtin, capi.INTERIOR_FACES)

    def firstCell(self, faces):
        return self._set(self.lib.eqg_first_cell, faces.h)

    def secondCell(self, faces):
        return self._set(self.lib.eqg_second_cell, faces.h)

    def norm(self, x):
        if isinstance(x, EntitySet):
            return self._coll(self.lib.eqg_measure, x.h)
        if isinstance(x, CollOfVector):
            n2 = x.col(0) * x.col(0)
            for d in range(1, x.numCols()):
                n2 = n2 + x.col(d) * x.col(d)
            return self.sqrt(n2)
        return self._coll(self.lib.eqg_unary, capi.ABS, x.h)

    def centroid(self, s):
        return CollOfVector(self._coll(self.lib.eqg_centroid, s.h, d) for d in range(self.dimensions))

    def normal(self, faces):
        return CollOfVector(self._coll(self.lib.eqg_normal, faces.h, d) for d in range(self.dimensions))

    # -- math ------------------------------------------------------------
    def sqrt(self, x):
        return self._coll(self.lib.eqg_unary, capi.SQRT, x.h)

    def dot(self, v1, v2):
        r = v1.col(0) * v2.col(0)
        for d in range(1, self.dimensions):
            r = r + v1.col(d) * v2.col(d)
        return r

    def gradient(self, x):
        return self._coll(self.lib.eqg_gradient, x.h)

    def negGradient(self, x):
        return self._coll(self.lib.eqg_neg_gradient, x.h)

    def divergence(self, x):
        return self._coll(self.lib.eqg_divergence, x.h)

    def interiorDivergence(self, x):
        return self._coll(self.lib.eqg_interior_divergence, x.h)

    def isEmpty(self, s):
        return self._mask(self.lib.eqg_set_is_empty, s.h)

    def operatorExtend(self, data, a, b=None):
        if b is None:
            return self.constant(data, len(a))
        if isinstance(data, EntitySet):
            return self._set(self.lib.eqg_set_extend, data.h, a.h, b.h)
        return self._coll(self.lib.eqg_extend, data.h, a.h, b.h)

    def operatorOn(self, data, from_set, to_set):
        if isinstance(data, EntitySet):
            return self._set(self.lib.eqg_set_on, data.h, from_set.h, to_set.h)
        return self._coll(self.lib.eqg_on, data.h, from_set.h, to_set.h)

    def trinaryIf(self, pred, a, b):
        if isinstance(a, EntitySet):
            return self._set(self.lib.eqg_set_select, pred.h, a.h, b.h)
        return self._coll(self.lib.eqg_select, pred.h, a.h, b.h)

    # -- reductions ------------------------------------------------------
    def _reduce(self, op, x):
        r = C.c_double()
        self._ok(self.lib.eqg_reduce(self.h, op, x.h, C.byref(r)))
        return r.value

    def minReduce(self, x):
        return self._reduce(capi.MIN, x)

    def maxReduce(self, x):
        return self._reduce(capi.MAX, x)

    def sumReduce(self, x):
        return self._reduce(capi.SUM, x)

    def prodReduce(self, x):
        return self._reduce(capi.PROD, x)

    def twoNorm(self, x):
        r = C.c_double()
        self._ok(self.lib.eqg_two_norm(self.h, x.h, C.byref(r)))
        return r.value

    # -- solvers ---------------------------------------------------------
    def newtonSolve(self, rescomp, u0):
        err = []

        def tramp(user, u, out):
            try:
                self.lib.eqg_coll_retain(u)
                r = rescomp(CollOfScalar(self, u))
                self.lib.eqg_coll_retain(r.h)
                out[0] = r.h
                return 0
            except Exception as e:  # reported after the C call returns
                err.append(e)
                return 1

        cb = capi.RESIDUAL_FN(tramp)
        out = C.c_void_p()
        st = self.lib.eqg_newton_solve(self.h, cb, None, u0.h, C.byref(out))
        if err:
            raise err[0]
        self._ok(st)
        return CollOfScalar(self, out.value)

    def newtonSolveSystem(self, rescomps, u0s):
        """EquelleRuntimeCPU_impl.hpp:282-339 for any number of blocks."""
        num = [len(u) for u in u0s]
        start = np.concatenate([[0], np.cumsum(num)[:-1]]).astype(int)
        total = int(sum(num))

        def sub(u, i):
            return self._coll(self.lib.eqg_span_subset, u.h, int(start[i]), int(num[i]))

        def sup(x, i):
            return self._coll(self.lib.eqg_span_superset, x.h, int(start[i]), total)

        def combined(u):
            parts = [sub(u, i) for i in range(len(num))]
            res = [f(*parts) for f in rescomps]
            r = sup(res[0], 0)
            for i in range(1, len(res)):
                r = r + sup(res[i], i)
            return r

        u0 = sup(u0s[0], 0)
        for i in range(1, len(u0s)):
            u0 = u0 + sup(u0s[i], i)
        u = self.newtonSolve(combined, u0)
        return tuple(sub(u, i) for i in range(len(num)))

    def spanSubset(self, u, start, num):
        """Opm::subset(u, ESpan(num, 1, start))."""
        return self._coll(self.lib.eqg_span_subset, u.h, int(start), int(num))

    def spanSuperset(self, u, start, total):
        """Opm::superset(u, ESpan(len(u), 1, start), total)."""
        return self._coll(self.lib.eqg_span_superset, u.h, int(start), int(total))

    def solveForUpdate(self, residual):
        return self._coll(self.lib.eqg_solve_for_update, residual.h)

    # -- stats and timing ------------------------------------------------
    def stats(self):
        s = capi.Stats()
        self._ok(self.lib.eqg_runtime_stats(self.h, C.byref(s)))
        return s.as_dict()

    def reset_stats(self):
        self._ok(self.lib.eqg_runtime_reset_stats(self.h))

    def mark(self):
        m = C.c_int()
        self._ok(self.lib.eqg_runtime_mark(self.h, C.byref(m)))
        return m.value

    def elapsed_ms(self, a, b):
        ms = C.c_double()
        self._ok(self.lib.eqg_runtime_elapsed_ms(self.h, a, b, C.byref(ms)))
        return ms.value

    def solve_marks(self, k):
        s, e = C.c_int(), C.c_int()
        self._ok(self.lib.eqg_runtime_solve_marks(self.h, k, C.byref(s), C.byref(e)))
        return s.value, e.value

    def synchronize(self):
        self._ok(self.lib.eqg_runtime_synchronize(self.h))

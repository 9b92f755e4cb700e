"""Deferred evaluation of value-only elementwise operations (runtime
parameter lazy=1): every field is bit-identical to the
one-kernel-per-operation path (lazy=0 fuse=0), with fewer kernel launches."""
import numpy as np
import pytest

import opstream
from equelle_b200 import programs
from equelle_b200.runtime import Runtime

pytestmark = pytest.mark.gpu


def _same(a, b):
    assert len(a) == len(b)
    for x, y in zip(a, b):
        if isinstance(x, (tuple, list)):
            _same(x, y)
        else:
            assert np.array_equal(np.asarray(x), np.asarray(y))


def test_lazy_shallow_water_identical(gpu_lib):
    grid, case = programs.swe_case(64, 48, steps=6, sigma=6.0)
    lazy = Runtime(gpu_lib, dict(grid, lazy=1))
    eager = Runtime(gpu_lib, dict(grid, lazy=0, fuse=0))
    _same(programs.swe(lazy, **case), programs.swe(eager, **case))
    assert lazy.stats()["kernel_launches"] < 0.5 * eager.stats()["kernel_launches"]


def test_lazy_implicit_programs_identical(gpu_lib):
    grid, case = programs.two_phase_case(8, 8, 4, steps=2)
    params = dict(grid, abs_res_tol=1e-10, linsolver_residual_tolerance=1e-10, linsolver_max_iterations=5000)
    _same(programs.two_phase(Runtime(gpu_lib, dict(params, lazy=1)), **case),
          programs.two_phase(Runtime(gpu_lib, dict(params, lazy=0, fuse=0)), **case))
    grid, case = programs.heat_case(32, 32, steps=4)
    params = dict(grid, abs_res_tol=1e-10, linsolver_residual_tolerance=1e-12)
    _same(programs.heat_equation(Runtime(gpu_lib, dict(params, lazy=1)), 0.3, 1.0, **case),
          programs.heat_equation(Runtime(gpu_lib, dict(params, lazy=0, fuse=0)), 0.3, 1.0, **case))


@pytest.mark.parametrize("grid", opstream.GRIDS, ids=["2d", "3d"])
def test_lazy_op_stream_identical(gpu_lib, grid):
    lazy = Runtime(gpu_lib, dict(grid, lazy=1))
    eager = Runtime(gpu_lib, dict(grid, lazy=0, fuse=0))
    a, b = opstream.op_stream(lazy), opstream.op_stream(eager)
    for k in a:
        assert np.array_equal(a[k].value(), b[k].value()), k
        ja, jb = a[k].jacobian(), b[k].jacobian()
        assert (ja is None) == (jb is None), k
        if ja is not None:
            for x, y in zip(ja, jb):
                assert np.array_equal(np.asarray(x), np.asarray(y)), k
    assert opstream.reductions(lazy) == opstream.reductions(eager)
    ma, mb = opstream.masks(lazy), opstream.masks(eager)
    for k in ma:
        assert np.array_equal(ma[k], mb[k]), k

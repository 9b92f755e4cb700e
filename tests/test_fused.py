"""Fused explicit steps (runtime parameter fuse, fused.cu): the shallow-water
step computed by the fused kernels when the deferred operations match it,
bit-identical to one kernel per operation (fuse=0), on grids whose size is
not a multiple of the kernels' tiles, with dry cells and with non-square
cells; programs that do not match evaluate per operation, with the same
bits as well."""
import os

import numpy as np
import pytest

from equelle_b200 import cases, programs, simrun
from equelle_b200.runtime import Runtime

pytestmark = pytest.mark.gpu


def _same(a, b):
    assert len(a) == len(b)
    for step, (x, y) in enumerate(zip(a, b)):
        for k, (u, v) in enumerate(zip(x, y)):
            assert np.array_equal(np.asarray(u), np.asarray(v)), "field %d step %d" % (k, step)


def _dry_case(nx, ny, steps, dx=1.0, dy=1.0):
    """A lake: wet bumps over a domain whose left third is (nearly) dry."""
    grid, case = programs.swe_case(nx, ny, steps=steps, sigma=4.0, amplitude=0.3, dx=dx, dy=dy)
    h = case["h_init"].reshape(ny, nx).copy()
    h[:, : nx // 3] = 0.02
    h[ny // 2:, : nx // 6] = 0.0
    case["h_init"] = np.ascontiguousarray(h.reshape(-1))
    return grid, case


@pytest.mark.parametrize("shape,kind", [((64, 48), "plain"), ((33, 70), "plain"), ((5, 3), "plain"),
                                        ((45, 37), "dry"), ((40, 24), "cells")],
                         ids=["64x48", "33x70", "5x3", "dry", "non-square-cells"])
def test_fused_step_identical_to_per_operation(gpu_lib, shape, kind):
    if kind == "dry":
        grid, case = _dry_case(*shape, steps=8)
    elif kind == "cells":
        grid, case = programs.swe_case(*shape, steps=8, sigma=5.0, dx=2.0, dy=0.5)
    else:
        grid, case = programs.swe_case(*shape, steps=8, sigma=5.0)
    fused = Runtime(gpu_lib, dict(grid, fuse=1))
    plain = Runtime(gpu_lib, dict(grid, fuse=0))
    a = programs.swe(fused, **case)
    b = programs.swe(plain, **case)
    _same(a, b)
    sf, sp = fused.stats(), plain.stats()
    # one fused step and one fused wave-speed maximum per time step
    assert sf["fused_evaluations"] >= 2 * 8 - 1
    assert sp["fused_evaluations"] == 0
    assert sf["kernel_launches"] < 0.2 * sp["kernel_launches"]
    if kind == "dry":
        w, hu, hv = a[-1]
        bottom = (case["b_north"] + case["b_south"] + case["b_east"] + case["b_west"]) / 4.0
        assert np.sum(w - bottom <= 0.05) > 0  # dry cells remain


def test_fused_simulator_identical(gpu_lib, tmp_path):
    """The generated-style C++ program (sims/swe.cpp) on the device: its
    outputs with fusion are those without, and fusion ran."""
    outs = {}
    for fuse in (1, 0):
        d = tmp_path / ("f%d" % fuse)
        d.mkdir()
        args = cases.swe(str(d), 50, 38, steps=6, sigma=5.0)
        rep = simrun.run("swe", args + ["output_values=last", "output_dir=%s/" % d, "fuse=%d" % fuse])
        assert rep.solves == 6
        outs[fuse] = [np.loadtxt(os.path.join(d, "%s-last.output" % t)) for t in ("q1", "q2", "q3")]
        if fuse:
            assert rep.stats.fused_evaluations >= 11
        else:
            assert rep.stats.fused_evaluations == 0
    for x, y in zip(outs[1], outs[0]):
        assert np.array_equal(x, y)


def test_unmatched_programs_evaluate_per_operation(gpu_lib):
    """Programs that are not the fused step (an implicit heat equation and
    two-phase flow on a 2D grid, whose set-up values are deferred) give
    the same bits with and without fusion, and no fused step runs."""
    grid, case = programs.heat_case(32, 32, steps=3)
    params = dict(grid, abs_res_tol=1e-10, linsolver_residual_tolerance=1e-12)
    rf, rp = Runtime(gpu_lib, dict(params, fuse=1)), Runtime(gpu_lib, dict(params, fuse=0))
    a = programs.heat_equation(rf, 0.3, 1.0, **case)
    b = programs.heat_equation(rp, 0.3, 1.0, **case)
    for x, y in zip(a, b):
        assert np.array_equal(np.asarray(x), np.asarray(y))
    assert rf.stats()["fused_evaluations"] == 0
    grid, case = programs.two_phase_case(12, 10, steps=2)
    params = dict(grid, abs_res_tol=1e-10, linsolver_residual_tolerance=1e-10, linsolver_max_iterations=5000)
    rf, rp = Runtime(gpu_lib, dict(params, fuse=1)), Runtime(gpu_lib, dict(params, fuse=0))
    _same(programs.two_phase(rf, **case), programs.two_phase(rp, **case))
    assert rf.stats()["fused_evaluations"] == 0


def test_changed_step_is_not_fused(gpu_lib):
    """A step that differs from the fused one in one operation (a different
    Heun weight) is evaluated per operation: still identical to fuse=0,
    and only the wave-speed maximum is fused."""
    grid, case = programs.swe_case(24, 20, steps=4, sigma=4.0)
    runs = {}
    for fuse in (1, 0):
        rt = Runtime(gpu_lib, dict(grid, fuse=fuse))
        runs[fuse] = (programs.swe(rt, heun_weight=0.25, **case), rt.stats())
    _same(runs[1][0], runs[0][0])
    assert runs[1][1]["fused_evaluations"] <= 4

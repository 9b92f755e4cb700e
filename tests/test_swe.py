"""Explicit shallow-water program (equelle_b200/sims/swe.cpp and its Python
mirror programs.swe): the value-only path of the runtime.

CPU tests run the oracle; GPU tests compare the device library with the
oracle through the same op stream, and the C++ simulator with the Python
mirror on the device."""
import os

import numpy as np
import pytest

from equelle_b200 import cases, programs, simrun
from equelle_b200.runtime import Runtime

ORACLE_SIM = os.path.join(os.path.dirname(__file__), "..", "oracle", "_build", "libsim_swe_oracle.so")


def _bottom(case):
    return (case["b_north"] + case["b_south"] + case["b_east"] + case["b_west"]) / 4.0


def _last_outputs(d):
    return [np.loadtxt(os.path.join(d, "%s-last.output" % tag)) for tag in ("q1", "q2", "q3")]


def test_swe_oracle_conserves_mass_and_matches_simulator(oracle_lib, tmp_path):
    """On the oracle: the water volume is conserved to rounding over the
    run, and the C++ simulator gives the Python mirror's fields."""
    grid, case = programs.swe_case(48, 40, steps=6, sigma=5.0)
    out = programs.swe(Runtime(oracle_lib, grid), **case)
    b = _bottom(case)
    v0 = case["h_init"].sum()
    for w, hu, hv in out:
        assert abs((w - b).sum() - v0) <= 1e-12 * v0
        assert np.all(np.isfinite(hu)) and np.all(np.isfinite(hv))
    assert np.max(np.abs(out[-1][1])) > 1e-3  # the bumps have started to move
    args = cases.swe(str(tmp_path), 48, 40, steps=6, sigma=5.0)
    rep = simrun.run("swe", args + ["output_values=last", "output_dir=%s/" % tmp_path], path=ORACLE_SIM)
    assert rep.solves == 6
    for got, want in zip(_last_outputs(str(tmp_path)), out[-1]):
        assert np.array_equal(got, want)


@pytest.mark.gpu
@pytest.mark.parametrize("shape", [(64, 48), (33, 70)])
def test_swe_device_matches_oracle(gpu_lib, oracle_lib, shape):
    """Device vs oracle, 10 steps: every field within 1e-9 relative to its
    largest magnitude after every step."""
    grid, case = programs.swe_case(*shape, steps=10, sigma=6.0)
    g = programs.swe(Runtime(gpu_lib, grid), **case)
    o = programs.swe(Runtime(oracle_lib, grid), **case)
    for step, (fg, fo) in enumerate(zip(g, o)):
        for k, (a, b) in enumerate(zip(fg, fo)):
            scale = max(np.max(np.abs(b)), 1e-300)
            assert np.max(np.abs(a - b)) <= 1e-9 * scale, "field %d step %d" % (k, step)


@pytest.mark.gpu
def test_swe_simulator_matches_mirror_on_device(gpu_lib, tmp_path):
    """The C++ simulator and the Python mirror issue the same operations:
    bit-identical fields on the device."""
    grid, case = programs.swe_case(40, 36, steps=5, sigma=5.0)
    out = programs.swe(Runtime(gpu_lib, grid), **case)
    args = cases.swe(str(tmp_path), 40, 36, steps=5, sigma=5.0)
    rep = simrun.run("swe", args + ["output_values=last", "output_dir=%s/" % tmp_path])
    assert rep.solves == 5
    for got, want in zip(_last_outputs(str(tmp_path)), out[-1]):
        assert np.array_equal(got, want)

"""The reference's generated simulators (examples/app/out_*.cpp, built
unchanged on the oracle by `make -C oracle ref`) on the CPU: each runs on
the inputs of the GPU tests and its outputs hold what the physics
guarantees (finite values, water volume conserved by the explicit
shallow-water program, saturations in [0, 1]); explicit programs report
their time steps from the tag they output most often."""
import glob
import os

import numpy as np
import pytest

import test_reference_programs as ref
from equelle_b200 import cases, simrun

REF_BUILD = ref.REF_BUILD


def _oracle(name):
    path = os.path.join(REF_BUILD, "libref_%s_oracle.so" % name)
    if not os.path.exists(path):
        pytest.skip("%s is not built (the reference tree was absent at build time)" % path)
    return path


def _series(d, tag):
    return [np.atleast_1d(np.loadtxt(f)) for f in sorted(glob.glob(os.path.join(d, tag + "-*.output")))]


def _programs():
    seen = {}
    for p in ref.PROGRAMS:
        values = p.values if hasattr(p, "marks") else p  # a pytest.param, or a plain tuple
        seen.setdefault(values[0], values[1])
    return sorted(seen.items())


@pytest.mark.parametrize("name,inputs", _programs(), ids=[n for n, _ in _programs()])
def test_reference_program_runs_on_oracle(tmp_path, name, inputs):
    d = str(tmp_path / "in")
    os.makedirs(d)
    out = str(tmp_path / "out")
    ref._run(name, _oracle(name), inputs(d), out)
    files = glob.glob(os.path.join(out, "*.output"))
    assert files
    for f in files:
        v = np.atleast_1d(np.loadtxt(f))
        assert np.all(np.isfinite(v)), f
    if name.startswith("out_twophase"):
        for sw in _series(out, "saturation"):
            assert sw.min() >= -1e-9 and sw.max() <= 1.0 + 1e-9


def test_reference_shallow_water_conserves_volume(tmp_path):
    """out_swe.cpp: walls all around, so the water volume (the sum of
    w - b over the cells) stays the initial one to rounding; its step count
    comes from q1, the tag it outputs every step."""
    d = str(tmp_path / "in")
    args = cases.swe_reference(d, 40, 30, steps=6, dt=0.3)
    out = str(tmp_path / "out")
    rep = ref._run("out_swe", _oracle("out_swe"), args, out)
    bottom = np.loadtxt(glob.glob(os.path.join(out, "bottom-*.output"))[0])
    q1 = _series(out, "q1")
    assert len(q1) == 7
    v0 = float(np.sum(q1[0] - bottom))
    for w in q1[1:]:
        assert abs(float(np.sum(w - bottom)) - v0) <= 1e-11 * abs(v0)
    assert float(np.max(np.abs(q1[-1] - q1[0]))) > 1e-6  # the bumps have moved
    rep2 = simrun.run("out_swe", args + ["output_values=off"], path=_oracle("out_swe"))
    assert rep2.solves == 6

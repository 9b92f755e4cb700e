"""The reference's other generated simulators (sintefmath/equelle
examples/app/out_*.cpp), compiled unchanged against the header twice by
`make -C oracle ref` (oracle/_ref/libref_<program>_{device,oracle}.so), run
on the same seeded inputs: every output file of the device build equals the
oracle build's within 1e-9 of the file's largest magnitude (1e-8 where a
Newton or linear solve runs, 1e-7 for the conservation form below; the
pressures of systems without a pressure anchor up to their mean, since
every Jacobian there is singular with the constant pressure as null
vector).  Heat, the fully implicit two-phase program and
shallow water are in test_sims.py."""
import glob
import os

import numpy as np
import pytest

from equelle_b200 import cases, programs, simrun

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_BUILD = os.path.join(ROOT, "oracle", "_ref")


def _write(d, name, values, fmt="%.17g"):
    path = os.path.join(d, name + ".txt")
    np.savetxt(path, np.asarray(values).reshape(-1), fmt=fmt)
    return path


def _grid_only(d):
    return ["grid_dim=2", "nx=7", "ny=5", "dx=1.5", "dy=2.0"]


def _sw(d):
    grid, c = programs.swe_case(20, 16, steps=1, sigma=3.0)
    return ["%s=%s" % kv for kv in grid.items()] + [
        "h0_from_file=true", "h0_filename=" + _write(d, "h0", c["h_init"]), "hu0=0", "hv0=0"]


def _compressible(d):
    nx, ny = 16, 12
    q = np.zeros(nx * ny)
    q[0], q[-1] = 1e-2, -1e-2
    return ["grid_dim=2", "nx=%d" % nx, "ny=%d" % ny, "dx=10", "dy=10",
            "source_from_file=true", "source_filename=" + _write(d, "source", q),
            "timesteps_filename=" + _write(d, "timesteps", [3600.0] * 3),
            "abs_res_tol=1e-10", "linsolver_residual_tolerance=1e-12", "linsolver_max_iterations=20000"]


def _impes_2d(d):
    # one linear pressure solve per step: fluxes derived from its gradient
    # are compared, so the solves run to 1e-12
    return cases.two_phase(d, 12, 10, None, steps=3, corr_len=4.0) + [
        "abs_res_tol=1e-10", "linsolver_residual_tolerance=1e-12", "linsolver_max_iterations=50000"]


def _conservation_2d(d):
    # The conservation form stacks a water and an oil equation, each
    # depending on pressure: the constant pressure shift is a null vector of
    # every Jacobian and so is, on the left, the sum of all rows, whose
    # (sw - sw0) + (so - so0) terms cancel only to rounding.  The right-hand
    # side is therefore off the Jacobian's range by about one rounding error
    # per cell, which no linear tolerance relative to a small Newton residual
    # can beat (the oracle itself fails at abs_res_tol 1e-12).  Newton stops
    # at 1e-6 here, so every linear solve runs at a residual of 3e-4 or more;
    # its last update leaves ~3e-8, so fields are compared to 1e-7.
    return cases.two_phase(d, 16, 16, None, steps=3, corr_len=4.0) + [
        "abs_res_tol=1e-6", "linsolver_residual_tolerance=1e-9", "linsolver_max_iterations=20000"]


PROGRAMS = [
    ("out_testops", _grid_only, 1e-9, False, []),
    ("out_test_normals_dot", _grid_only, 1e-9, False, []),
    ("out_sw", _sw, 1e-9, False, []),
    ("out_compr_singlephase", _compressible, 1e-8, False, []),
    ("out_twophase", _impes_2d, 1e-8, True, []),
    ("out_twophase_grav", _impes_2d, 1e-8, True, []),
    pytest.param("out_twophase_fully_implicit_conservation", _conservation_2d, 1e-7, True, [],
                 id="out_twophase_fully_implicit_conservation-multigrid"),
    pytest.param("out_twophase_fully_implicit_conservation", _conservation_2d, 1e-7, True,
                 ["linsolver_preconditioner=ilu0"], id="out_twophase_fully_implicit_conservation-ilu0"),
]


def _run(name, lib, args, out):
    os.makedirs(out, exist_ok=True)
    return simrun.run(name, args + ["output_to_file=true", "output_dir=%s/" % out], path=lib)


@pytest.mark.parametrize("name,inputs,tol,unanchored,device_args", PROGRAMS,
                         ids=[None if hasattr(p, "marks") else p[0] for p in PROGRAMS])
def test_reference_program_device_matches_oracle(tmp_path, name, inputs, tol, unanchored, device_args):
    libs = {}
    for side in ("device", "oracle"):
        libs[side] = os.path.join(REF_BUILD, "libref_%s_%s.so" % (name, side))
        if not os.path.exists(libs[side]):
            pytest.fail("%s is not built (python -c 'import __graft_entry__ as g; g.build()')" % libs[side])
    d = str(tmp_path / "in")
    os.makedirs(d)
    args = inputs(d)
    outs = {side: str(tmp_path / side) for side in libs}
    for side in libs:
        _run(name, libs[side], args + (device_args if side == "device" else []), outs[side])
    files = {side: sorted(os.path.basename(f) for f in glob.glob(os.path.join(outs[side], "*.output")))
             for side in libs}
    assert files["device"] == files["oracle"] and files["device"], name
    for f in files["device"]:
        a = np.atleast_1d(np.loadtxt(os.path.join(outs["device"], f)))
        b = np.atleast_1d(np.loadtxt(os.path.join(outs["oracle"], f)))
        assert a.shape == b.shape, f
        if unanchored and f.startswith("pressure"):
            a, b = a - a.mean(), b - b.mean()
        scale = max(float(np.max(np.abs(b))), 1e-300)
        err = float(np.max(np.abs(a - b)))
        assert err <= tol * scale, "%s %s: %g of %g" % (name, f, err, scale)

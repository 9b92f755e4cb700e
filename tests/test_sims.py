"""Generated simulators built twice from one C++ source: once against the
device library (libeqg.so) and once against the CPU oracle, run with the
same input files, their output files compared field by field.

Programs:
- equelle_b200/sims/heateq.cpp and twophase.cpp, the programs bench.py
  times (C++ header layer: systemSolve stacking, CollOfVector, the
  inputCollectionOfScalar / inputDomainSubsetOf / inputSequenceOfScalar
  readers and the output_to_file writer, `tag-%05d.output`);
- sintefmath/equelle's own generated examples/app/out_heateq.cpp and
  out_twophase_fully_implicit.cpp, compiled unchanged by `make -C oracle ref`
  into oracle/_ref/ (libref_<program>_{device,oracle}.so).

Tolerances: heat fields 1e-9 relative per cell; saturation 1e-8 relative
per cell; pressure 1e-8 of its largest magnitude.
"""
import glob
import os

import numpy as np
import pytest

from equelle_b200 import LIB_DIR, cases, simrun

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_BUILD = os.path.join(ROOT, "oracle", "_build")
REF_BUILD = os.path.join(ROOT, "oracle", "_ref")


def _series(d, tag):
    files = sorted(glob.glob(os.path.join(d, tag + "-*.output")))
    return [np.loadtxt(f) for f in files]


def _run(name, path, args, out):
    os.makedirs(out, exist_ok=True)
    rep = simrun.run(name, args + ["output_to_file=true", "output_dir=%s/" % out], path=path)
    return rep


def _pair(name, device_path, oracle_path, args, tmp, device_args=()):
    """Runs the device and oracle builds of one program; returns the two
    output directories and reports."""
    dev, ora = os.path.join(tmp, "device"), os.path.join(tmp, "oracle")
    rd = _run(name, device_path, list(args) + list(device_args), dev)
    ro = _run(name, oracle_path, list(args), ora)
    return dev, ora, rd, ro


def _need(path):
    if not os.path.exists(path):
        pytest.fail("%s is not built (python -c 'import __graft_entry__ as g; g.build()')" % path)
    return path


def _rel_per_cell(a, b):
    return float(np.max(np.abs(a - b) / np.abs(b)))


def _check_heat(dev, ora, steps):
    ug, uo = _series(dev, "u"), _series(ora, "u")
    assert len(ug) == len(uo) == steps + 1
    for k, (a, b) in enumerate(zip(ug, uo)):
        err = _rel_per_cell(a, b)
        assert err <= 1e-9, "u after step %d: max rel err %g" % (k, err)


def _check_two_phase(dev, ora, steps, pressure_mod_constant=False):
    sg, so = _series(dev, "saturation"), _series(ora, "saturation")
    pg, po = _series(dev, "pressure"), _series(ora, "pressure")
    assert len(sg) == len(so) == len(pg) == len(po) == steps + 1
    worst = 0.0
    for k in range(steps + 1):
        err = _rel_per_cell(sg[k], so[k])
        worst = max(worst, err)
        assert err <= 1e-8, "Sw after step %d: max rel err %g" % (k, err)
        a, b = pg[k], po[k]
        if pressure_mod_constant:
            a, b = a - a.mean(), b - b.mean()
        scale = max(float(np.max(np.abs(b))), 1e-300)
        assert float(np.max(np.abs(a - b))) <= 1e-8 * scale, "p after step %d" % k
    return worst


# --------------------------------------------------------------------------
def test_heat_simulator_matches_oracle(tmp_path):
    """sims/heateq.cpp on the 64x64 heat configuration (20 steps of 0.5,
    Dirichlet u = 0.5 on the left faces): every output field."""
    args = cases.heat(str(tmp_path / "in"), 64, 64, steps=20)
    dev, ora, rd, _ = _pair("heateq", os.path.join(LIB_DIR, "libsim_heateq.so"),
                            _need(os.path.join(ORACLE_BUILD, "libsim_heateq_oracle.so")), args, str(tmp_path))
    assert rd.solves == 20
    _check_heat(dev, ora, 20)


def test_reference_heat_program_matches_oracle(tmp_path):
    """sintefmath/equelle's examples/app/out_heateq.cpp, unchanged, on the
    same inputs."""
    args = cases.heat(str(tmp_path / "in"), 64, 64, steps=20)
    dev, ora, rd, _ = _pair("out_heateq", _need(os.path.join(REF_BUILD, "libref_out_heateq_device.so")),
                            _need(os.path.join(REF_BUILD, "libref_out_heateq_oracle.so")), args, str(tmp_path))
    assert rd.solves == 20
    _check_heat(dev, ora, 20)


def _check_swe(dev, ora, steps):
    for tag in ("q1", "q2", "q3"):
        g, o = _series(dev, tag), _series(ora, tag)
        assert len(g) == len(o) == steps + 1
        for k, (a, b) in enumerate(zip(g, o)):
            scale = max(float(np.max(np.abs(b))), 1e-300)
            assert float(np.max(np.abs(a - b))) <= 1e-9 * scale, "%s after step %d" % (tag, k)


def test_reference_swe_program_matches_oracle(tmp_path):
    """sintefmath/equelle's examples/app/out_swe.cpp (Kurganov-Levy fluxes,
    time steps read from a file), unchanged: every output field within 1e-9
    of its largest magnitude after every step.  On the device its values
    are deferred (fuse=1, a 2D Cartesian grid) and, its step not being the
    fused one, evaluated one kernel per operation: the same bits as
    without deferral (fuse=0)."""
    args = cases.swe_reference(str(tmp_path / "in"), 40, 30, steps=6, dt=0.3)
    device = _need(os.path.join(REF_BUILD, "libref_out_swe_device.so"))
    dev, ora, rd, _ = _pair("out_swe", device, _need(os.path.join(REF_BUILD, "libref_out_swe_oracle.so")), args,
                            str(tmp_path))
    _check_swe(dev, ora, 6)
    assert rd.stats.fused_evaluations == 0
    last = {}
    for fuse in (1, 0):
        d = str(tmp_path / ("last%d" % fuse))
        os.makedirs(d)
        simrun.run("out_swe", args + ["output_values=last", "output_dir=%s/" % d, "fuse=%d" % fuse], path=device)
        last[fuse] = [np.loadtxt(os.path.join(d, "%s-last.output" % t)) for t in ("q1", "q2", "q3")]
    for a, b in zip(last[1], last[0]):
        assert np.array_equal(a, b)


TWO_PHASE_TOL = ["abs_res_tol=1e-8", "linsolver_residual_tolerance=1e-8", "linsolver_max_iterations=50000"]


@pytest.mark.parametrize("shape,steps", [((16, 16, 8), 3), ((48, 40, None), 3)], ids=["16x16x8", "48x40"])
def test_two_phase_simulator_matches_oracle(tmp_path, shape, steps):
    """sims/twophase.cpp (the program bench.py times), FP64 default
    solver."""
    nx, ny, nz = shape
    args = cases.two_phase(str(tmp_path / "in"), nx, ny, nz, steps=steps,
                           corr_len=8.0 if nz else 4.0) + TWO_PHASE_TOL
    dev, ora, rd, _ = _pair("twophase", os.path.join(LIB_DIR, "libsim_twophase.so"),
                            _need(os.path.join(ORACLE_BUILD, "libsim_twophase_oracle.so")), args, str(tmp_path))
    assert rd.solves == steps
    _check_two_phase(dev, ora, steps)


_BIG = {}


def _big_case(tmp_root):
    """32x32x32 two-phase, 3 steps: 65,536 unknowns, so at the default
    settings the V-cycle has five levels, the top one above the A P
    up-leg's 40,000-unknown threshold with coarse-correction factor 1.4, and
    every lower level inside the fused cluster kernel (its coarsest in one
    block's shared memory).  The oracle runs once per session."""
    if "args" not in _BIG:
        d = os.path.join(tmp_root, "big")
        args = cases.two_phase(os.path.join(d, "in"), 32, 32, 32, steps=3) + TWO_PHASE_TOL
        ora = os.path.join(d, "oracle")
        _run("twophase", _need(os.path.join(ORACLE_BUILD, "libsim_twophase_oracle.so")), args, ora)
        _BIG.update(args=args, oracle=ora)
    return _BIG["args"], _BIG["oracle"]


@pytest.mark.parametrize("precision", ["double", "mixed", "refine"])
def test_two_phase_32x32x32_every_solver_feature_matches_oracle(tmp_path_factory, precision):
    """The default solver with all its parts engaged, in each precision
    form: Sw within 1e-8 of the FP64 oracle after every step."""
    args, ora = _big_case(str(tmp_path_factory.getbasetemp()))
    dev = str(tmp_path_factory.mktemp("dev_" + precision))
    rd = _run("twophase", os.path.join(LIB_DIR, "libsim_twophase.so"),
              args + ["linsolver_precision=" + precision, "verbose=0"], dev)
    assert rd.solves == 3
    _check_two_phase(dev, ora, 3)


@pytest.mark.parametrize("precond", ["multigrid", "ilu0"])
def test_reference_two_phase_program_matches_oracle(tmp_path, precond):
    """sintefmath/equelle's examples/app/out_twophase_fully_implicit.cpp,
    unchanged, 2D 16x16, 3 steps.  Its pressure equation has no anchor, so
    every Jacobian is singular with the null vector (p = 1, Sw = 0); a
    Krylov solve of the consistent system still converges, and pressure is
    compared up to its mean."""
    args = cases.two_phase(str(tmp_path / "in"), 16, 16, None, steps=3, corr_len=4.0) + [
        "abs_res_tol=1e-12", "linsolver_residual_tolerance=1e-9", "linsolver_max_iterations=20000"]
    dev, ora, rd, _ = _pair("out_twophase_fully_implicit",
                            _need(os.path.join(REF_BUILD, "libref_out_twophase_fully_implicit_device.so")),
                            _need(os.path.join(REF_BUILD, "libref_out_twophase_fully_implicit_oracle.so")),
                            args, str(tmp_path), device_args=["linsolver_preconditioner=" + precond])
    assert rd.solves == 3
    _check_two_phase(dev, ora, 3, pressure_mod_constant=True)

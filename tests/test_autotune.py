"""Launch-shape autotuning of the linear solver (linsolver_autotune).

The tuner picks threads per block for every launch-per-step V-cycle level
and the fused cycle's cluster size by timing preconditioner applications.
A row's arithmetic does not depend on the launch shape, so a solve with the
tuner gives bit-identical fields to one without it; the choices are cached
in a JSON file that a later runtime reads back.
"""
import json
import os

import numpy as np
import pytest

from equelle_b200 import programs
from equelle_b200.runtime import Runtime

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("shape,extra", [((16, 16, 8), dict(linsolver_mg_fuse_rows=0)),
                                         ((24, 24, 16), dict()),
                                         ((16, 16, 8), dict(linsolver_preconditioner="ilu0"))],
                         ids=["launch-levels", "default", "ilu0"])
def test_autotuned_solves_are_bit_identical(gpu_lib, tmp_path, shape, extra):
    grid, case = programs.two_phase_case(*shape, steps=2)
    params = dict(grid, abs_res_tol=1e-10, linsolver_residual_tolerance=1e-10, linsolver_max_iterations=5000,
                  **extra)
    tune_file = str(tmp_path / "tune.json")
    plain = programs.two_phase(Runtime(gpu_lib, dict(params, linsolver_autotune=0)), **case)
    tuned = programs.two_phase(Runtime(gpu_lib, dict(params, linsolver_tune_file=tune_file)), **case)
    for (pa, sa), (pb, sb) in zip(plain, tuned):
        assert np.array_equal(pa, pb) and np.array_equal(sa, sb)
    with open(tune_file) as f:
        entries = json.load(f)
    assert len(entries) >= 1
    for choice in entries.values():
        assert all(t in (128, 256, 512) for t in choice["threads"])
        assert choice["cluster"] >= 0
    # a new runtime takes the choices from the file: the same fields again
    again = programs.two_phase(Runtime(gpu_lib, dict(params, linsolver_tune_file=tune_file)), **case)
    for (pa, sa), (pb, sb) in zip(plain, again):
        assert np.array_equal(pa, pb) and np.array_equal(sa, sb)
    assert os.path.exists(tune_file)

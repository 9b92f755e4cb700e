"""The allocation-free 2-norm entry point (include/eqg_noalloc.h).

Callers that cannot allocate device memory -- code inside a stream capture
that must not add allocation nodes, programs whose device memory an outside
pool owns -- pass their own input and output buffers to
eqg_two_norm_noalloc, which keeps its scratch in a fixed array inside the
library.  The test checks it, through the C ABI, against the runtime's own
two-norm (eqg_two_norm) on the same values, on two calls in a row, within
the relative tolerance the parity tests use (1e-12).  Device buffers come
from torch, owned by the test.

This file sorts last so that a run stopping at the first failure has run
every other test first.
"""
import ctypes

import numpy as np
import pytest

from equelle_b200.runtime import Runtime
from parity import RTOL

pytestmark = pytest.mark.gpu

MAX_ELEMENTS = 65536 * 256


def _bind(lib):
    fn = lib.eqg_two_norm_noalloc
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p]
    return fn


def _reference_norm(lib, values):
    rt = Runtime(lib, dict(grid_dim=2, nx=4, ny=3))
    return rt.twoNorm(rt.collection(values))


def test_two_norm_noalloc_matches_runtime(gpu_lib):
    import torch

    fn = _bind(gpu_lib)
    gen = torch.Generator(device="cuda").manual_seed(7)
    result = torch.empty(1, dtype=torch.float64, device="cuda")
    # two calls in a row on the shared scratch, the second smaller than the
    # first, then a third of the first size again
    for n in (3_000_017, 4_099, 3_000_017):
        x = torch.rand(n, dtype=torch.float64, device="cuda", generator=gen) - 0.5
        result.fill_(-1.0)
        st = fn(ctypes.c_void_p(x.data_ptr()), n, ctypes.c_void_p(result.data_ptr()), None)
        assert st == 0, gpu_lib.eqg_last_error().decode()
        torch.cuda.synchronize()
        got = float(result.item())
        want = _reference_norm(gpu_lib, x.cpu().numpy())
        assert abs(got - want) <= RTOL * abs(want), (n, got, want)


def test_two_norm_noalloc_limits(gpu_lib):
    import torch

    fn = _bind(gpu_lib)
    result = torch.empty(1, dtype=torch.float64, device="cuda")
    x = torch.zeros(1, dtype=torch.float64, device="cuda")
    # one element over the maximum is rejected before anything runs
    st = fn(ctypes.c_void_p(x.data_ptr()), MAX_ELEMENTS + 1, ctypes.c_void_p(result.data_ptr()), None)
    assert st == 1
    assert "outside" in gpu_lib.eqg_last_error().decode()
    # an empty input has norm zero
    result.fill_(-1.0)
    assert fn(None, 0, ctypes.c_void_p(result.data_ptr()), None) == 0
    torch.cuda.synchronize()
    assert float(result.item()) == 0.0
    # the largest input the scratch holds
    big = torch.full((MAX_ELEMENTS,), 0.5, dtype=torch.float64, device="cuda")
    assert fn(ctypes.c_void_p(big.data_ptr()), MAX_ELEMENTS, ctypes.c_void_p(result.data_ptr()), None) == 0
    torch.cuda.synchronize()
    want = 0.5 * np.sqrt(MAX_ELEMENTS)
    assert abs(float(result.item()) - want) <= RTOL * want

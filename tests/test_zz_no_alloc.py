"""The allocation-free 2-norm entry point (include/eqg_noalloc.h).

Callers that cannot allocate device memory -- a plugin inside a host
application whose own pool owns every device allocation, a program whose
device memory is budgeted once, up front -- pass their own input and output
buffers to eqg_two_norm_noalloc, which keeps its scratch in a fixed array
inside the library.  The test calls it through the C ABI and checks it
against a host FP64 sum of the same values and against the runtime's own
two-norm (eqg_two_norm), on two calls in a row, within the relative
tolerance the parity tests use (1e-12); and that the calls take no device
memory.  Device buffers come from torch, owned by the test.

This file sorts last so that a run stopping at the first failure has run
every other test first.
"""
import ctypes
import gc

import numpy as np
import pytest

from equelle_b200.runtime import Runtime
from parity import RTOL

pytestmark = pytest.mark.gpu


def _header_max_elements():
    """EQG_NOALLOC_MAX_ELEMENTS as include/eqg_noalloc.h defines it."""
    import os
    import re
    path = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "eqg_noalloc.h")
    with open(path) as f:
        m = re.search(r"#define\s+EQG_NOALLOC_MAX_ELEMENTS\s+\((\d+)LL\s*\*\s*(\d+)LL\)", f.read())
    assert m, "EQG_NOALLOC_MAX_ELEMENTS not found in %s" % path
    return int(m.group(1)) * int(m.group(2))


MAX_ELEMENTS = _header_max_elements()


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
    # the first call on the device loads the library's scratch array with
    # its module (memory held until exit); the calls checked come after it
    warm = torch.ones(8, dtype=torch.float64, device="cuda")
    assert fn(ctypes.c_void_p(warm.data_ptr()), 8, ctypes.c_void_p(result.data_ptr()), None) == 0
    # two calls in a row on the shared scratch, the second smaller than the
    # first, then a third of the first size again
    for n in (3_000_017, 4_099, 3_000_017):
        x = torch.rand(n, dtype=torch.float64, device="cuda", generator=gen) - 0.5
        result.fill_(-1.0)
        gc.collect()
        gc.disable()
        try:
            torch.cuda.synchronize()
            allocated, free = torch.cuda.memory_allocated(), torch.cuda.mem_get_info()[0]
            st = fn(ctypes.c_void_p(x.data_ptr()), n, ctypes.c_void_p(result.data_ptr()), None)
            assert st == 0, gpu_lib.eqg_last_error().decode()
            torch.cuda.synchronize()
            # nothing allocated: neither through torch's pool nor from the
            # driver (free memory did not shrink)
            assert torch.cuda.memory_allocated() == allocated
            assert torch.cuda.mem_get_info()[0] >= free
        finally:
            gc.enable()
        got = float(result.item())
        host = x.cpu().numpy()
        exact = float(np.sqrt(np.sum(host * host, dtype=np.float64)))
        assert abs(got - exact) <= RTOL * exact, (n, got, exact)
        want = _reference_norm(gpu_lib, host)
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

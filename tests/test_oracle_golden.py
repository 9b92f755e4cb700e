"""Pins the CPU oracle against the reference's golden vectors, and checks
that both libraries export every function include/eqg.h declares."""
import ctypes
import os
import re

import pytest

import kat
from conftest import ROOT
from equelle_b200 import capi


def test_oracle_grid_4x3(oracle_lib):
    kat.check_grid_4x3(oracle_lib)


def test_oracle_vals_on_grid(oracle_lib):
    kat.check_vals_on_grid(oracle_lib)


def _header_symbols():
    text = open(os.path.join(ROOT, "include", "eqg.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(eqg_\w+)\s*\(", text)))


def test_binding_covers_header():
    hdr = _header_symbols()
    assert hdr, "no declarations parsed"
    assert sorted(capi.SYMBOLS) == hdr


def test_oracle_exports_header(oracle_lib):
    for name in _header_symbols():
        assert hasattr(oracle_lib, name), name
    assert oracle_lib.eqg_backend_name() == b"cpu-oracle"


def test_device_library_exports_other_headers():
    """libeqg.so also exports what the other headers under include/ declare
    (the allocation-free entry point, which the oracle does not have)."""
    path = os.path.join(ROOT, "equelle_b200", "lib", "libeqg.so")
    if not os.path.exists(path):
        pytest.fail("libeqg.so not built: run __graft_entry__.build()")
    lib = ctypes.CDLL(path)
    inc = os.path.join(ROOT, "include")
    names = []
    for h in sorted(os.listdir(inc)):
        if h.endswith(".h") and h != "eqg.h":
            names += re.findall(r"\b(eqg_\w+)\s*\(", open(os.path.join(inc, h)).read())
    assert names, "no declarations parsed"
    for name in sorted(set(names)):
        assert hasattr(lib, name), name


def test_device_library_exports_header():
    """libeqg.so loads without a GPU and exports the whole ABI."""
    path = os.path.join(ROOT, "equelle_b200", "lib", "libeqg.so")
    if not os.path.exists(path):
        pytest.fail("libeqg.so not built: run __graft_entry__.build()")
    lib = ctypes.CDLL(path)
    for name in _header_symbols():
        assert hasattr(lib, name), name
    capi.bind(lib)
    assert lib.eqg_backend_name() == b"cuda-sm100a"

"""equelle_b200: a B200-native runtime for Equelle-generated simulators.

The product is the shared library libeqg.so (CUDA for sm_100a) behind the C
ABI of include/eqg.h, plus the header-only C++ layer include/equelle/ that
generated simulators compile against.  This Python package holds the build
recipe, ctypes bindings and a Python mirror of the runtime API used by
tests and bench.py.
"""
import ctypes
import os

from . import capi  # noqa: F401

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
ROOT_DIR = os.path.dirname(PKG_DIR)
LIB_DIR = os.path.join(PKG_DIR, "lib")
LIB_PATH = os.path.join(LIB_DIR, "libeqg.so")
INCLUDE_DIR = os.path.join(ROOT_DIR, "include")

_lib = None


def load_library(path=LIB_PATH):
    """Load and bind libeqg.so.  Raises if it has not been built: there is
    no fallback implementation."""
    global _lib
    if _lib is not None and path == LIB_PATH:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(
            "libeqg.so is not built (%s); run `python -c \"import __graft_entry__ as g; g.build()\"`" % path)
    lib = capi.bind(ctypes.CDLL(path, mode=ctypes.RTLD_LOCAL))
    if path == LIB_PATH:
        _lib = lib
    return lib


def Runtime(params, lib=None):
    """An EquelleRuntimeCPU mirror on the device library."""
    from .runtime import Runtime as _R
    return _R(lib or load_library(), params)

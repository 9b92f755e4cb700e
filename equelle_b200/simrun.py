"""Run a generated-style simulator in this process through its shared
library's `eqg_sim_main` (equelle_b200/sims/sim_entry.cpp)."""
import ctypes as C
import os
import threading

from . import LIB_DIR, capi

MAX_SOLVES = 4096


class SimReport(C.Structure):
    _fields_ = [
        ("solves", C.c_int64),
        ("solve_ms", C.c_double * MAX_SOLVES),
        ("gap_ms", C.c_double * MAX_SOLVES),
        ("info", capi.SolveInfo * MAX_SOLVES),
        ("total_ms", C.c_double),
        ("stats", capi.Stats),
        ("error", C.c_char * 512),
        ("profile", C.c_char * 16384),
    ]


_loaded = {}
_load_lock = threading.Lock()


def sim_library(name, path=None):
    """The device build (equelle_b200/lib/libsim_<name>.so) unless `path`
    names another build of the same simulator source."""
    path = path or os.path.join(LIB_DIR, "libsim_%s.so" % name)
    with _load_lock:
        return _load(path)


def _load(path):
    if path not in _loaded:
        if not os.path.exists(path):
            raise RuntimeError("simulator library %s is not built" % path)
        lib = C.CDLL(path, mode=C.RTLD_LOCAL)
        lib.eqg_sim_main.restype = C.c_int
        lib.eqg_sim_main.argtypes = [C.c_int, C.POINTER(C.c_char_p), C.POINTER(SimReport)]
        _loaded[path] = lib
    return _loaded[path]


def run(name, args, path=None, allow_failure=False):
    """Runs the simulator with `key=value` args; returns the report.  With
    allow_failure, a run that stopped with an exception returns its report
    (counters up to the failure, message in report.error)."""
    lib = sim_library(name, path)
    argv = [b"sim_" + name.encode()] + [a.encode() for a in args]
    arr = (C.c_char_p * len(argv))(*argv)
    rep = SimReport()
    rc = lib.eqg_sim_main(len(argv), arr, C.byref(rep))
    if rc != 0 and not allow_failure:
        raise RuntimeError("simulator %s failed: %s" % (name, rep.error.decode()))
    return rep

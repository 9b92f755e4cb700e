"""Build recipe for libeqg.so (sm_100a) and the generated-style simulators.

    python -m equelle_b200.build            # library + simulators
    python -m equelle_b200.build --lib      # library only

nvcc cross-compiles for sm_100a without a GPU; each .cu file is compiled in
parallel and linked into equelle_b200/lib/libeqg.so.  The simulators in
equelle_b200/sims/ are plain C++ (g++) against include/ and link libeqg.so.
"""
import argparse
import concurrent.futures as cf
import glob
import os
import subprocess
import sys

from . import INCLUDE_DIR, LIB_DIR, LIB_PATH, PKG_DIR

CSRC = os.path.join(PKG_DIR, "csrc")
SIMS = os.path.join(PKG_DIR, "sims")
OBJ_DIR = os.path.join(PKG_DIR, "_build")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
# The system compiler.  A wrapper g++ that puts its own include directories
# ahead of the system C++ headers built shared objects that crashed in
# std::istringstream once loaded into a Python process, so the build does
# not take g++ from $CXX or the PATH.
CXX = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "-Xcompiler", "-fPIC",
    "-Xcompiler", "-fopenmp",  # host loops of the solver analysis
    "-Xptxas", "-v" if os.environ.get("EQG_PTXAS_VERBOSE") else "-O3",
    "-I" + INCLUDE_DIR, "-I" + CSRC,
    "-ccbin", CXX,
]


def _run(cmd):
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if r.returncode != 0:
        raise RuntimeError("command failed: %s\n%s" % (" ".join(cmd), r.stdout))
    return r.stdout


def _stale(target, sources):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def build_library(force=False, verbose=False):
    os.makedirs(OBJ_DIR, exist_ok=True)
    os.makedirs(LIB_DIR, exist_ok=True)
    headers = glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(INCLUDE_DIR, "*.h"))
    sources = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    jobs = []
    objs = []
    for src in sources:
        obj = os.path.join(OBJ_DIR, os.path.basename(src) + ".o")
        objs.append(obj)
        if force or _stale(obj, [src] + headers):
            jobs.append([NVCC] + NVCC_FLAGS + ["-c", src, "-o", obj])
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        for out in ex.map(_run, jobs):
            if verbose and out.strip():
                print(out)
    if force or jobs or _stale(LIB_PATH, objs):
        # -Bsymbolic: calls between the library's own exported functions bind
        # inside the library, even when another library exporting the same
        # C ABI (the CPU oracle) is loaded into the process.
        # cudart is linked statically: the library does not depend on which
        # libcudart.so another component of the process loaded first.
        _run([NVCC, "-shared", "-cudart", "static", "-Xlinker", "-Bsymbolic", "-o", LIB_PATH] + objs + ["-lgomp"])
    return LIB_PATH


def build_simulators(force=False):
    """Each simulator becomes an executable and a shared library exposing
    `int eqg_sim_main(int argc, char** argv)` for in-process use."""
    out = []
    entry = os.path.join(SIMS, "sim_entry.cpp")
    hdrs = glob.glob(os.path.join(INCLUDE_DIR, "equelle", "*.hpp")) + [os.path.join(INCLUDE_DIR, "eqg.h")]
    for src in sorted(glob.glob(os.path.join(SIMS, "*.cpp"))):
        if src == entry:
            continue
        name = os.path.splitext(os.path.basename(src))[0]
        exe = os.path.join(LIB_DIR, "sim_" + name)
        so = os.path.join(LIB_DIR, "libsim_" + name + ".so")
        common = [CXX, "-std=c++17", "-O2", "-I" + INCLUDE_DIR]
        rpath = "-Wl,-rpath,$ORIGIN"
        if force or _stale(exe, [src, LIB_PATH] + hdrs):
            _run(common + ["-o", exe, src, "-L" + LIB_DIR, "-leqg", rpath])
        if force or _stale(so, [src, entry, LIB_PATH] + hdrs):
            _run(common + ["-fPIC", "-shared", "-DEQUELLE_NO_MAIN", "-o", so, src, entry,
                           "-L" + LIB_DIR, "-leqg", rpath])
        out += [exe, so]
    return out


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--lib", action="store_true")
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", action="store_true")
    a = ap.parse_args(argv)
    print(build_library(force=a.force, verbose=a.v))
    if not a.lib:
        for p in build_simulators(force=a.force):
            print(p)


if __name__ == "__main__":
    sys.exit(main())

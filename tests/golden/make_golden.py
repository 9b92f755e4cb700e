"""Extract the golden vectors of the reference's CUDA-backend tests into JSON.

Reads, as text, the known-answer arrays that sintefmath/equelle's
backends/cuda/test/gridTest.cpp and valsOnGrid.cpp hold (plus their .param
and .mat inputs) and writes them to this directory:

    grid_4x3.json       gridTest.cpp:104-170 with gridTest.param
    vals_on_grid.json   valsOnGrid.cpp:100-390 with valsOnGrid.param and
                        valsOnGrid_*.mat

Run once in a container where the reference tree exists:

    python tests/golden/make_golden.py [/path/to/reference]

The JSON files are committed; nothing at test time reads the reference.
"""
import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ARRAY_RE = re.compile(r"\b(int|double)\s+(\w+)\s*\[\s*\d*\s*\]\s*=\s*\{([^}]*)\}\s*;")
# scalar constants some arrays are written with, e.g. `double x = 0.3;`
SCALAR_RE = re.compile(r"\bdouble\s+(\w+)\s*=\s*([-+0-9.eE]+)\s*;")


def arrays(path):
    text = open(path).read()
    consts = dict(SCALAR_RE.findall(text))
    out = {}
    for kind, name, body in ARRAY_RE.findall(text):
        vals = [v.strip() for v in body.replace("\n", " ").split(",") if v.strip()]
        if kind == "int":
            out[name] = [int(v) for v in vals]
        else:
            out[name] = [float(consts.get(v, v)) for v in vals]
    return out


def params(path):
    out = {}
    for line in open(path):
        line = line.split("#")[0].strip()
        if "=" in line:
            k, v = line.split("=", 1)
            out[k.strip()] = v.strip()
    return out


def mat(path):
    return [float(v) for v in open(path).read().split()]


def main(ref):
    test_dir = os.path.join(ref, "backends", "cuda", "test")
    grid = arrays(os.path.join(test_dir, "gridTest.cpp"))
    keep = ["boundary_faces", "int_faces", "bnd_cells", "int_cells", "first_cells",
            "second_cells", "first_bound_sol", "second_bound_sol", "inner_bnd_sol"]
    grid_json = {
        "source": "backends/cuda/test/gridTest.cpp:104-170",
        "params": params(os.path.join(test_dir, "gridTest.param")),
        "expected": {k: grid[k] for k in keep},
    }
    with open(os.path.join(HERE, "grid_4x3.json"), "w") as f:
        json.dump(grid_json, f, indent=1)

    vals = arrays(os.path.join(test_dir, "valsOnGrid.cpp"))
    prm = params(os.path.join(test_dir, "valsOnGrid.param"))
    inputs = {}
    for k, v in prm.items():
        if k.endswith("_filename"):
            inputs[v] = mat(os.path.join(test_dir, v))
    # faces_sol is built by a loop in the test: faces_sol[i] = i*10
    # (valsOnGrid.cpp:125-128); the literal array there is all ones.
    vals["faces_sol"] = [10.0 * i for i in range(31)]
    keep = ["a_full_sol", "b_full_sol", "faces_sol", "intCell_sol", "ext_intCell_allCell_sol",
            "intFace_sol", "ext_intFace_allFace_sol", "on_allCell_intCell_sol", "subset_ans",
            "subsetVals_sol", "extendSubsetCell_sol", "extendSubsetFace_sol", "boundVals_sol",
            "onSubsetCell_sol", "fromScalar_sol", "vol_sol", "area_sol", "area_bnd_sol",
            "a_big_sol", "a_big_grad_sol", "div_sol", "centrCells0_sol", "centrCells1_sol",
            "centr_bnd0_sol", "centr_bnd1_sol", "centr_intface0_sol", "centr_intface1_sol",
            "normalAll0_sol", "normalAll1_sol", "normals0_sol", "normals1_sol"]
    missing = [k for k in keep if k not in vals]
    if missing:
        raise SystemExit("arrays not found: %s" % missing)
    vals_json = {
        "source": "backends/cuda/test/valsOnGrid.cpp:100-390",
        "params": prm,
        "inputs": inputs,
        "expected": {k: vals[k] for k in keep},
        "note": ("normalAll*/normals* are the CUDA backend's area-scaled normals; the serial "
                 "backend returns unit normals (EquelleRuntimeCPU.cpp:306-308), so tests "
                 "scale them by 1/area."),
    }
    with open(os.path.join(HERE, "vals_on_grid.json"), "w") as f:
        json.dump(vals_json, f, indent=1)


if __name__ == "__main__":
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("EQUELLE_REFERENCE")
    if not ref:
        sys.exit("usage: make_golden.py <sintefmath/equelle checkout> (or set EQUELLE_REFERENCE)")
    main(ref)

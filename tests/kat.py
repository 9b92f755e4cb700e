"""Known-answer checks from the reference's own tests, runnable on any
library that exports include/eqg.h.

The expected arrays come from tests/golden/*.json, extracted from
sintefmath/equelle backends/cuda/test/gridTest.cpp and valsOnGrid.cpp by
tests/golden/make_golden.py.  Values are compared with the absolute
tolerance the reference test uses there: 1000 * DBL_EPSILON
(valsOnGrid.cpp:437).
"""
import json
import os

import numpy as np

from equelle_b200 import capi
from equelle_b200.runtime import Runtime

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
KAT_ATOL = 1000 * np.finfo(np.float64).eps


def load(name):
    with open(os.path.join(GOLDEN, name)) as f:
        return json.load(f)


def _grid_params(prm):
    return {k: prm[k] for k in ("grid_dim", "nx", "ny", "dx", "dy") if k in prm}


def close(got, want, what):
    got = np.asarray(got, dtype=np.float64)
    want = np.asarray(want, dtype=np.float64)
    assert got.shape == want.shape, "%s: size %s, expected %s" % (what, got.shape, want.shape)
    bad = np.abs(got - want) > KAT_ATOL
    assert not bad.any(), "%s: got %s expected %s" % (what, got[bad][:8], want[bad][:8])


def same(got, want, what):
    got = np.asarray(got)
    want = np.asarray(want)
    assert got.shape == want.shape and (got == want).all(), "%s: got %s expected %s" % (what, got, want)


def check_grid_4x3(lib):
    """gridTest.cpp:86-170 on the 4x3 unit grid."""
    g = load("grid_4x3.json")
    ex = g["expected"]
    er = Runtime(lib, _grid_params(g["params"]))
    assert len(er.allCells()) == 12
    assert len(er.allFaces()) == 31
    same(er.allCells().indices(), np.arange(12), "allCells")
    same(er.allFaces().indices(), np.arange(31), "allFaces")
    same(er.boundaryFaces().indices(), ex["boundary_faces"], "boundaryFaces")
    same(er.interiorFaces().indices(), ex["int_faces"], "interiorFaces")
    same(er.boundaryCells().indices(), ex["bnd_cells"], "boundaryCells")
    same(er.interiorCells().indices(), ex["int_cells"], "interiorCells")
    same(er.firstCell(er.allFaces()).indices(), ex["first_cells"], "firstCell(allFaces)")
    same(er.secondCell(er.allFaces()).indices(), ex["second_cells"], "secondCell(allFaces)")
    first_b = er.firstCell(er.boundaryFaces())
    second_b = er.secondCell(er.boundaryFaces())
    same(first_b.indices(), ex["first_bound_sol"], "firstCell(boundaryFaces)")
    same(second_b.indices(), ex["second_bound_sol"], "secondCell(boundaryFaces)")
    inner = er.trinaryIf(er.isEmpty(second_b), first_b, second_b)
    same(inner.indices(), ex["inner_bnd_sol"], "trinaryIf(isEmpty(second), first, second)")


def check_vals_on_grid(lib):
    """valsOnGrid.cpp:100-390 on the 4x3 grid with dx=0.5, dy=0.3."""
    g = load("vals_on_grid.json")
    prm, inp, ex = g["params"], g["inputs"], g["expected"]
    er = Runtime(lib, _grid_params(prm))

    def file_input(name):
        return er.collection(inp[prm[name + "_filename"]])

    a = file_input("a")
    close(a.value(), ex["a_full_sol"], "input a")
    b = er.constant(float(prm["b"]), len(er.allCells()))
    close(b.value(), ex["b_full_sol"], "input b")
    faces = file_input("faces")
    close(faces.value(), ex["faces_sol"], "input faces")

    int_cell = file_input("intCell")
    close(int_cell.value(), ex["intCell_sol"], "input intCell")
    close(er.operatorExtend(int_cell, er.interiorCells(), er.allCells()).value(),
          ex["ext_intCell_allCell_sol"], "Extend(intCell, interiorCells, allCells)")
    int_face = file_input("intFace")
    close(int_face.value(), ex["intFace_sol"], "input intFace")
    close(er.operatorExtend(int_face, er.interiorFaces(), er.allFaces()).value(),
          ex["ext_intFace_allFace_sol"], "Extend(intFace, interiorFaces, allFaces)")
    close(er.operatorOn(a, er.allCells(), er.interiorCells()).value(),
          ex["on_allCell_intCell_sol"], "On(a, allCells, interiorCells)")

    sub_idx = np.array(inp[prm["subset_filename"]], dtype=np.int32)
    subset_face = er.entity_set(capi.FACES, sub_idx)
    subset_cell = er.entity_set(capi.CELLS, sub_idx)
    for sub, sup in ((subset_face, er.interiorFaces()), (subset_cell, er.boundaryCells())):
        srt, inc = _check_subset(er, sub, sup)
        assert srt and inc, "inputDomainSubsetOf(subset)"
    same(subset_face.indices(), ex["subset_ans"], "subset faces")
    subset_vals = file_input("subsetVals")
    close(subset_vals.value(), ex["subsetVals_sol"], "input subsetVals")
    close(er.operatorExtend(subset_vals, subset_cell, er.boundaryCells()).value(),
          ex["extendSubsetCell_sol"], "Extend(subset cells -> boundaryCells)")
    close(er.operatorExtend(subset_vals, subset_face, er.interiorFaces()).value(),
          ex["extendSubsetFace_sol"], "Extend(subset faces -> interiorFaces)")
    bound_vals = file_input("boundCellVals")
    close(bound_vals.value(), ex["boundVals_sol"], "input boundCellVals")
    close(er.operatorOn(bound_vals, er.boundaryCells(), subset_cell).value(),
          ex["onSubsetCell_sol"], "On(boundaryCells -> subset cells)")
    close(er.operatorExtend(9.124, er.interiorCells()).value(), ex["fromScalar_sol"], "Extend(9.124)")

    close(er.norm(er.allCells()).value(), ex["vol_sol"], "Norm(AllCells)")
    close(er.norm(er.allFaces()).value(), ex["area_sol"], "Norm(AllFaces)")
    close(er.norm(er.boundaryFaces()).value(), ex["area_bnd_sol"], "Norm(BoundaryFaces)")

    a_big = er.trinaryIf(a > er.operatorExtend(50, er.allCells()), a * 2, a / 2)
    close(a_big.value(), ex["a_big_sol"], "trinaryIf(a > 50, a*2, a/2)")
    a_big_grad = er.gradient(a_big)
    close(a_big_grad.value(), ex["a_big_grad_sol"], "Gradient(a_big)")
    close(er.divergence(a_big_grad).value(), ex["div_sol"], "Divergence(a_big_grad)")

    cc = er.centroid(er.allCells())
    close(cc[0].value(), ex["centrCells0_sol"], "Centroid(AllCells)[0]")
    close(cc[1].value(), ex["centrCells1_sol"], "Centroid(AllCells)[1]")
    cb = er.centroid(er.boundaryCells())
    close(cb[0].value(), ex["centr_bnd0_sol"], "Centroid(boundaryCells)[0]")
    close(cb[1].value(), ex["centr_bnd1_sol"], "Centroid(boundaryCells)[1]")
    cf = er.centroid(er.interiorFaces())
    close(cf[0].value(), ex["centr_intface0_sol"], "Centroid(interiorFaces)[0]")
    close(cf[1].value(), ex["centr_intface1_sol"], "Centroid(interiorFaces)[1]")

    # The reference CUDA test expects area-scaled normals; the serial
    # backend (and this runtime) return unit normals, so scale by 1/area.
    for faces, n0, n1 in ((er.allFaces(), "normalAll0_sol", "normalAll1_sol"),
                          (er.interiorFaces(), "normals0_sol", "normals1_sol")):
        area = er.norm(faces).value()
        nrm = er.normal(faces)
        close(nrm[0].value(), np.asarray(ex[n0]) / area, "normal[0]")
        close(nrm[1].value(), np.asarray(ex[n1]) / area, "normal[1]")

    v2 = er.collection(np.arange(2, 42, 3, dtype=np.float64))
    close(er.sqrt(v2).value(), np.sqrt(np.arange(2, 42, 3, dtype=np.float64)), "sqrt(vec2)")


def _check_subset(er, sub, sup):
    import ctypes as C
    s, i = C.c_int(), C.c_int()
    er._ok(er.lib.eqg_set_check_subset(er.h, sub.h, sup.h, C.byref(s), C.byref(i)))
    return bool(s.value), bool(i.value)

"""Grids read from a file (grid_filename; the reference builds
Opm::GridManager(grid_filename), backends/serial/src/EquelleRuntimeCPU.cpp:
20-24).

CPU: the oracle reading a file that holds the Cartesian grid gives the same
topology, geometry and operator results, bit for bit, as the oracle's
built-in Cartesian grid; malformed files are rejected.
GPU: the device library against the oracle on non-Cartesian grids (jittered
quadrilaterals mixed with triangles in 2D, their extrusion into prism and
hexahedron layers in 3D): topology and geometry bit-exact, every AD op of
the op stream (Jacobian patterns bit-exact, values within 1e-12), and the
reference's own generated heat program (examples/app/out_heateq.cpp,
unchanged) within 1e-9 per cell.
"""
import os

import numpy as np
import pytest

import opstream
from equelle_b200 import cases, grids, programs, simrun
from equelle_b200.runtime import Runtime
from parity import assert_colls, assert_values

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_BUILD = os.path.join(ROOT, "oracle", "_ref")


def _topology(r):
    out = {}
    for name in ("allCells", "boundaryCells", "interiorCells", "allFaces", "boundaryFaces", "interiorFaces"):
        out[name] = getattr(r, name)().indices()
    for side in ("firstCell", "secondCell"):
        out[side] = getattr(r, side)(r.allFaces()).indices()
    dim = r.info.dimensions
    for s in ("allCells", "allFaces", "boundaryFaces"):
        for d in range(dim):
            out["centroid_%s_%d" % (s, d)] = r.centroid(getattr(r, s)())[d].value()
        out["norm_" + s] = r.norm(getattr(r, s)()).value()
    for d in range(dim):
        out["normal_%d" % d] = r.normal(r.allFaces())[d].value()
    return out


CART = [dict(grid_dim=2, nx=5, ny=4, dx=0.7, dy=1.3), dict(grid_dim=3, nx=4, ny=3, nz=3, dx=1.0, dy=2.0, dz=0.5)]


@pytest.mark.parametrize("grid", CART, ids=["2d", "3d"])
def test_oracle_cartesian_file_equals_builtin_grid(oracle_lib, tmp_path, grid):
    g = grids.cartesian(grid["nx"], grid["ny"], grid.get("nz") if grid["grid_dim"] == 3 else None,
                        grid["dx"], grid["dy"], grid.get("dz", 1.0))
    path = g.write(str(tmp_path / "cart.grid"))
    built = Runtime(oracle_lib, grid)
    filed = Runtime(oracle_lib, dict(grid_filename=path))
    assert filed.info.number_of_cells == built.info.number_of_cells
    assert filed.info.number_of_faces == built.info.number_of_faces
    tb, tf = _topology(built), _topology(filed)
    for k in tb:
        assert np.array_equal(tb[k], tf[k]), k
    ob, of = opstream.op_stream(built), opstream.op_stream(filed)
    for k in ob:
        assert_colls(of[k], ob[k], k, rtol=0.0)


def test_oracle_rejects_malformed_grid_files(oracle_lib, tmp_path):
    g = grids.mixed_2d(3, 2, seed=1)
    good = g.write(str(tmp_path / "good.grid"))
    Runtime(oracle_lib, dict(grid_filename=good))
    text = open(good).read()
    bad_cells = text.replace("face_cells ", "face_cells 99 ", 1)
    p = tmp_path / "bad.grid"
    p.write_text(bad_cells)
    with pytest.raises(RuntimeError):
        Runtime(oracle_lib, dict(grid_filename=str(p)))
    p.write_text(text.replace("eqg-grid 1", "eqg-grid 7", 1))
    with pytest.raises(RuntimeError):
        Runtime(oracle_lib, dict(grid_filename=str(p)))
    with pytest.raises(RuntimeError):
        Runtime(oracle_lib, dict(grid_filename=str(tmp_path / "missing.grid")))


def _unstructured(kind, tmp_path):
    if kind == "mixed2d":
        g = grids.mixed_2d(9, 7, seed=3)
    else:
        g = grids.extruded(grids.mixed_2d(5, 4, seed=4), 3, dz=0.4)
    return g, g.write(str(tmp_path / (kind + ".grid")))


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["mixed2d", "extruded3d"])
def test_unstructured_topology_and_ops_match_oracle(gpu_lib, oracle_lib, tmp_path, kind):
    g, path = _unstructured(kind, tmp_path)
    dev = Runtime(gpu_lib, dict(grid_filename=path))
    ora = Runtime(oracle_lib, dict(grid_filename=path))
    assert dev.info.nx == 0 and dev.info.number_of_cells == g.nc
    td, to = _topology(dev), _topology(ora)
    for k in to:
        assert np.array_equal(td[k], to[k]), k
    od, oo = opstream.op_stream(dev), opstream.op_stream(ora)
    for k in oo:
        assert_colls(od[k], oo[k], k)
    rd, ro = opstream.reductions(dev), opstream.reductions(ora)
    for k in ro:
        assert_values([rd[k]], [ro[k]], k)


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["mixed2d", "extruded3d"])
def test_reference_heat_program_on_unstructured_grid(tmp_path, kind):
    """examples/app/out_heateq.cpp, unchanged, 10 steps, Dirichlet values on
    every other boundary face: every u field within 1e-9 per cell."""
    g, path = _unstructured(kind, tmp_path)
    rng = np.random.default_rng(11)
    d = tmp_path / "in"
    d.mkdir()
    bfaces = g.boundary_faces()[::2]
    np.savetxt(d / "u0.txt", rng.uniform(0.5, 1.5, g.nc), fmt="%.17g")
    np.savetxt(d / "dir_faces.txt", bfaces, fmt="%d")
    np.savetxt(d / "dir_val.txt", np.full(len(bfaces), 0.5), fmt="%.17g")
    np.savetxt(d / "timesteps.txt", np.full(10, 0.5), fmt="%.17g")
    args = ["grid_filename=" + path, "k=0.3", "cv=1.0",
            "u_initial_from_file=true", "u_initial_filename=%s" % (d / "u0.txt"),
            "dir_boundary_filename=%s" % (d / "dir_faces.txt"),
            "dir_val_from_file=true", "dir_val_filename=%s" % (d / "dir_val.txt"),
            "timesteps_filename=%s" % (d / "timesteps.txt"),
            "abs_res_tol=1e-10", "linsolver_residual_tolerance=1e-12", "output_to_file=true"]
    fields = {}
    for side in ("device", "oracle"):
        out = tmp_path / side
        out.mkdir()
        lib = os.path.join(REF_BUILD, "libref_out_heateq_%s.so" % side)
        if not os.path.exists(lib):
            pytest.fail("%s is not built" % lib)
        rep = simrun.run("out_heateq", args + ["output_dir=%s/" % out], path=lib)
        assert rep.solves == 10
        fields[side] = [np.loadtxt(out / ("u-%05d.output" % k)) for k in range(11)]
    for k, (a, b) in enumerate(zip(fields["device"], fields["oracle"])):
        err = float(np.max(np.abs(a - b) / np.abs(b)))
        assert err <= 1e-9, "u after step %d: %g" % (k, err)
    # the run did something: heat left through the Dirichlet faces
    assert fields["oracle"][-1].mean() < fields["oracle"][0].mean()


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["mixed2d", "extruded3d"])
def test_two_phase_on_unstructured_grid(gpu_lib, oracle_lib, tmp_path, kind):
    """The fully implicit oil-water program (programs.two_phase, the Python
    twin of sims/twophase.cpp) on a non-Cartesian grid: injector in cell 0,
    producer and pressure anchor in the last cell, each passing its own pore
    volume per day, i.i.d. log-normal permeability; 3 steps of one day,
    block ILU(0) on the device against the oracle's natural ILU(0): Sw
    within 1e-8 per cell and p within 1e-8 of its largest magnitude after
    every step."""
    if kind == "mixed2d":
        g = grids.mixed_2d(10, 8, seed=5, dx=10.0, dy=10.0)
    else:
        g = grids.extruded(grids.mixed_2d(6, 5, seed=6, dx=10.0, dy=10.0), 3, dz=2.0)
    path = g.write(str(tmp_path / (kind + ".grid")))
    rng = np.random.default_rng(21)
    mD = 9.869233e-16
    n = g.nc
    inj, prod = 0, n - 1
    rate = 0.2 * g.cell_volumes[inj] / 86400.0
    case = dict(perm=np.exp(rng.normal(np.log(100 * mD), 0.5, n)), poro=np.full(n, 0.2), watervisc=1e-3,
                oilvisc=5e-3, source_cells=np.array([inj, prod], dtype=np.int32),
                source_values=np.array([rate, -rate]), sw_initial=np.full(n, 0.2), timesteps=[86400.0] * 3,
                corey=2.0, anchor_cells=np.array([prod], dtype=np.int32))
    params = dict(grid_filename=path, abs_res_tol=1e-11, linsolver_residual_tolerance=1e-12,
                  linsolver_max_iterations=5000)
    og = programs.two_phase(Runtime(gpu_lib, params), **case)
    oo = programs.two_phase(Runtime(oracle_lib, params), **case)
    assert len(og) == len(oo) == 3
    for step, ((pg, sg), (po, so)) in enumerate(zip(og, oo)):
        assert np.max(np.abs(sg - so) / np.abs(so)) <= 1e-8, "Sw step %d" % step
        assert np.max(np.abs(pg - po)) <= 1e-8 * np.max(np.abs(po)), "p step %d" % step
    assert np.max(oo[-1][1]) > 0.2 + 1e-3  # water has entered

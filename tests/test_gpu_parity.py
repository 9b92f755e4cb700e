"""Device library vs CPU oracle, through the C ABI (needs a GPU)."""
import numpy as np
import pytest

import kat
import opstream
from equelle_b200 import programs
from equelle_b200.runtime import Runtime
from parity import assert_colls, assert_values

pytestmark = pytest.mark.gpu

# the V-cycle's up-leg through A P on every level outside the fused cycle,
# and no fused levels (the defaults take it only above 40000 unknowns)
AP_EVERYWHERE = dict(linsolver_mg_ap_rows=0, linsolver_mg_fuse_rows=0)


def test_gpu_grid_4x3_golden(gpu_lib):
    kat.check_grid_4x3(gpu_lib)


def test_gpu_vals_on_grid_golden(gpu_lib):
    kat.check_vals_on_grid(gpu_lib)


@pytest.mark.parametrize("grid", opstream.GRIDS, ids=["2d", "3d"])
def test_op_stream_parity(gpu_lib, oracle_lib, grid):
    g = Runtime(gpu_lib, grid)
    o = Runtime(oracle_lib, grid)
    og = opstream.op_stream(g)
    oo = opstream.op_stream(o)
    for k in oo:
        assert_colls(og[k], oo[k], k)
    # a second pass reuses every cached pattern and must give the same numbers
    og2 = opstream.op_stream(g)
    for k in oo:
        assert_colls(og2[k], oo[k], k + " (cached)")
    assert g.stats()["pattern_cache_hits"] > 0


@pytest.mark.parametrize("grid", opstream.GRIDS, ids=["2d", "3d"])
def test_reductions_and_masks(gpu_lib, oracle_lib, grid):
    g = Runtime(gpu_lib, grid)
    o = Runtime(oracle_lib, grid)
    rg, ro = opstream.reductions(g), opstream.reductions(o)
    for k in ro:
        assert_values([rg[k]], [ro[k]], k)
    mg, mo = opstream.masks(g), opstream.masks(o)
    for k in mo:
        assert np.array_equal(mg[k], mo[k]), k


@pytest.mark.parametrize("grid", opstream.GRIDS, ids=["2d", "3d"])
def test_topology_parity(gpu_lib, oracle_lib, grid):
    g = Runtime(gpu_lib, grid)
    o = Runtime(oracle_lib, grid)
    for name in ("allCells", "boundaryCells", "interiorCells", "allFaces", "boundaryFaces", "interiorFaces"):
        assert np.array_equal(getattr(g, name)().indices(), getattr(o, name)().indices()), name
    for side in ("firstCell", "secondCell"):
        assert np.array_equal(getattr(g, side)(g.allFaces()).indices(), getattr(o, side)(o.allFaces()).indices())
    for s in ("allCells", "allFaces", "boundaryFaces"):
        for d in range(grid["grid_dim"]):
            assert np.array_equal(g.centroid(getattr(g, s)())[d].value(), o.centroid(getattr(o, s)())[d].value())
        assert np.array_equal(g.norm(getattr(g, s)()).value(), o.norm(getattr(o, s)()).value())
    for d in range(grid["grid_dim"]):
        assert np.array_equal(g.normal(g.allFaces())[d].value(), o.normal(o.allFaces())[d].value())


@pytest.mark.parametrize("ordering,precond,extra", [("multicolor", "multigrid", {}), ("multicolor", "ilu0", {}),
                                                    ("natural", "ilu0", {}), ("natural", "multigrid", {}),
                                                    ("natural", "multigrid", AP_EVERYWHERE),
                                                    ("multicolor", "multigrid", AP_EVERYWHERE)],
                         ids=["mc-mg", "mc-ilu0", "nat-ilu0", "nat-mg", "nat-mg-ap", "mc-mg-ap"])
def test_heat_64x64_parity(gpu_lib, oracle_lib, ordering, precond, extra):
    """Implicit heat equation, 64x64, 20 steps: fields within 1e-9 relative
    (scalar unknowns; with the A P up-leg on every launch-path level too)."""
    grid, case = programs.heat_case(64, 64, steps=20)
    params = dict(grid, abs_res_tol=1e-10, linsolver_residual_tolerance=1e-12)
    og = programs.heat_equation(Runtime(gpu_lib, dict(params, linsolver_ordering=ordering,
                                                      linsolver_preconditioner=precond, **extra)), 0.3, 1.0, **case)
    oo = programs.heat_equation(Runtime(oracle_lib, params), 0.3, 1.0, **case)
    for step, (a, b) in enumerate(zip(og, oo)):
        assert np.max(np.abs(a - b) / np.abs(b)) <= 1e-9, "step %d" % step


@pytest.mark.parametrize("shape,precision,precond", [((16, 16, None), "double", "multigrid"),
                                                     ((16, 16, None), "mixed", "multigrid"),
                                                     ((16, 16, None), "refine", "multigrid"),
                                                     ((8, 8, 4), "double", "multigrid"),
                                                     ((8, 8, 4), "mixed", "multigrid"),
                                                     ((16, 16, 8), "double", "multigrid"),
                                                     ((16, 16, 8), "mixed", "multigrid"),
                                                     ((16, 16, 8), "double", "ilu0"),
                                                     ((16, 16, 8), "mixed", "ilu0"),
                                                     ((16, 16, 8), "refine", "ilu0")])
def test_two_phase_parity(gpu_lib, oracle_lib, shape, precision, precond):
    """Fully implicit two-phase flow: saturation within 1e-8 relative of the
    FP64 oracle after every step, in plain FP64, with the FP32 preconditioner
    (mixed) and with FP32 BiCGStab inside FP64 refinement (refine)."""
    grid, case = programs.two_phase_case(*shape, steps=3)
    params = dict(grid, abs_res_tol=1e-11, linsolver_residual_tolerance=1e-12, linsolver_max_iterations=5000)
    eg = Runtime(gpu_lib, dict(params, linsolver_precision=precision, linsolver_preconditioner=precond))
    og = programs.two_phase(eg, **case)
    oo = programs.two_phase(Runtime(oracle_lib, params), **case)
    for step, ((pg, sg), (po, so)) in enumerate(zip(og, oo)):
        assert np.max(np.abs(sg - so) / np.abs(so)) <= 1e-8, "Sw step %d" % step
        assert np.max(np.abs(pg - po)) <= 1e-8 * np.max(np.abs(po)), "p step %d" % step
    st = eg.stats()
    if precision == "refine":
        assert st["refinement_sweeps"] >= st["linear_solves"] > 0



def reaction_diffusion3(er, fields, rates, timesteps):
    """Three species on all cells, implicit in time: diffusion with no-flow
    boundaries and a nonlinear exchange a <-> b <-> c, solved together with
    newtonSolveSystem (3 x 3 blocks per cell).  Returns (a, b, c) per step."""
    ifaces = er.interiorFaces()
    first = er.firstCell(ifaces)
    second = er.secondCell(ifaces)
    trans = er.norm(ifaces) / er.norm(er.centroid(first) - er.centroid(second))
    vol = er.norm(er.allCells())
    k1, k2, d = rates

    def div_flux(x, diff):
        return er.divergence(er.operatorExtend(-(diff * trans) * er.gradient(x), er.interiorFaces(), er.allFaces()))

    olds = [er.collection(f) for f in fields]
    out = []
    for dt in timesteps:
        a0, b0, c0 = olds

        def ra(a, b, c):
            return (a - a0) + (dt / vol) * div_flux(a, d[0]) + dt * (k1 * a * b - k2 * c)

        def rb(a, b, c):
            return (b - b0) + (dt / vol) * div_flux(b, d[1]) + dt * (k1 * a * b - k2 * c)

        def rc(a, b, c):
            return (c - c0) + (dt / vol) * div_flux(c, d[2]) - dt * (k1 * a * b - k2 * c)

        olds = list(er.newtonSolveSystem([ra, rb, rc], olds))
        out.append(tuple(x.value() for x in olds))
    return out


@pytest.mark.parametrize("shape,precond", [((12, 10, 6), "multigrid"), ((12, 10, 6), "ilu0"), ((40, 30, None), "multigrid"),
                                           ((12, 10, 6), "multigrid-ap")])
def test_three_species_blocks_parity(gpu_lib, oracle_lib, shape, precond):
    """A 3-unknowns-per-cell system (3 x 3 block ILU(0)): every species
    within 1e-9 relative of the FP64 oracle after every step."""
    nx, ny, nz = shape
    grid = dict(grid_dim=2 if nz is None else 3, nx=nx, ny=ny, nz=nz or 1, dx=1.0, dy=1.0, dz=1.0)
    n = nx * ny * (nz or 1)
    rng = np.random.RandomState(3)
    fields = [1.0 + rng.rand(n), 0.5 + rng.rand(n), 0.1 * rng.rand(n)]
    args = (fields, (2.0, 0.5, (1.0, 0.3, 0.05)), [0.1, 0.2, 0.2])
    params = dict(grid, abs_res_tol=1e-12, linsolver_residual_tolerance=1e-12, linsolver_max_iterations=5000)
    extra = AP_EVERYWHERE if precond.endswith("-ap") else {}
    og = reaction_diffusion3(Runtime(gpu_lib, dict(params, linsolver_preconditioner=precond.split("-")[0], **extra)),
                             *args)
    oo = reaction_diffusion3(Runtime(oracle_lib, params), *args)
    for step, (g, o) in enumerate(zip(og, oo)):
        for k in range(3):
            assert np.max(np.abs(g[k] - o[k]) / np.abs(o[k])) <= 1e-9, "species %d step %d" % (k, step)


@pytest.mark.parametrize("block,ordering", [(0, "multicolor"), (0, "natural"), (1, "multicolor")])
def test_two_phase_block_layouts(gpu_lib, oracle_lib, block, ordering):
    """The same two-phase case with 2 x 2 blocks per cell and with 1 x 1
    blocks (scalar ILU(0), multicolour or natural order): saturation within
    1e-8 relative of the oracle."""
    grid, case = programs.two_phase_case(8, 8, 4, steps=2)
    params = dict(grid, abs_res_tol=1e-11, linsolver_residual_tolerance=1e-12, linsolver_max_iterations=5000)
    eg = Runtime(gpu_lib, dict(params, linsolver_block=block, linsolver_ordering=ordering))
    og = programs.two_phase(eg, **case)
    oo = programs.two_phase(Runtime(oracle_lib, params), **case)
    for step, ((pg, sg), (po, so)) in enumerate(zip(og, oo)):
        assert np.max(np.abs(sg - so) / np.abs(so)) <= 1e-8, "Sw step %d" % step


@pytest.mark.parametrize("precision", ["double", "mixed"])
@pytest.mark.parametrize("shape", [(16, 16, 8), (64, 64, None)])
def test_coarse_correction_through_ap(gpu_lib, oracle_lib, shape, precision):
    """The V-cycle's up-leg through A P (t -= alpha A P zc on the residual of
    the down-leg, z += alpha P zc; levels above linsolver_mg_ap_rows unknowns,
    every launch-path level here): pressure and saturation within 1e-8 of
    the oracle and of the up-leg that prolongs and recomputes r - A z."""
    grid, case = programs.two_phase_case(*shape, steps=3)
    params = dict(grid, abs_res_tol=1e-11, linsolver_residual_tolerance=1e-12, linsolver_max_iterations=5000)
    dev = dict(params, linsolver_precision=precision, linsolver_mg_fuse_rows=0)
    eg = Runtime(gpu_lib, dict(dev, linsolver_mg_ap_rows=0))
    with_ap = programs.two_phase(eg, **case)
    plain = programs.two_phase(Runtime(gpu_lib, dict(dev, linsolver_mg_ap_rows=10**9)), **case)
    oo = programs.two_phase(Runtime(oracle_lib, params), **case)
    for step, ((pa, sa), (pb, sb), (po, so)) in enumerate(zip(with_ap, plain, oo)):
        for s_ in (sa, sb):
            assert np.max(np.abs(s_ - so) / np.abs(so)) <= 1e-8, "Sw step %d" % step
        for p_ in (pa, pb):
            assert np.max(np.abs(p_ - po)) <= 1e-8 * np.max(np.abs(po)), "p step %d" % step
    assert eg.stats()["krylov_iterations"] > 0


@pytest.mark.parametrize("precision", ["double", "mixed"])
@pytest.mark.parametrize("shape", [(16, 16, 8), (64, 64, None)])
def test_fused_coarse_cycle_identical(gpu_lib, shape, precision):
    """The V-cycle's coarse levels fused into one cluster kernel compute every
    element with the same operations as the launch-per-step cycle: pressure
    and saturation are bit-identical with no levels fused, some fused, all
    fused, for cluster sizes 1, 8 and 16, and with the coarsest fused levels
    in block 0's shared memory or not (linsolver_mg_local)."""
    grid, case = programs.two_phase_case(*shape, steps=2)
    params = dict(grid, abs_res_tol=1e-10, linsolver_residual_tolerance=1e-10, linsolver_max_iterations=5000,
                  linsolver_precision=precision)
    runs = {}
    for fuse, cluster, local in [(0, 16, 1), (600, 16, 1), (600, 16, 0), (40000, 1, 1), (40000, 8, 1),
                                 (40000, 16, 1), (40000, 16, 0)]:
        eg = Runtime(gpu_lib, dict(params, linsolver_mg_fuse_rows=fuse, linsolver_mg_cluster=cluster,
                                   linsolver_mg_local=local))
        runs[(fuse, cluster, local)] = (programs.two_phase(eg, **case), eg.stats())
    base, st0 = runs[(0, 16, 1)]
    for key, (out, st) in runs.items():
        assert st["krylov_iterations"] == st0["krylov_iterations"], key
        for (pa, sa), (pb, sb) in zip(out, base):
            assert np.array_equal(pa, pb) and np.array_equal(sa, sb), key


@pytest.mark.parametrize("grid", opstream.GRIDS, ids=["2d", "3d"])
def test_assembly_fast_paths_match_generic_kernels(gpu_lib, grid):
    """The Cartesian stencil kernels (gradient, divergence values), the
    position plans of operator products, the shared values of span
    supersets, the concatenation of row-disjoint sums and the row rules
    deferred into their readers give the same values and Jacobians, bit for
    bit, as the generic kernels they replace."""
    fast = opstream.op_stream(Runtime(gpu_lib, grid))
    generic = opstream.op_stream(Runtime(gpu_lib, dict(grid, stencil_ops=0, spgemm_plan=0, span_share=0,
                                                      jac_concat=0, jac_defer=0)))
    for k in generic:
        assert_colls(fast[k], generic[k], k, rtol=0.0)

"""One op stream that touches every AD rule of the C ABI, run identically
on the device library and on the oracle by the parity tests."""
import numpy as np

from equelle_b200 import capi


def op_stream(er, seed=0):
    rng = np.random.default_rng(seed)
    n = er.info.number_of_cells
    nif = er.info.number_of_interior_faces
    u0 = er.collection(rng.uniform(0.5, 1.5, n))
    u = er.variable(u0)
    w = er.collection(rng.uniform(0.5, 2.0, n))
    out = {}
    out["add"] = u + w
    out["add_ad"] = u + u * w
    out["sub"] = w - u
    out["sub_ad"] = u * u - u
    out["mul"] = u * u
    out["mul_c"] = w * u
    out["div"] = w / u
    out["div2"] = u / w
    out["div_ad"] = (u * u) / (u + w)
    out["smul"] = 2.5 * u
    out["smul_r"] = u * 2.5
    out["sdiv"] = u / 3.0
    out["rdiv"] = 3.0 / u
    out["sadd"] = u + 1.0
    out["rsub"] = 1.0 - u
    out["neg"] = -u
    out["sqrt"] = er.sqrt(u * w)
    out["abs"] = er.norm(u - 1.0)
    g = er.gradient(u * u)
    out["grad"] = g
    out["ngrad"] = er.negGradient(u)
    t = er.collection(rng.uniform(0.1, 1.0, nif))
    out["div_int"] = er.divergence(g * t)
    ff = er.operatorExtend(g * t, er.interiorFaces(), er.allFaces())
    out["ext"] = ff
    bf = er.boundaryFaces()
    bcells = er.trinaryIf(er.isEmpty(er.firstCell(bf)), er.secondCell(bf), er.firstCell(bf))
    bflux = er.operatorOn(u, er.allCells(), bcells) * 0.5
    full = ff + er.operatorExtend(bflux, bf, er.allFaces())
    out["div_full"] = er.divergence(full)
    out["on_first"] = er.operatorOn(u, er.allCells(), er.firstCell(er.interiorFaces()))
    out["on_int"] = er.operatorOn(u * w, er.allCells(), er.interiorCells())
    ic = er.operatorOn(u, er.allCells(), er.interiorCells())
    out["ext_int"] = er.operatorExtend(ic, er.interiorCells(), er.allCells())
    out["select_mixed"] = er.trinaryIf(u > 1.0, u * u, w)
    out["select_ad"] = er.trinaryIf(u > 1.0, u, er.sqrt(u))
    out["select_rev"] = er.trinaryIf(u <= 1.0, w, -u)
    # two unknown blocks, as newtonSolveSystem stacks them
    v = er.variable(er.collection(rng.uniform(0.5, 1.5, 2 * n)))
    p = er.spanSubset(v, 0, n)
    s = er.spanSubset(v, n, n)
    r = er.spanSuperset(er.divergence(er.gradient(p) * er.operatorOn(s, er.allCells(), er.firstCell(er.interiorFaces()))), 0, 2 * n)
    r = r + er.spanSuperset(s * s - p, n, 2 * n)
    out["system"] = r
    return out


def reductions(er, seed=0):
    rng = np.random.default_rng(seed)
    x = er.collection(rng.uniform(-1.0, 1.0, er.info.number_of_cells))
    y = er.collection(rng.uniform(0.9, 1.1, er.info.number_of_cells))
    return {"min": er.minReduce(x), "max": er.maxReduce(x), "sum": er.sumReduce(x),
            "prod": er.prodReduce(y), "twoNorm": er.twoNorm(x)}


def masks(er, seed=0):
    rng = np.random.default_rng(seed)
    x = er.collection(rng.uniform(-1.0, 1.0, er.info.number_of_cells))
    m1, m2 = x > 0.0, x < 0.5
    return {"and": (m1 & m2).values(), "or": (m1 | m2).values(), "not": (~m1).values(),
            "eq": x.eq(x).values(), "ne": x.ne(0.25).values()}


GRIDS = [
    dict(grid_dim=2, nx=5, ny=4, dx=0.7, dy=1.3),
    dict(grid_dim=3, nx=4, ny=3, nz=3, dx=1.0, dy=2.0, dz=0.5),
]

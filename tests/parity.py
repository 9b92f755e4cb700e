"""Helpers comparing the device library with the CPU oracle.

Tolerances (per-op contract: FP64 values within 1e-12 relative; sparsity
patterns bit-exact):
  - values: |got - want| <= 1e-12 * max(|want|, 1e-3 * max|want|), i.e.
    relative 1e-12, with entries a thousand times smaller than the largest
    compared at 1e-15 of the largest (sums that cancel);
  - Jacobian patterns: rowptr and colind identical;
  - Jacobian values: the same rule as values.
"""
import numpy as np

RTOL = 1e-12


def assert_values(got, want, what, rtol=RTOL):
    got = np.asarray(got, dtype=np.float64)
    want = np.asarray(want, dtype=np.float64)
    assert got.shape == want.shape, "%s: shape %s vs %s" % (what, got.shape, want.shape)
    if want.size == 0:
        return
    scale = np.maximum(np.abs(want), 1e-3 * np.max(np.abs(want)))
    bad = ~(np.abs(got - want) <= rtol * scale)
    if bad.any():
        i = np.flatnonzero(bad)[:5]
        raise AssertionError("%s: %d mismatches, e.g. idx %s got %s want %s" % (what, bad.sum(), i, got[i], want[i]))


def assert_colls(g, o, what, rtol=RTOL):
    """Compare two CollOfScalar (device, oracle): values and Jacobians."""
    assert_values(g.value(), o.value(), what + " value", rtol)
    jg, jo = g.jacobian(), o.jacobian()
    assert (jg is None) == (jo is None), "%s: Jacobian presence differs" % what
    if jg is None:
        return
    rg, cg, pg, colg, vg = jg
    ro, co, po, colo, vo = jo
    assert (rg, cg) == (ro, co), "%s: Jacobian shape %s vs %s" % (what, (rg, cg), (ro, co))
    assert np.array_equal(pg, po), "%s: Jacobian rowptr differs" % what
    assert np.array_equal(colg, colo), "%s: Jacobian colind differs" % what
    assert_values(vg, vo, what + " Jacobian", rtol)

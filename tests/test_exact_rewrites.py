"""The exact rewrites the fused shallow-water kernels make (fused.cu), checked
in IEEE double arithmetic on the host (numpy float64, round to nearest):

- sqrt(fl(x * x)) == |x| whenever x * x is a normal double;
- x / 2**k == x * 2**-k for every x (both round the same real number);
- a * t + b * f with (t, f) = (1, 0) or (0, 1) equals the chosen operand
  plus the other one times 0, bit for bit, signed zeros, infinities and NaN
  included (NaN compared as NaN).

The device kernels use round-to-nearest intrinsics for these operations, so
the same identities hold there; the GPU tests compare the fused results
with the one-kernel-per-operation path bit for bit."""
import numpy as np

RNG = np.random.default_rng(20261204)


def _bits(x):
    return np.asarray(x, dtype=np.float64).view(np.uint64)


def _sample(n):
    # log-uniform magnitudes over the range where x * x is normal, both
    # signs, plus values next to powers of two and the range's edges
    e = RNG.uniform(-510.9, 510.9, n)
    x = np.sign(RNG.uniform(-1, 1, n)) * np.exp2(e)
    p = np.exp2(np.arange(-510, 511, dtype=np.float64))
    edges = np.concatenate([p, np.nextafter(p, 0), np.nextafter(p, np.inf),
                            [2.0 ** -511, 2.0 ** 511, np.nextafter(2.0 ** 511, 0)]])
    return np.concatenate([x, edges, -edges])


def test_sqrt_of_square_is_abs_in_the_normal_range():
    x = _sample(2_000_000)
    with np.errstate(all="raise"):
        y = np.sqrt(x * x)
    assert np.array_equal(_bits(y), _bits(np.abs(x)))


def test_sqrt_of_square_differs_below_the_range():
    # outside it the kernels perform both operations: the identity fails
    x = np.array([1e-170, 3e-200, 1e-320])
    with np.errstate(under="ignore"):
        assert not np.array_equal(np.sqrt(x * x), np.abs(x))


def test_division_by_a_power_of_two_is_the_exact_reciprocal_product():
    x = np.concatenate([_sample(500_000), [0.0, -0.0, np.inf, -np.inf, 5e-324, -5e-324]])
    for k in (-3, -1, 1, 2, 10):
        d = 2.0 ** k
        with np.errstate(all="ignore"):
            assert np.array_equal(_bits(x / d), _bits(x * (1.0 / d)))


def test_one_product_selection():
    base = np.concatenate([RNG.standard_normal(200_000) * 1e3, [0.0, -0.0, np.inf, -np.inf, np.nan, 1e308, -1e-310]])
    a = RNG.permutation(base)
    b = RNG.permutation(base)
    for m in (True, False):
        t, f = (1.0, 0.0) if m else (0.0, 1.0)
        with np.errstate(all="ignore"):
            want = a * t + b * f
            got = (a if m else b) + (b if m else a) * 0.0
        nan = np.isnan(want)
        assert np.array_equal(np.isnan(got), nan)
        assert np.array_equal(_bits(got[~nan]), _bits(want[~nan]))

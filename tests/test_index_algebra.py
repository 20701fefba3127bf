"""Exactness of the rewritten steps of the packed resampling index (CPU).

The packed two-sample index takes the fractional part of y = ph / 2 pi as
fl(y - floor(y)) where the reference (src/science.cpp:20-35) takes
y - trunc(y) and adds 1 when that is negative.  Both are IEEE float32
operations here (numpy rounds every float32 operation to nearest), so the
identity is checked bit for bit over random, negative, integral, near-integral,
tiny and large arguments.  The other rewrites (a - b as a + (-b), -(x y) as
(-x) y) are exact by definition of IEEE negation.
"""
import numpy as np

F = np.float32


def reference_frac(y):
    a = (y - np.trunc(y)).astype(F)  # exact in IEEE arithmetic
    return np.where(a < 0, (a + F(1)).astype(F), a)


def floor_frac(y):
    return (y + (-np.floor(y)).astype(F)).astype(F)


def check(y):
    y = np.asarray(y, F)
    r, f = reference_frac(y), floor_frac(y)
    assert np.array_equal(r.view(np.uint32), f.view(np.uint32)), y[r.view(np.uint32) != f.view(np.uint32)][:5]


def test_random_phases_both_signs():
    rng = np.random.default_rng(7)
    for scale in (1e-3, 1.0, 3.0, 50.0, 1e4):
        check(rng.uniform(-scale, scale, 1_000_000).astype(F))


def test_integers_and_neighbours():
    ints = np.arange(-5000, 5001, dtype=F)
    check(ints)
    check(np.nextafter(ints, F(np.inf)))
    check(np.nextafter(ints, F(-np.inf)))


def test_tiny_and_large_arguments():
    tiny = np.array([0.0, -0.0, 1e-45, -1e-45, 1e-38, -1e-38, 1e-10, -1e-10, 5.96e-8, -5.96e-8], F)
    check(tiny)
    big = np.array([2.0 ** 22 + 0.5, -(2.0 ** 22 + 0.5), 2.0 ** 23, -(2.0 ** 23), 2.0 ** 24, -(2.0 ** 24),
                    3.0e7, -3.0e7], F)
    check(big)


def test_every_float_in_windows_below_zero():
    # the negative branch of the reference, exhaustively over two windows of
    # 2^22 consecutive float32 values: the smallest negative subnormals and
    # the values from -1 down to -1.5
    for start in (0x80000001, 0xBF800000):
        bits = np.arange(np.uint32(start), np.uint32(start) + np.uint32(1 << 22), dtype=np.uint32)
        check(bits.view(F))

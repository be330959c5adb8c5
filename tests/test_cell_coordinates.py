"""The cell coordinate without a division (floor_quot in csrc/ks_kernels.cu).

The reference's cell coordinate is floor(x / cell) of the correctly rounded
quotient (src/core/collision.cpp:393-395). The key builder multiplies by the
correctly rounded 1/cell instead and divides only when that product lies within
2^-50 |y| of an integer. The same IEEE double operations, in numpy, must give
the quotient's floor for every input: here on random coordinates and on
coordinates a few units in the last place from cell boundaries, where the
product and the quotient straddle an integer.
"""
import numpy as np


def floor_quot(x, c):
    inv = 1.0 / c
    y = x * inv
    f = np.floor(y)
    tol = np.abs(y) * 2.0 ** -50 + 2.0 ** -1000
    fast = ((y - f) > tol) & (((f + 1.0) - y) > tol)
    exact = np.floor(x / c)
    return np.where(fast, f, exact), fast


def check(x, c):
    got, fast = floor_quot(x, c)
    want = np.floor(x / c)
    assert np.array_equal(got, want), (x[got != want][:5], c[got != want][:5] if np.ndim(c) else c)
    return fast


def test_random_coordinates_and_cell_edges():
    rng = np.random.default_rng(20260801)
    n = 2_000_000
    c = np.exp(rng.uniform(np.log(1.0), np.log(5000.0), n))  # cell edges of 1 km and up
    x = rng.uniform(-60000.0, 60000.0, n)                     # out past GEO
    fast = check(x, c)
    assert fast.mean() > 0.999  # the exact division is the rare path


def test_coordinates_next_to_cell_boundaries():
    rng = np.random.default_rng(7)
    n = 200_000
    c = np.exp(rng.uniform(np.log(1.0), np.log(5000.0), n))
    k = rng.integers(-400, 400, n).astype(np.float64)
    base = k * c
    for ulps in range(-8, 9):
        x = base.copy()
        step = np.inf if ulps > 0 else -np.inf
        for _ in range(abs(ulps)):
            x = np.nextafter(x, step)
        check(x, c)
    # Quotients that round to the integer itself from either side.
    check(np.nextafter(base, np.inf), c)
    check(np.nextafter(base, -np.inf), c)


def test_tiny_and_zero_coordinates():
    c = np.full(6, 213.7)
    x = np.array([0.0, -0.0, 1e-300, -1e-300, 5e-324, -5e-324])
    check(x, c)

"""The pair kernel's column box test (boxes_apart in csrc/ks_kernels.cu).

A column is skipped when the distance d between its record and the row tile's
box exceeds gate + dt w, w the largest relative speed. The kernel compares d^2
and takes one approximate square root for w, with factors chosen so that the
test is at least as strict as the form with two correctly rounded roots:
    d (1 - 1e-5) - dt w (1 + 1e-5) > gate.
Here both forms run in FP32 (numpy), the approximate root at its worst (2^-21
below the correctly rounded one), on random cases and on cases at the
decision boundary: whenever the kernel's form skips a column, the reference
form does too.
"""
import numpy as np

f32 = np.float32


def fma(a, b, c):
    return (a.astype(np.float64) * b.astype(np.float64) + c.astype(np.float64)).astype(f32)


def reference_form(d2, w2, dt, gate):
    return np.sqrt(d2) * f32(1.0 - 1e-5) - dt * np.sqrt(w2) * f32(1.0 + 1e-5) > gate


def kernel_form(d2, w2, dt, gate):
    w = (np.sqrt(w2) * f32(1.0 - 2.0 ** -21)).astype(f32)  # the approximate root, low by its bound
    reach = fma(dt, (w * f32(1.0 + 1e-4)).astype(f32), gate)
    return d2 * f32(1.0 - 4e-5) > reach * reach * f32(1.0 + 1e-5)


def test_kernel_form_implies_the_reference_form():
    rng = np.random.default_rng(11)
    n = 2_000_000
    dt = np.full(n, 10.0, f32)
    gate = rng.uniform(5.0, 6.0, n).astype(f32)
    w = np.exp(rng.uniform(np.log(1e-4), np.log(30.0), n)).astype(f32)  # km/s
    # Distances spread around the decision boundary gate + dt w.
    d = ((gate + dt * w) * rng.uniform(0.999, 1.001, n)).astype(f32)
    d2, w2 = (d * d).astype(f32), (w * w).astype(f32)
    k = kernel_form(d2, w2, dt, gate)
    r = reference_form(d2, w2, dt, gate)
    assert not np.any(k & ~r)
    # The kernel's form stays useful: it skips almost every column the
    # reference form skips away from the boundary.
    far = d > (gate + dt * w) * f32(1.0002)
    assert k[far].mean() > 0.999


def test_random_boxes():
    rng = np.random.default_rng(12)
    n = 1_000_000
    dt = np.full(n, 10.0, f32)
    gate = np.full(n, 5.002, f32)
    d2 = rng.uniform(0.0, 4e4, n).astype(f32)
    w2 = rng.uniform(0.0, 400.0, n).astype(f32)
    assert not np.any(kernel_form(d2, w2, dt, gate) & ~reference_form(d2, w2, dt, gate))

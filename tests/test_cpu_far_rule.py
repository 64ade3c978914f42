"""Error model of the far-pair rule (no GPU): the device integrates far
regular pairs of the periodic domain (element centre at least 5 circumradii
R from the nearest lattice image of the node, k 2R <= 2) with an 8 x 8 rule
instead of the reference's 12 x 12 per quad or triangle part.  Here the
integrand exp(ikr)/r and its gradient, times an interpolation function, is
integrated over a curved quad and a flat triangle with both rules and with a
converged 40-point rule, for targets at 5 R in every direction: the 8 x 8
rule matches the converged integral (and so the reference's 12 x 12, itself
converged there) to 1e-13 of the entry."""
import numpy as np

K = 2 * np.pi
SQ3 = np.sqrt(3.0)


def quad_integrals(n, tgt, h, curv):
    x, w = np.polynomial.legendre.leggauss(n)
    Z, E = np.meshgrid(x, x, indexing="ij")
    W = np.outer(w, w)
    X, Y, Zc = h * Z, h * E, curv * h * (Z ** 2 + E ** 2)
    R = np.sqrt((X - tgt[0]) ** 2 + (Y - tgt[1]) ** 2 + (Zc - tgt[2]) ** 2)
    g = np.exp(1j * K * R) / R
    N = 0.25 * (1 - Z) * (1 - E)
    return np.array([np.sum(W * g * N), np.sum(W * g * N * (X - tgt[0]) / R ** 2)])


def tri_parts(n, tgt, R):
    """The reference's rule: 3 quadrilateral parts of the triangle, n x n each."""
    x, w = np.polynomial.legendre.leggauss(n)
    A, B = np.meshgrid(x, x, indexing="ij")
    W = np.outer(w, w) * (1 + 0.25 * A + 0.25 * B) / 24
    out = np.zeros(2, complex)
    for part in range(3):
        ab = A * B
        if part == 0:
            z, e = 0.125 * (3 + 2 * A + 2 * B + ab), 0.125 * SQ3 * (-A + B)
        elif part == 1:
            z, e = 0.0625 * (-3 + A - 5 * B - ab), 0.0625 * SQ3 * (3 + 3 * A + B + ab)
        else:
            z, e = 0.0625 * (-3 - 5 * A + B - ab), 0.0625 * SQ3 * (-3 - A - 3 * B - ab)
        out += _tri_terms(z, e, W, tgt, R)
    return out


def tri_collapsed(n, tgt, R):
    """The device's far rule: collapsed Gauss over the whole triangle,
    (z, e) = (1 - 3u/2, sqrt3/2 u (1 - 2v)), weight u w_u w_v."""
    x, w = np.polynomial.legendre.leggauss(n)
    u, v = 0.5 * (x + 1), 0.5 * (x + 1)
    U, V = np.meshgrid(u, v, indexing="ij")
    W = np.outer(0.5 * w, 0.5 * w) * U
    return _tri_terms(1 - 1.5 * U, 0.5 * SQ3 * U * (1 - 2 * V), W, tgt, R)


def _tri_terms(z, e, W, tgt, R):
    X, Y = R * z, R * e
    r = np.sqrt((X - tgt[0]) ** 2 + (Y - tgt[1]) ** 2 + tgt[2] ** 2)
    g = np.exp(1j * K * r) / r
    N = 1 / 3 + 2 / 3 * z
    return np.array([np.sum(W * g * N), np.sum(W * g * N * (X - tgt[0]) / r ** 2)])


def _targets(d):
    for ang in np.linspace(0, 2 * np.pi, 9):
        for elev in (0.0, 0.3, 1.0):
            yield (d * np.cos(ang) * np.cos(elev), d * np.sin(ang) * np.cos(elev), d * np.sin(elev) + 1e-3 * d)


def test_quad_far_rule_error():
    worst = 0.0
    for h in (0.039, 0.08, 0.12):          # half-size; k 2R = 2 sqrt2 h k up to 2.1
        Rs = h * np.sqrt(2)
        for tgt in _targets(5.0 * Rs):
            ref = quad_integrals(40, tgt, h, 0.2)
            worst = max(worst, np.max(np.abs(quad_integrals(8, tgt, h, 0.2) - ref) / np.abs(ref)))
    assert worst < 1e-13


def test_triangle_far_rule_error():
    worst = 0.0
    for R in (0.026, 0.06, 0.15):           # circumradius; k 2R up to 1.9
        for tgt in _targets(5.0 * R):
            ref = tri_parts(40, tgt, R)
            assert np.max(np.abs(tri_parts(12, tgt, R) - ref) / np.abs(ref)) < 1e-13  # the reference's own rule
            worst = max(worst, np.max(np.abs(tri_collapsed(8, tgt, R) - ref) / np.abs(ref)))
    assert worst < 1e-13


def test_closer_pairs_need_the_reference_rule():
    """At 3 R the 8 x 8 rule is no longer within the bar: the 5 R threshold is needed."""
    h = 0.039
    Rs = h * np.sqrt(2)
    worst = 0.0
    for tgt in _targets(3.0 * Rs):
        ref = quad_integrals(40, tgt, h, 0.2)
        worst = max(worst, np.max(np.abs(quad_integrals(8, tgt, h, 0.2) - ref) / np.abs(ref)))
    assert worst > 1e-12

"""The oracle pinned against the reference's own known-answer tests (CPU)."""
import json
import os

import numpy as np
import pytest

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def test_hankel2_known_answers(oracle_lib):
    """lib_math_bessel.f90: test_lib_math_bessel_spherical_third_kind_2_real (x = 2,
    orders 0..40, |log(value) - log(truth)| <= 1e-13 for Re and Im)."""
    g = json.load(open(os.path.join(GOLD, "hankel2_x2.json")))
    h = oracle_lib.hankel2(g["x"], len(g["re"]))
    re, im = np.array(g["re"]), np.array(g["im"])
    # orders 0 (negative imaginary part) compared on the magnitude like the reference
    assert np.all(np.abs(np.log(np.abs(h.real)) - np.log(np.abs(re))) <= 1e-13)
    assert np.all(np.abs(np.log(np.abs(h.imag)) - np.log(np.abs(im))) <= 1e-13)
    assert np.all(np.sign(h.real) == np.sign(re)) and np.all(np.sign(h.imag) == np.sign(im))


def test_hankel2_complex_known_answers(oracle_lib):
    """lib_math_bessel.f90: test_lib_math_bessel_spherical_third_kind_2_cmplx (z = 2 + 2i,
    orders 0..40, |log|value| - log|truth|| <= 1e-13 for Re and Im, signs equal).  The
    translation tables evaluate h2 at complex k R in a lossy medium; this pins the
    recurrence off the real axis."""
    g = json.load(open(os.path.join(GOLD, "hankel2_x2p2i.json")))
    h = oracle_lib.hankel2(complex(*g["x"]), len(g["re"]))
    re, im = np.array(g["re"]), np.array(g["im"])
    assert np.all(np.abs(np.log(np.abs(h.real)) - np.log(np.abs(re))) <= g["tolerance_log"])
    assert np.all(np.abs(np.log(np.abs(h.imag)) - np.log(np.abs(im))) <= g["tolerance_log"])
    assert np.all(np.sign(h.real) == np.sign(re)) and np.all(np.sign(h.imag) == np.sign(im))


@pytest.mark.parametrize("z", [3.7 + 0.0j, 12.0 + 0.0j, 25.3 + 0.0j, 5.0 - 0.3j, 9.0 - 1.0j])
def test_hankel2_vs_scipy(oracle_lib, z):
    from scipy.special import spherical_jn, spherical_yn
    n = np.arange(19)
    ref = spherical_jn(n, z) - 1j * spherical_yn(n, z)
    h = oracle_lib.hankel2(z, 19)
    assert np.allclose(h, ref, rtol=1e-11, atol=0)


def test_hankel2_lossy_argument_is_accurate(oracle_lib):
    """For k2 R with a large negative imaginary part, h2 = i^(n+1) e^{-iz}/z * poly(1/z)
    is tiny; the upward recurrence keeps its relative accuracy (A&S 10.1.17)."""
    from math import factorial
    z = 3.0 - 40.0j
    h = oracle_lib.hankel2(z, 12)
    for n in range(12):
        s = sum(factorial(n + k) / (factorial(k) * factorial(n - k)) / (2j * z) ** k for k in range(n + 1))
        exact = 1j ** (n + 1) * np.exp(-1j * z) / z * s
        assert abs(h[n] - exact) <= 1e-12 * abs(exact)


@pytest.mark.parametrize("n", [3, 7, 19, 33])
def test_gauss_legendre(oracle_lib, n):
    x, w = oracle_lib.gauss_legendre(n)
    xr, wr = np.polynomial.legendre.leggauss(n)
    assert np.allclose(x, xr, atol=1e-14) and np.allclose(w, wr, atol=1e-14)


def test_gmres_tridiagonal_all_ones(oracle_lib):
    """lib_math_solver_GMRES.f90 GMRES_test: 100 x 100, diagonal 4, off-diagonals
    -2+i, b = A * ones, restart 60; the solution is the all-ones vector."""
    g = json.load(open(os.path.join(GOLD, "gmres_tridiag.json")))
    n = g["n"]
    A = np.diag(np.full(n, complex(*g["diag"]))) + np.diag(np.full(n - 1, complex(*g["offdiag"])), 1) \
        + np.diag(np.full(n - 1, complex(*g["offdiag"])), -1)
    b = A @ np.ones(n)
    x, info = oracle_lib.zgmres(lambda v: A @ v, b, g["restart"], 1e-13, 1000)
    assert info["converged"]
    assert np.allclose(x, np.ones(n), atol=1e-9)


def test_tree_universal_index_known_answers(oracle_lib):
    """lib_tree_helper_functions.f90: test_lib_tree_hf_get_universal_index (3-D branch:
    (0.75, 0.5, 2^-9 + 2^-8) at level 1 is box 6) and
    test_lib_tree_hf_get_universal_index_l_max (double points, 8-byte index: every
    coordinate 1 - 2^-21 at level 21 = int(64 / 3) is box 2^63 - 1)."""
    assert oracle_lib.universal_index([0.75, 0.5, 2.0 ** -9 + 2.0 ** -8], 1) == 6
    f = 1.0 - 2.0 ** -21
    assert oracle_lib.universal_index([f, f, f], 21) == 2 ** 63 - 1


def test_tree_neighbours_known_answers(oracle_lib):
    """lib_tree_helper_functions.f90: test_lib_tree_hf_get_neighbour_all_xD (3-D, k = 1,
    box 35 at level 2, all 26 neighbours inside the domain) and
    test_lib_tree_hf_get_neighbour_all_xD_2 (box 5 at level 1, a corner box with 7).
    The reference lists them in its loop order, which the oracle keeps."""
    truth = [4, 5, 12, 6, 7, 14, 20, 21, 28, 32, 33, 40, 34, 42, 48, 49, 56,
             36, 37, 44, 38, 39, 46, 52, 53, 60]
    assert oracle_lib.neighbours(35, 2).tolist() == truth
    assert oracle_lib.neighbours(5, 1).tolist() == [0, 1, 2, 3, 4, 6, 7]


@pytest.mark.parametrize("ngp,degree", [(1, 1), (3, 2), (4, 3), (6, 4), (7, 5), (12, 6)])
def test_triangle_rules_match_the_reference_tables(oracle_lib, ngp, degree):
    """Quadrature_tri (lib_sie_integration_points.f90:7-143): the oracle holds every
    point and weight as the binary32 value of the reference's decimal literal (the
    reference is compiled without real-kind promotion), and each rule integrates the
    monomials a^i b^j, i + j <= degree, over the unit triangle to binary32 accuracy:
    sum w a^i b^j = 2 i! j! / (i + j + 2)!."""
    from math import factorial
    g = json.load(open(os.path.join(GOLD, "quadrature_tri.json")))["rules"][str(ngp)]
    a, b, w = oracle_lib.quad_rule(ngp)
    f32 = lambda v: np.asarray(v, np.float32).astype(np.float64)
    assert np.array_equal(a, f32(g["alpha"]))
    assert np.array_equal(b, f32(g["beta"]))
    assert np.array_equal(w, f32(g["ww"]))
    for i in range(degree + 1):
        for j in range(degree + 1 - i):
            exact = 2.0 * factorial(i) * factorial(j) / factorial(i + j + 2)
            assert abs(np.sum(w * a ** i * b ** j) - exact) <= 3e-7, (i, j)

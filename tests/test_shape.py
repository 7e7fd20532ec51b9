"""Host-side shape parameterisation (no GPU): the B-spline height map and the observation
cone used by the shape gradient."""
import numpy as np

from specklesim_b200.shape import BSplineHeight, SpeckleProblem, bspline_basis_1d, cone_points
from tests import problems as P


def test_bspline_partition_of_unity_and_support():
    x = np.linspace(-1.0, 1.0, 101)
    B = bspline_basis_1d(x, -1.0, 1.0, 8)
    assert B.shape == (101, 8)
    assert np.allclose(B.sum(axis=1), 1.0, atol=1e-14)
    assert (B >= 0).all()
    # every point sees at most four functions
    assert ((B > 0).sum(axis=1) <= 4).all()


def test_bspline_reproduces_linear_functions():
    """Cubic B-splines reproduce linear functions with control values at their centres."""
    n, x0, x1 = 10, -2.0, 3.0
    h = (x1 - x0) / (n - 3)
    c = x0 + (np.arange(n) - 1) * h
    x = np.linspace(x0, x1, 57)
    B = bspline_basis_1d(x, x0, x1, n)
    assert np.allclose(B @ (0.7 * c - 0.2), 0.7 * x - 0.2, atol=1e-12)


def test_height_matrix_is_a_tensor_product():
    s = BSplineHeight(6, 0.0, 1.0, 0.0, 2.0)
    xy = np.array([[0.3, 1.1], [0.9, 0.2]])
    M = s.matrix(xy)
    Bx = bspline_basis_1d(xy[:, 0], 0.0, 1.0, 6)
    By = bspline_basis_1d(xy[:, 1], 0.0, 2.0, 6)
    assert M.shape == (2, 36)
    assert np.allclose(M[1].reshape(6, 6), np.outer(Bx[1], By[1]))
    assert np.allclose(M.sum(axis=1), 1.0)


def test_cone_points_lie_in_the_cone():
    axis = np.array([np.sin(0.3), 0.0, np.cos(0.3)])
    p = cone_points(500, axis, 20.0, seed=4, r=5.0)
    r = np.linalg.norm(p, axis=1)
    assert np.allclose(r, 5.0)
    cosang = p @ axis / r
    assert cosang.min() >= np.cos(np.deg2rad(20.0)) - 1e-12


def test_problem_moves_only_the_top_face():
    cells, L = 6, 1.5
    V, T = P.slab(cells=cells, length_wl=L, seed=2, rms_wl=0.2, corr_wl=0.5, thickness_wl=0.5)
    top = np.arange((cells + 1) ** 2)
    half = 0.5 * L * P.WL
    pb = SpeckleProblem(V, T, top, BSplineHeight(5, -half, half, -half, half), P.WL, P.EPS_METAL,
                        [0, 0, -1.0], [1.0, 0, 0], np.zeros((1, 3)), dense=True)
    c = np.random.default_rng(0).standard_normal(25) * 1e-3 * P.WL
    W = pb.vertices(c)
    assert np.array_equal(W[len(top):], V[len(top):])
    assert np.array_equal(W[:, :2], V[:, :2])
    assert np.allclose(W[top, 2] - V[top, 2], pb.B @ c)

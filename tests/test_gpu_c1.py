"""The small-sphere configuration at its stated size (needs a B200): icosphere of radius
0.5 lambda, subdivision 3 (1280 flat triangles, 1920 RWG edges, 3840 unknowns),
lambda = 632.8 nm, eps = -11.7 - 1.26i, one x-polarised plane wave along -z, 7-point rule,
dense matrix (no MLFMM), GMRES restart 50 to 1e-6, and the 181-point far-field cut.

The reference runs this through its normal solver (lib_sie_tri_solver_normal_I,
src/lib_sie_tri_solver_normal.f90:64-217: dense fill and ZGESV) or through GMRES on the
same matrix; the oracle's dense matrix solved by numpy stands for ZGESV."""
import numpy as np
import pytest

from tests import problems as P

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.fixture(scope="module")
def c1(oracle_lib, gpu_lib):
    from specklesim_b200 import Sie, incidence
    from specklesim_b200.observation import evaluation_points
    V, T = P.sphere(3)
    assert T.shape[0] == 1280
    o = oracle_lib.Oracle(V, T, P.WL, P.EPS_METAL, ngp=7, threads=8)
    g = Sie(V, T, P.WL, P.EPS_METAL, ngp=7, dense=True).setup()
    assert g.n_edges == 1920
    k, E = incidence(0.0, 0.0, "TM", 2)  # k along -z, E along x
    assert np.allclose(k, [0, 0, -1]) and abs(E[0]) > 0.99
    b = o.rhs(k, E)
    x_ref = np.linalg.solve(o.dense(), b)
    # the 181-point cut: theta 0 .. 180 degrees at phi = 0, r = 5 m (the reference's
    # far-field observation distance, position_c)
    pts = evaluation_points("rcs_p", (0.0, np.pi), (0.0, 0.0), 5.0, 181)
    yield o, g, b, x_ref, pts
    g.close()
    o.close()


def test_direct_solves_match_dense_oracle(c1):
    o, g, b, x_ref, pts = c1
    assert _rel(g.rhs_planewave(*__import__("specklesim_b200").incidence(0.0, 0.0, "TM", 2)), b) < 1e-12
    x64 = g.solve_direct(b)
    assert _rel(x64, x_ref) < 1e-9
    xm, st = g.solve_direct_mixed(b, tolerance=1e-12)
    assert st["converged"] and _rel(xm, x_ref) < 1e-9
    _, _, I_ref = o.field(x_ref, pts)
    _, _, I = g.farfield(x64, pts)
    assert I.shape == (181,) and _rel(I, I_ref) < 1e-8
    g.release_factors()


def test_gmres_to_1e6_on_the_dense_matrix(c1):
    o, g, b, x_ref, pts = c1
    x, st = g.solve(b, restart=50, max_iterations=3000, tolerance=1e-6)
    assert st["converged"] and st["backward_error_true"] <= 1e-6
    Z = o.dense()
    assert np.linalg.norm(Z @ x - b) / np.linalg.norm(b) < 1.5e-6
    # the far-field cut of the iterative solution against the direct one
    _, _, I_ref = o.field(x_ref, pts)
    _, _, I = g.farfield(x, pts)
    assert _rel(I, I_ref) < 1e-3

"""Shape gradient of the far-field speckle objective against central finite differences of
the solver itself (needs a B200).

J = sum of far-field intensities over observation points in a 20-degree cone around the
specular direction.  The gradient (one adjoint solve plus the derivative kernels) must
match (J(z + d) - J(z - d)) / 2d to 1e-4 relative, on vertex heights of a dense-LU slab
and on B-spline controls of an MLFMM slab (solved exactly, so that the differences are
not swamped by the iterative solver's tolerance)."""
import numpy as np
import pytest

from tests import problems as P

pytestmark = pytest.mark.gpu


def _small_slab():
    return P.slab(cells=6, length_wl=1.5, seed=2, rms_wl=0.2, corr_wl=0.5, thickness_wl=0.5)


def _dense_J(V, T, k, E, pts):
    """J of the oracle's own dense system (the reference's fill restated on the CPU, solved
    by numpy's LU as ZGESV would), the function the finite differences are taken of."""
    from oracle import oracle
    o = oracle.Oracle(V, T, P.WL, P.EPS_METAL, threads=8)
    try:
        x = np.linalg.solve(o.dense(), o.rhs(k, E))
        return float(np.sum(o.field(x, pts)[2]))
    finally:
        o.close()


def test_vertex_gradient_matches_finite_differences_dense(gpu_lib, oracle_lib):
    from specklesim_b200 import Sie, incidence
    from specklesim_b200.shape import cone_points
    V, T = _small_slab()
    k, E = incidence(np.deg2rad(10.0), 0.0, "TM", 2)
    pts = cone_points(16, [np.sin(np.deg2rad(10.0)), 0, np.cos(np.deg2rad(10.0))], 20.0, seed=1)
    g = Sie(V, T, P.WL, P.EPS_METAL, dense=True).setup()
    x = g.solve_direct(g.rhs_planewave(k, E))
    J, dz, st = g.grad(x, k, E, pts)
    g.close()
    # the GPU's J is the oracle's to the fill's rounding (blocks agree to 1e-9)
    assert abs(J - _dense_J(V, T, k, E, pts)) <= 1e-8 * abs(J)
    # rough top face and a side-wall vertex.  Vertices of the exactly flat bottom face are
    # left out: there the singular terms of coplanar pairs sit on the zero-height branch of
    # the reference's formulas (unsigned solid angle, line logarithms), where Z is not
    # smooth and finite differences themselves change with the step (~1e-3 between steps
    # of 1e-4 and 1e-6 lambda).
    verts = [3, 17, 24, 40, len(V) - 3]
    d = 1e-4 * P.WL
    for v in verts:
        Vp, Vm = V.copy(), V.copy()
        Vp[v, 2] += d
        Vm[v, 2] -= d
        fd = (_dense_J(Vp, T, k, E, pts) - _dense_J(Vm, T, k, E, pts)) / (2 * d)
        assert abs(dz[v] - fd) <= 1e-4 * abs(fd) + 1e-7 * np.abs(dz).max(), (v, dz[v], fd)


@pytest.fixture(scope="module")
def mlfmm_problem(gpu_lib):
    from specklesim_b200 import incidence
    from specklesim_b200.shape import BSplineHeight, SpeckleProblem, cone_points
    cells, L = 16, 4.0
    V, T = P.slab(cells=cells, length_wl=L, seed=2)
    top = np.arange((cells + 1) ** 2)
    half = 0.5 * L * P.WL
    spline = BSplineHeight(6, -half, half, -half, half)
    k, E = incidence(0.0, 0.0, "TM", 2)
    # observation points 100 lambda away: at 5 m the distances carry a rounding of ~1e-16 m,
    # which a 1e-6 lambda step would not clear
    pts = cone_points(32, [0, 0, 1], 20.0, seed=3, r=100 * P.WL)
    return SpeckleProblem(V, T, top, spline, P.WL, P.EPS_DIELECTRIC, k, E, pts, dense=False, tree_s_opt=60,
                          tolerance=1e-10)


def _exact(pb, c):
    """J and x of the MLFMM system at controls c, solved exactly: the operator is assembled
    column by column with batched products and factorised on the GPU.  (An iterative solve
    leaves J accurate to ~cond(Z) x its tolerance, too coarse for small steps.)"""
    import torch
    from specklesim_b200 import Sie
    g = Sie(pb.vertices(c), pb.T, P.WL, pb.eps, tree_s_opt=pb.s_opt).setup()
    try:
        assert g.l_max > g.l_min  # the far field goes through the MLFMM passes
        Z = g.matvec(np.eye(g.n, dtype=np.complex128))
        b = g.rhs_planewave(pb.k_in, pb.E_in)
        x = torch.linalg.solve(torch.from_numpy(Z).cuda(), torch.from_numpy(b).cuda()).cpu().numpy()
        return float(np.sum(g.farfield(x, pb.pts)[2])), x, g.grad(x, pb.k_in, pb.E_in, pb.pts, tolerance=1e-10,
                                                                   max_iterations=4000)
    finally:
        g.close()


def test_control_gradient_matches_finite_differences_mlfmm(mlfmm_problem):
    """B-spline controls of an MLFMM slab: dJ/dc = B^T dJ/dz against central differences
    of the exact solve with step 1e-6 lambda.  The step is small because the operator is
    only piecewise smooth in the vertex positions: a pair whose centroid distance crosses
    the singular-quadrature threshold (or an edge midpoint that changes box) makes J jump,
    and a step of 1e-4 lambda over a control's 3-lambda support meets such crossings."""
    pb = mlfmm_problem
    c0 = np.zeros(pb.B.shape[1])
    J, x, (Jg, dz, st) = _exact(pb, c0)
    assert st["converged"] and abs(Jg - J) <= 1e-10 * abs(J)
    dc = pb.B.T @ dz[pb.top]
    d = 1e-6 * P.WL
    # The differences of the exact solve carry a noise floor of ~1e-11 (rounding of the
    # assembled operator, which varies with the geometry); relative to it, only controls
    # with a large derivative resolve 1e-4, so the check takes the four largest.
    for i in np.argsort(-np.abs(dc))[:4]:
        e = np.zeros_like(c0)
        e[i] = d
        fd = (_exact(pb, c0 + e)[0] - _exact(pb, c0 - e)[0]) / (2 * d)
        assert abs(dc[i] - fd) <= 1e-4 * abs(fd) + 1e-7 * np.abs(dc).max(), (i, dc[i], fd)


def test_torch_autograd_function(mlfmm_problem):
    import torch
    from specklesim_b200.shape import speckle_objective
    pb = mlfmm_problem
    f = speckle_objective(pb)
    c = torch.zeros(pb.B.shape[1], dtype=torch.float64, requires_grad=True)
    J = f(c)
    J.backward()
    J2, dc = pb.value_and_grad(np.zeros(pb.B.shape[1]))
    assert abs(J.item() - J2) <= 1e-12 * abs(J2)
    assert np.allclose(c.grad.numpy(), dc, rtol=1e-12, atol=0)

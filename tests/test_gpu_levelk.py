"""MLFMM product with a truncation number per level (sie_set_level_truncation) against the
oracle's product with the same truncation numbers (needs a B200).

The reference's per-level branch (Truncation_number_calculation, lib_sie_mlfmm.f90:631-701,
dormant: every level gets truncation_number_default) interpolates a child level's
coefficients to its parent's sampling in SS (Lagrange_Interpolation_New, :268-390, called
from lib_sie_tri_mlfmm_interface.f90:486-507) and goes back down in RR.  The oracle
restates it with three departures, each needed for a correct product (per-level SR
weights, anterpolation in RR, the -z pole of the receive); the GPU path follows the oracle.
The two implementations share the interpolation stencils (interp_csr against
lagrange_interp to 1e-13), so the products agree to the translation's rounding."""
import numpy as np
import pytest

from tests import problems as P

pytestmark = pytest.mark.gpu

CASES = {
    # 4 lambda slab, levels 2..3 (0.5 lambda leaves): one interpolation step
    "two_levels": dict(cells=16, length_wl=4.0, s_opt=60, K={3: 14, 2: 16}),
    # 6 lambda slab, levels 2..4 (0.375 lambda leaves): interpolation into a non-leaf
    # level and from it
    "three_levels": dict(cells=24, length_wl=6.0, s_opt=40, K={4: 12, 3: 16, 2: 21}),
}


@pytest.fixture(scope="module", params=sorted(CASES))
def pair(request, oracle_lib, gpu_lib):
    from specklesim_b200 import Sie
    c = CASES[request.param]
    V, T = P.slab(cells=c["cells"], length_wl=c["length_wl"], seed=3)
    o = oracle_lib.Oracle(V, T, P.WL, P.EPS_METAL, tree_s_opt=c["s_opt"], threads=8)
    o.tree()
    o.set_level_truncation(c["K"])
    o.setup_fmm()
    g = Sie(V, T, P.WL, P.EPS_METAL, tree_s_opt=c["s_opt"], level_truncation=c["K"]).setup()
    yield request.param, o, g
    g.close()
    o.close()


def _rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def test_level_truncation_product_matches_oracle(pair):
    name, o, g = pair
    assert g.l_max - g.l_min == (1 if name == "two_levels" else 2)
    Q = np.zeros(1, np.int32)
    from specklesim_b200 import _lib
    import ctypes as C
    _lib.check(g._lib.sie_num_directions(g._h, Q.ctypes.data_as(C.POINTER(C.c_int))))
    K_leaf = CASES[name]["K"][g.l_max]
    assert Q[0] == 2 * K_leaf * K_leaf + 2
    for seed in (1, 2):
        x = P.random_x(g.n, seed=seed)
        assert _rel(g.matvec(x), o.matvec(x)) < 1e-10


def test_level_truncation_complex64_and_batched_products(pair):
    _, o, g = pair
    X = np.stack([P.random_x(g.n, seed=s) for s in range(3, 6)], axis=1)
    Y = g.matvec(X)
    for j in range(X.shape[1]):
        y1 = g.matvec(X[:, j])
        assert _rel(Y[:, j], y1) < 1e-12
        assert _rel(g.matvec(X[:, j], precision="mixed"), y1) < 2e-4
    Y32 = g.matvec(X, precision="mixed")
    for j in range(X.shape[1]):
        assert _rel(Y32[:, j], Y[:, j]) < 2e-4


def test_level_truncation_solves_and_refuses_adjoint(pair):
    """On the smaller slab the preconditioned solve converges; on the 6 lambda metal slab a
    budgeted solve's reported residual is the one the oracle's product gives for its
    currents (the same operator)."""
    from specklesim_b200 import SieError, _lib, incidence
    name, o, g = pair
    k, E = incidence(0.0, 0.0, "TM", 2)
    b = g.rhs_planewave(k, E)
    g.set_preconditioner("near")
    if name == "two_levels":
        x, st = g.solve(b, restart=200, max_iterations=400, tolerance=1e-6)
        assert st["converged"]
        assert _rel(o.matvec(x), b) < 2e-6
    else:
        x, st = g.solve(b, restart=100, max_iterations=100, tolerance=1e-6, raise_on_noconv=False)
        r = _rel(o.matvec(x), b)
        assert st["iterations"] == 100 and abs(r - st["backward_error_true"]) < 1e-8 * r
    g.set_preconditioner(None)
    with pytest.raises(SieError) as e:
        g.matvec_adjoint(x)
    assert e.value.code == _lib.SIE_ERR_STATE


def test_level_truncation_growing_toward_leaf_is_refused(gpu_lib):
    from specklesim_b200 import Sie, SieError, _lib
    V, T = P.slab(cells=16, length_wl=4.0, seed=3)
    with pytest.raises(SieError) as e:
        Sie(V, T, P.WL, P.EPS_METAL, tree_s_opt=60, level_truncation={3: 16, 2: 14})
    assert e.value.code == _lib.SIE_ERR_ARG

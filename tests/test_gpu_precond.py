"""Near-field restricted additive Schwarz preconditioner (sie_set_preconditioner) against
a numpy construction of the same operator from the oracle's near-field CSR, and the
preconditioned solvers against the unpreconditioned ones (needs a B200).

The reference has no such preconditioner (its only option is the left Jacobi scaling of
lib_sie_ml_fmm_preconditioner_left, src/lib_sie_tri_mlfmm_interface.f90:323-339); the
operator checked here is defined from the reference's own near matrix
(precalculation_near_field_csr_tri, :779-863): for each leaf box A, the near entries
among the edges of E2(A) form a local system L_A, and the rows of L_A^{-1} that belong to
A's unknowns are the preconditioner's rows."""
import numpy as np
import pytest

from tests import problems as P

pytestmark = pytest.mark.gpu


def ras_dense(o, leaf):
    """P as a dense matrix in the reference's unknown order (x(1:M) = J, x(M+1:2M) = M);
    o has its tree and near field set up, leaf is the leaf box of every edge."""
    ia, ja, v = o.near_csr()
    M = o.M
    near = np.zeros((2 * M, 2 * M), complex)
    for m in range(M):
        cols = ja[ia[m]:ia[m + 1]]
        near[m, cols] = v[ia[m]:ia[m + 1], 0]
        near[m, cols + M] = v[ia[m]:ia[m + 1], 1]
        near[m + M, cols] = v[ia[m]:ia[m + 1], 2]
        near[m + M, cols + M] = v[ia[m]:ia[m + 1], 3]
    Pm = np.zeros((2 * M, 2 * M), complex)
    for bx in np.unique(leaf):
        e = np.nonzero(leaf == bx)[0]
        s = ja[ia[e[0]]:ia[e[0] + 1]]          # E2(A): the columns of A's near rows
        idx = np.concatenate([s, s + M])
        inv = np.linalg.inv(near[np.ix_(idx, idx)])
        pos = np.searchsorted(s, e)
        rows = np.concatenate([pos, pos + len(s)])
        Pm[np.ix_(np.concatenate([e, e + M]), idx)] = inv[rows]
    return Pm


@pytest.fixture(scope="module")
def metal_slab(oracle_lib, gpu_lib):
    from specklesim_b200 import Sie
    V, T = P.slab(cells=16, length_wl=3.0, seed=3)
    o = oracle_lib.Oracle(V, T, P.WL, P.EPS_METAL, tree_s_opt=60, threads=8)
    leaf = o.tree()["leaf"]
    o.setup_fmm()
    g = Sie(V, T, P.WL, P.EPS_METAL, tree_s_opt=60).setup()
    yield o, g, leaf
    g.close()
    o.close()


def test_preconditioner_matches_numpy_construction(metal_slab):
    o, g, leaf = metal_slab
    Pm = ras_dense(o, leaf)
    g.set_preconditioner("near")
    for seed in (1, 2):
        x = P.random_x(g.n, seed=seed)
        y = g.precondition_right(x)
        ye = Pm @ x
        err = np.linalg.norm(y - ye) / np.linalg.norm(ye)
        # the local systems' condition numbers (~1e5) times rounding: measured 2.9e-10
        assert err < 1e-8, err


def test_preconditioned_solve_converges_where_plain_gmres_stalls(metal_slab):
    """The plasmonic slab: GMRES(50) on Z stalls far above 1e-6 within 300 steps; right
    preconditioned by P it converges, and its currents solve the unpreconditioned system
    (true residual of the oracle's product)."""
    from specklesim_b200 import incidence
    o, g, _ = metal_slab
    k, E = incidence(0.0, 0.0, "TM", 2)
    b = g.rhs_planewave(k, E)
    g.set_preconditioner(None)
    _, st0 = g.solve(b, restart=50, max_iterations=300, tolerance=1e-6, raise_on_noconv=False)
    assert not st0["converged"] and st0["backward_error_true"] > 1e-2
    g.set_preconditioner("near")
    x, st = g.solve(b, restart=300, max_iterations=300, tolerance=1e-6)
    assert st["converged"]
    r = np.linalg.norm(b - o.matvec(x)) / np.linalg.norm(b)
    assert r < 2e-6 and abs(r - st["backward_error_true"]) < 1e-7 + 1e-6 * r
    g.set_preconditioner(None)


def test_preconditioned_mixed_solve(oracle_lib, gpu_lib):
    """The mixed-precision solver (FP64 flexible GMRES around complex64 GMRES on Z P)
    reaches the FP64 solution.  Its inner complex64 product needs a leaf truncation number
    sized to the 0.375 lambda leaves: K = 19 there loses all digits to the translation's
    cancellation in FP32, so the leaf level runs K = 12 (the upper level 16)."""
    from specklesim_b200 import Sie, incidence
    V, T = P.slab(cells=16, length_wl=3.0, seed=3)
    kk = {3: 12, 2: 16}
    o = oracle_lib.Oracle(V, T, P.WL, P.EPS_METAL, tree_s_opt=60, threads=8)
    o.tree()
    o.set_level_truncation(kk)
    o.setup_fmm()
    g = Sie(V, T, P.WL, P.EPS_METAL, tree_s_opt=60, level_truncation=kk).setup()
    k, E = incidence(0.0, 0.0, "TM", 2)
    b = g.rhs_planewave(k, E)
    g.set_preconditioner("near")
    x, st = g.solve(b, restart=300, max_iterations=300, tolerance=1e-6)
    xm, sm = g.solve(b, restart=30, max_iterations=150, tolerance=1e-6, precision="mixed",
                     inner_restart=150, inner_tolerance=1e-2)
    assert sm["converged"]
    rm = np.linalg.norm(b - o.matvec(xm)) / np.linalg.norm(b)
    assert rm < 2e-6
    assert np.linalg.norm(xm - x) / np.linalg.norm(x) < 5e-5
    g.close()
    o.close()


def test_preconditioner_refuses_dense_contexts_and_bad_kinds(gpu_lib):
    from specklesim_b200 import Sie, SieError, _lib
    V, T = P.sphere(1)
    d = Sie(V, T, P.WL, P.EPS_METAL, dense=True)
    with pytest.raises(SieError) as e:
        d.set_preconditioner("near")  # before set-up
    assert e.value.code == _lib.SIE_ERR_STATE
    d.setup()
    with pytest.raises(SieError) as e:
        d.set_preconditioner("near")
    assert e.value.code == _lib.SIE_ERR_STATE
    with pytest.raises(SieError) as e:
        _lib.check(d._lib.sie_set_preconditioner(d._h, 7))
    assert e.value.code == _lib.SIE_ERR_ARG
    with pytest.raises(SieError) as e:
        d.precondition_right(np.ones(d.n, complex))
    assert e.value.code == _lib.SIE_ERR_STATE
    d.close()

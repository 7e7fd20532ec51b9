"""Batches of right-hand sides through one product and one lockstep solve (needs a B200).

A batched product must give every column the same result as the one-vector product up
to summation order, and the batched mixed-precision solve must reach the same solutions
as the plain FP64 solver."""
import numpy as np
import pytest

from tests import problems as P

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.linalg.norm(np.ravel(a - b)) / np.linalg.norm(np.ravel(b))


def _ctx(eps, dense=False):
    from specklesim_b200 import Sie
    if dense:
        V, T = P.sphere(sub=2)
        return Sie(V, T, P.WL, eps, dense=True).setup()
    V, T = P.slab(cells=24, length_wl=6.0, seed=3)
    return Sie(V, T, P.WL, eps, tree_s_opt=100).setup()


@pytest.fixture(scope="module")
def diel(gpu_lib):
    g = _ctx(P.EPS_DIELECTRIC)
    yield g
    g.close()


@pytest.fixture(scope="module")
def metal(gpu_lib):
    g = _ctx(P.EPS_METAL)
    yield g
    g.close()


def _columns(n, k, seed):
    return np.stack([P.random_x(n, seed=seed + j) for j in range(k)], axis=1)


# one batched launch sequence, a batch of 16 and a batch that is cut into slices (16 + 3)
@pytest.mark.parametrize("k", [2, 5, 16, 19])
@pytest.mark.parametrize("which", ["diel", "metal"])
def test_batched_fp64_product_equals_single(which, k, request):
    g = request.getfixturevalue(which)
    X = _columns(g.n, k, 100)
    Y = g.matvec(X)
    for j in range(k):
        assert rel(Y[:, j], g.matvec(X[:, j])) < 1e-12, (j, rel(Y[:, j], g.matvec(X[:, j])))


@pytest.mark.parametrize("k", [3, 16])
def test_batched_complex64_product_equals_single(metal, k):
    """Same complex64 tables, different summation order.  Each complex64 product is
    within ~4e-5 of the FP64 one here (FP32 rounding amplified by the cancellation of the
    K = 19 translations on 0.75-lambda boxes), so two of them differ by up to that much."""
    X = _columns(metal.n, k, 200)
    Y32 = metal.matvec(X, precision="mixed")
    for j in range(k):
        y1 = metal.matvec(X[:, j], precision="mixed")
        assert rel(Y32[:, j], y1) < 1e-4, (j, rel(Y32[:, j], y1))
        assert rel(Y32[:, j], metal.matvec(X[:, j])) < 2e-4


def test_batched_dense_product_equals_single(gpu_lib):
    g = _ctx(P.EPS_METAL, dense=True)
    try:
        X = _columns(g.n, 4, 300)
        Y = g.matvec(X)
        for j in range(4):
            assert rel(Y[:, j], g.matvec(X[:, j])) < 1e-12
    finally:
        g.close()


def test_batched_mixed_solve_matches_fp64(diel):
    """Eight incidences solved together (FP64 outer FGMRES, complex64 inner GMRES in
    lockstep) reach the FP64 tolerance on each true residual, and agree with one-at-a-time
    FP64 solves in currents and far-field intensity."""
    from specklesim_b200 import incidence
    g = diel
    inc = [incidence(np.deg2rad(t), np.deg2rad(p), pol, 2)
           for t in (0, 20) for p in (0, 90) for pol in ("TM", "TE")]
    B = np.stack([g.rhs_planewave(k, E) for k, E in inc], axis=1)
    Xb, sb = g.solve(B, restart=10, max_iterations=60, tolerance=1e-8, precision="mixed",
                     inner_restart=30, inner_tolerance=1e-2)
    th = np.linspace(0.05, 1.4, 9)
    pts = 5.0 * np.stack([np.sin(th), 0 * th, np.cos(th)], axis=1)
    for j in range(B.shape[1]):
        assert sb[j]["converged"] and sb[j]["backward_error_true"] <= 1e-8, sb[j]
        x64, s64 = g.solve(B[:, j], restart=50, max_iterations=3000, tolerance=1e-8)
        assert rel(Xb[:, j], x64) < 1e-5, (j, rel(Xb[:, j], x64))
        I64 = g.farfield(x64, pts)[2]
        Ib = g.farfield(Xb[:, j], pts)[2]
        assert rel(Ib, I64) < 1e-5, (j, rel(Ib, I64))


def test_batched_solve_of_one_converged_column(diel):
    """A zero right-hand side in the batch is solved by x = 0 at once and does not disturb
    the other columns."""
    from specklesim_b200 import incidence
    g = diel
    k, E = incidence(0.0, 0.0, "TM", 2)
    b = g.rhs_planewave(k, E)
    B = np.stack([b, np.zeros_like(b), 2.0 * b], axis=1)
    X, st = g.solve(B, restart=10, max_iterations=60, tolerance=1e-7, precision="mixed",
                    inner_restart=30, inner_tolerance=1e-2)
    assert st[1]["converged"] and np.all(X[:, 1] == 0)
    assert st[0]["converged"] and st[2]["converged"]
    assert rel(X[:, 2], 2.0 * X[:, 0]) < 1e-6


def test_batched_overlap_gives_the_same_product(gpu_lib, monkeypatch):
    """The batched near product on the second stream, beside the translations, gives
    bit-identical results to the sequential order (FP64 and complex64)."""
    from specklesim_b200 import Sie
    V, T = P.slab(cells=24, length_wl=6.0, seed=3)
    out = []
    for ov in ("0", "1", "2", "3"):
        monkeypatch.setenv("SIE_OVERLAP", ov)
        g = Sie(V, T, P.WL, P.EPS_METAL, tree_s_opt=100).setup()
        X = _columns(g.n, 6, 400)
        out.append((g.matvec(X), g.matvec(X, precision="mixed")))
        g.close()
    for o in out[1:]:
        assert np.array_equal(out[0][0], o[0]) and np.array_equal(out[0][1], o[1])


def test_batched_mixed_solve_with_cheaper_inner_operator(diel, gpu_lib):
    """Inner complex64 products through a K = 12 context on the same mesh: the outer FP64
    products are unchanged, so the solutions still reach the FP64 tolerance and agree with
    one-at-a-time FP64 solves."""
    from specklesim_b200 import Sie, SieError, incidence
    g = diel
    V, T = P.slab(cells=24, length_wl=6.0, seed=3)
    gi = Sie(V, T, P.WL, P.EPS_DIELECTRIC, tree_s_opt=100, truncation_number=12).setup()
    other = Sie(*P.sphere(sub=1), P.WL, P.EPS_DIELECTRIC).setup()
    try:
        with pytest.raises(SieError):
            g.set_inner_operator(other)  # a different mesh
        g.set_inner_operator(gi)
        inc = [incidence(np.deg2rad(t), 0.0, "TM", 2) for t in (0, 20, 30)]
        B = np.stack([g.rhs_planewave(k, E) for k, E in inc], axis=1)
        X, st = g.solve(B, restart=10, max_iterations=60, tolerance=1e-8, precision="mixed",
                        inner_restart=30, inner_tolerance=1e-2)
        x1, s1 = g.solve(B[:, 1], restart=10, max_iterations=60, tolerance=1e-8, precision="mixed",
                         inner_restart=30, inner_tolerance=1e-2)
        g.set_inner_operator(None)
        assert s1["converged"] and s1["backward_error_true"] <= 1e-8
        for j in range(B.shape[1]):
            assert st[j]["converged"] and st[j]["backward_error_true"] <= 1e-8
            x64, _ = g.solve(B[:, j], restart=50, max_iterations=3000, tolerance=1e-8)
            assert rel(X[:, j], x64) < 1e-5, (j, rel(X[:, j], x64))
    finally:
        g.set_inner_operator(None)
        gi.close()
        other.close()


def test_batched_solve_graph_replay_matches_launches(diel, monkeypatch):
    """The inner cycle replayed from its captured CUDA graph gives bit-identical solutions to
    the same cycle launched kernel by kernel."""
    from specklesim_b200 import incidence
    g = diel
    inc = [incidence(np.deg2rad(t), 0.0, "TE", 2) for t in (0, 30)]
    B = np.stack([g.rhs_planewave(k, E) for k, E in inc], axis=1)
    kw = dict(restart=4, max_iterations=12, tolerance=1e-9, precision="mixed", inner_restart=20,
              inner_tolerance=1e-2, raise_on_noconv=False)
    monkeypatch.setenv("SIE_GRAPH", "0")
    X0, s0 = g.solve(B, **kw)
    assert g.timings()["graph_replays"] == 0
    monkeypatch.setenv("SIE_GRAPH", "1")
    X1, s1 = g.solve(B, **kw)
    assert s1[0]["iterations"] == s0[0]["iterations"] >= 8
    # every cycle after the first (uncaptured) and the second (captured, then launched)
    assert g.timings()["graph_replays"] == s1[0]["iterations"] - 1
    assert np.array_equal(X0, X1)

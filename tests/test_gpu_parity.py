"""CUDA path vs the CPU oracle, through the C-ABI (needs a B200)."""
import numpy as np
import pytest

from tests import problems as P

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.linalg.norm(np.ravel(a - b)) / np.linalg.norm(np.ravel(b))


# 6-lambda slabs, s_opt = 100: levels 2..3 with 0.75-lambda leaf boxes, where the
# K = 19 translation operator is well conditioned (see MATVEC_RTOL below).
@pytest.fixture(scope="module")
def slab_pair(oracle_lib, gpu_lib):
    from specklesim_b200 import Sie
    V, T = P.slab(cells=24, length_wl=6.0, seed=3)
    o = oracle_lib.Oracle(V, T, P.WL, P.EPS_DIELECTRIC, tree_s_opt=100, threads=8)
    info = o.tree()
    o.setup_fmm()
    g = Sie(V, T, P.WL, P.EPS_DIELECTRIC, tree_s_opt=100).setup()
    yield o, info, g
    g.close()


@pytest.fixture(scope="module")
def metal_pair(oracle_lib, gpu_lib):
    from specklesim_b200 import Sie
    V, T = P.slab(cells=24, length_wl=6.0, seed=3)
    o = oracle_lib.Oracle(V, T, P.WL, P.EPS_METAL, tree_s_opt=100, threads=8)
    info = o.tree()
    o.setup_fmm()
    g = Sie(V, T, P.WL, P.EPS_METAL, tree_s_opt=100).setup()
    yield o, info, g
    g.close()


def test_edges_and_tree_exact(slab_pair):
    o, info, g = slab_pair
    e1, c1 = o.edges()
    e2, c2 = g.edges()
    assert np.array_equal(e1, e2) and np.array_equal(c1, c2)
    D, xmin, leaf = g.tree()
    assert g.l_max == info["l_max"] and g.l_min == info["l_min"]
    assert D == info["D"] and np.array_equal(xmin, info["xmin"])
    assert np.array_equal(leaf, info["leaf"])
    assert g.near_nnz == o.nnz


def _pairs(o, rng, n=400):
    m = rng.integers(0, o.M, n)
    nn = rng.integers(0, o.M, n)
    # self, edge-adjacent and close pairs exercise the singular branch
    e, _ = o.edges()
    m2 = np.arange(0, o.M, max(1, o.M // 100))
    return np.concatenate([m, m2, m2]), np.concatenate([nn, m2, (m2 + 1) % o.M])


@pytest.mark.parametrize("which", ["slab_pair", "metal_pair"])
def test_blocks_match_oracle(which, request):
    o, _, g = request.getfixturevalue(which)
    rng = np.random.default_rng(0)
    m, n = _pairs(o, rng)
    a = g.blocks(m, n)
    b = o.blocks(m, n)
    scale = np.abs(b).max(axis=1, keepdims=True)
    err = np.abs(a - b) / scale
    assert err.max() < 1e-9, err.max()


def test_near_matrix_matches_oracle_csr(slab_pair):
    o, _, g = slab_pair
    ia, ja, v = o.near_csr()
    rows = np.arange(0, o.M, 13)
    mm = np.concatenate([np.full(ia[r + 1] - ia[r], r) for r in rows])
    nn = np.concatenate([ja[ia[r]:ia[r + 1]] for r in rows])
    vv = np.concatenate([v[ia[r]:ia[r + 1]] for r in rows])
    got = g.near_entries(mm, nn)
    scale = np.abs(vv).max(axis=1, keepdims=True)
    assert (np.abs(got - vv) / scale).max() < 1e-9


def test_radiation_patterns_match_oracle(slab_pair):
    o, _, g = slab_pair
    edges = np.arange(0, o.M, 17)
    a = g.rt(edges)
    b = o.rt()[edges]
    assert rel(a, b) < 1e-12


# The translation operator with K = 19 sums Hankel terms up to kappa times larger than
# the result (kappa = max (2n+1)|h_n(2 k d_c)| / |h_0|: ~1e4 on 0.75-lambda leaf boxes,
# ~1e8 on 0.5-lambda, ~1e10 on 0.375-lambda), so last-bit differences of the special
# functions reach ~kappa * 1e-16 in the product.
MATVEC_RTOL = 1e-10


@pytest.mark.parametrize("which", ["slab_pair", "metal_pair"])
def test_matvec_matches_oracle(which, request):
    o, _, g = request.getfixturevalue(which)
    x = P.random_x(o.N, seed=4)
    y_gpu = g.matvec(x)
    y_orc = o.matvec(x)
    assert rel(y_gpu, y_orc) < MATVEC_RTOL, rel(y_gpu, y_orc)


def test_sr_kernel_variants_agree(gpu_lib, monkeypatch):
    """The per-target and the sibling-group SR kernels give the same product."""
    from specklesim_b200 import Sie
    V, T = P.slab(cells=24, length_wl=6.0, seed=3)
    x = P.random_x(2 * 7000, seed=1)
    ys = []
    for mode in ("0", "1", "2", "3", "4", "5"):
        monkeypatch.setenv("SIE_SR_MODE", mode)
        g = Sie(V, T, P.WL, P.EPS_METAL, tree_s_opt=100).setup()
        ys.append(g.matvec(x[:g.n]))
        g.close()
    for y in ys[1:]:
        assert rel(ys[0], y) < 1e-13


@pytest.mark.parametrize("near", ["1", "2"])
def test_near_far_overlap_gives_the_same_product(gpu_lib, monkeypatch, near):
    """The near-field product on the second stream, concurrent with the translations and
    forked at any of the three points, gives bit-identical results to the sequential
    order (FP64 and complex64), with 8- and 4-warp blocks of the chunked near kernel."""
    from specklesim_b200 import Sie
    V, T = P.slab(cells=24, length_wl=6.0, seed=3)
    x = P.random_x(2 * 7000, seed=3)
    out = []
    monkeypatch.setenv("SIE_NEAR_MODE", near)
    for ov in ("0", "1", "2", "3"):
        monkeypatch.setenv("SIE_OVERLAP", ov)
        g = Sie(V, T, P.WL, P.EPS_METAL, tree_s_opt=100).setup()
        out.append((g.matvec(x[:g.n]), g.matvec(x[:g.n], precision="mixed")))
        g.close()
    for o in out[1:]:
        assert np.array_equal(out[0][0], o[0]) and np.array_equal(out[0][1], o[1])


def test_matvec_two_rhs_columns(slab_pair):
    o, _, g = slab_pair
    X = np.stack([P.random_x(o.N, seed=7), P.random_x(o.N, seed=8)], axis=1)
    Y = g.matvec(X)
    for j in range(2):
        assert rel(Y[:, j], o.matvec(X[:, j])) < MATVEC_RTOL


def test_rhs_matches_oracle(slab_pair):
    from specklesim_b200 import incidence
    o, _, g = slab_pair
    k, E = incidence(0.2, 0.5, "TE", 2)
    b1 = g.rhs_planewave(k, E)
    b2 = o.rhs(k, E)
    assert rel(b1, b2) < 1e-13


def test_host_copies_are_ordered_in_later_contexts(gpu_lib):
    """Right-hand sides and far fields from host buffers come out the same in every
    context of a process (host copies complete before the library's stream uses them)."""
    from specklesim_b200 import Sie, incidence
    V, T = P.sphere(1)
    k, E = incidence(0.3, 0.2, "TE", 2)
    pts = 5.0 * np.array([[0.1, 0.2, 0.97], [0.5, -0.3, 0.81]])
    outs = []
    for _ in range(3):
        g = Sie(V, T, P.WL, P.EPS_METAL, tree_s_opt=20).setup()
        b = g.rhs_planewave(k, E)
        outs.append((b, g.farfield(b, pts)[2]))
        g.close()
    for b, I in outs[1:]:
        assert np.array_equal(b, outs[0][0]) and np.array_equal(I, outs[0][1])


def test_solve_fixed_budget_matches_oracle_gmres(metal_pair, oracle_lib):
    """GPU GMRES (IMGS + Givens, two restarts) against the zgmres restatement driving the
    oracle matvec, on the metallic slab where both stop at the iteration budget
    (info(1) = -4 in the reference): the iterates agree."""
    from specklesim_b200 import incidence
    o, _, g = metal_pair
    k, E = incidence(0.0, 0.0, "TM", 2)
    b = o.rhs(k, E)
    x_o, info = oracle_lib.zgmres(o.matvec, b, 20, 1e-12, 45)
    x_g, st = g.solve(b, restart=20, max_iterations=45, tolerance=1e-12, raise_on_noconv=False)
    assert not st["converged"] and not info["converged"]
    assert st["iterations"] == info["iterations"] == 45
    assert rel(x_g, x_o) < 1e-7, rel(x_g, x_o)
    assert abs(st["backward_error_true"] - info["be"]) <= 1e-7 * info["be"]


def test_arnoldi_kernel_variants_agree(gpu_lib, monkeypatch):
    """The grid-barrier, tagged-exchange and single-cluster Arnoldi kernels run the same
    IMGS steps; only the order of the partial sums differs."""
    from specklesim_b200 import Sie, incidence
    V, T = P.slab(cells=24, length_wl=6.0, seed=3)
    xs = []
    for mode in ("0", "1", "2"):
        monkeypatch.setenv("SIE_ARNOLDI_MODE", mode)
        g = Sie(V, T, P.WL, P.EPS_METAL, tree_s_opt=100).setup()
        k, E = incidence(0.0, 0.0, "TM", 2)
        b = g.rhs_planewave(k, E)
        x, st = g.solve(b, restart=20, max_iterations=45, tolerance=1e-12, raise_on_noconv=False)
        assert st["iterations"] == 45
        xs.append(x)
        g.close()
    for x in xs[1:]:
        assert rel(x, xs[0]) < 1e-9, rel(x, xs[0])


def test_solve_converges_like_oracle(oracle_lib, gpu_lib):
    """A dielectric sphere converges to 1e-6; same iteration count, same currents.
    (s_opt = 500 keeps every pair in the near field: one level, no translation.)"""
    from specklesim_b200 import Sie, incidence
    V, T = P.sphere(2)
    o = oracle_lib.Oracle(V, T, P.WL, P.EPS_DIELECTRIC, tree_s_opt=500)
    o.tree()
    o.setup_fmm()
    g = Sie(V, T, P.WL, P.EPS_DIELECTRIC, tree_s_opt=500).setup()
    k, E = incidence(0.0, 0.0, "TM", 2)
    b = o.rhs(k, E)
    x_o, info = oracle_lib.zgmres(o.matvec, b, 50, 1e-6, 1000)
    x_g, st = g.solve(b, restart=50, max_iterations=1000, tolerance=1e-6)
    assert st["converged"] and info["converged"]
    assert abs(st["iterations"] - info["iterations"]) <= 1
    assert rel(x_g, x_o) < 1e-6
    r = b - o.matvec(x_g)
    assert np.linalg.norm(r) / np.linalg.norm(b) <= 1e-6
    g.close()


def test_farfield_matches_oracle(slab_pair):
    o, _, g = slab_pair
    x = P.random_x(o.N, seed=9)
    th = np.linspace(0.05, 1.4, 7)
    pts = 5.0 * np.stack([np.sin(th), 0 * th, np.cos(th)], axis=1)
    E1, H1, I1 = g.farfield(x, pts)
    E2, H2, I2 = o.field(x, pts)
    # random currents: the sums over edges cancel to ~1e-5 of their terms
    assert rel(E1, E2) < 1e-8 and rel(H1, H2) < 1e-8 and rel(I1, I2) < 1e-8


def test_dense_mode_matches_oracle_dense(oracle_lib, gpu_lib):
    from specklesim_b200 import Sie
    V, T = P.sphere(1)
    o = oracle_lib.Oracle(V, T, P.WL, P.EPS_METAL)
    Z = o.dense()
    g = Sie(V, T, P.WL, P.EPS_METAL, dense=True).setup()
    x = P.random_x(o.N, seed=3)
    assert rel(g.matvec(x), Z @ x) < 1e-10
    g.close()


def test_error_paths(gpu_lib):
    from specklesim_b200 import Sie, SieError
    from specklesim_b200 import _lib
    V, T = P.sphere(1)
    g = Sie(V, T, P.WL, P.EPS_METAL, tree_s_opt=20)
    with pytest.raises(SieError) as e:
        g.matvec(np.ones(g.n, complex))  # before set-up
    assert e.value.code == _lib.SIE_ERR_STATE
    g.setup()
    bad = np.ones(g.n, complex)
    bad[3] = np.nan
    with pytest.raises(SieError) as e:
        g.matvec(bad)
    assert e.value.code == _lib.SIE_ERR_NONFINITE
    with pytest.raises(SieError) as e:
        g.solve(np.ones(g.n, complex), restart=5, max_iterations=3, tolerance=1e-14)
    assert e.value.code == _lib.SIE_ERR_NOCONV
    x, st = g.solve(np.ones(g.n, complex), restart=5, max_iterations=3, tolerance=1e-14,
                    raise_on_noconv=False)
    assert not st["converged"] and st["iterations"] == 3
    g.close()
    T2 = T.copy()
    T2[0, 0] = 10 ** 6
    with pytest.raises(SieError) as e:
        Sie(V, T2, P.WL, P.EPS_METAL)
    assert e.value.code == _lib.SIE_ERR_MESH


def test_mixed_matvec_close_to_fp64(metal_pair):
    """The complex64 product stays within the FP32 rounding amplified by the cancellation
    of the K = 19 translations (~1e4 on these 0.75-lambda boxes, measured 4e-5)."""
    _, _, g = metal_pair
    x = P.random_x(g.n, seed=5)
    y64 = g.matvec(x)
    y32 = g.matvec(x, precision="mixed")
    assert rel(y32, y64) < 2e-4, rel(y32, y64)


def test_mixed_solve_matches_fp64_farfield(slab_pair):
    """FP64 flexible GMRES around FP32 inner GMRES reaches the FP64 tolerance on the true
    residual; its currents and far-field intensities agree with the plain FP64 solve."""
    from specklesim_b200 import incidence
    _, _, g = slab_pair
    k, E = incidence(0.0, 0.0, "TM", 2)
    b = g.rhs_planewave(k, E)
    x64, s64 = g.solve(b, restart=50, max_iterations=2000, tolerance=1e-8)
    xm, sm = g.solve(b, restart=10, max_iterations=60, tolerance=1e-8, precision="mixed",
                     inner_restart=30, inner_tolerance=1e-2)
    assert sm["converged"] and sm["backward_error_true"] <= 1e-8
    assert sm["inner_iterations"] > sm["iterations"]
    th = np.linspace(0.05, 1.4, 9)
    pts = 5.0 * np.stack([np.sin(th), 0 * th, np.cos(th)], axis=1)
    I64 = g.farfield(x64, pts)[2]
    Im = g.farfield(xm, pts)[2]
    assert rel(Im, I64) < 1e-5, rel(Im, I64)
    assert rel(xm, x64) < 1e-5, rel(xm, x64)


def test_later_small_context_keeps_earlier_context_working(gpu_lib):
    """Kernel launch limits are process-wide: setting up a small mesh after a large one
    must not break the large context's products."""
    from specklesim_b200 import Sie
    V, T = P.slab(cells=24, length_wl=6.0, seed=3)
    big = Sie(V, T, P.WL, P.EPS_METAL, tree_s_opt=100).setup()
    x = P.random_x(big.n, seed=2)
    y0 = big.matvec(x)
    Vs, Ts = P.sphere(1)
    small = Sie(Vs, Ts, P.WL, P.EPS_METAL, tree_s_opt=20).setup()
    small.matvec(P.random_x(small.n, seed=3))
    assert np.array_equal(big.matvec(x), y0)
    small.close()
    big.close()


@pytest.mark.parametrize("formulation,ngp", [("PMCHWT", 3), ("ICTF", 7), ("PMCHWT", 7)])
def test_other_formulations_and_rules(oracle_lib, gpu_lib, formulation, ngp):
    """PMCHWT (with the 12-point edge-adjacent Kt of edge_adjacent_tri) and the 7-point
    rule of the small-sphere configuration: blocks and matvec against the oracle."""
    from specklesim_b200 import Sie
    V, T = P.slab(cells=16, length_wl=4.0, seed=3)
    o = oracle_lib.Oracle(V, T, P.WL, P.EPS_METAL, formulation=formulation, ngp=ngp,
                          tree_s_opt=60, threads=8)
    o.tree()
    o.setup_fmm()
    g = Sie(V, T, P.WL, P.EPS_METAL, formulation=formulation, ngp=ngp, tree_s_opt=60).setup()
    rng = np.random.default_rng(1)
    m, n = _pairs(o, rng, 200)
    a, b = g.blocks(m, n), o.blocks(m, n)
    scale = np.abs(b).max(axis=1, keepdims=True)
    assert (np.abs(a - b) / scale).max() < 1e-9
    x = P.random_x(o.N, seed=6)
    assert rel(g.matvec(x), o.matvec(x)) < 1e-9
    g.close()


def test_dense_small_sphere_ngp7_solves_like_dense_oracle(oracle_lib, gpu_lib):
    """The small-sphere configuration in miniature: dense path (no MLFMM), 7-point rule,
    metal, GMRES to 1e-6 against a direct solve of the oracle's dense matrix."""
    from specklesim_b200 import Sie, incidence
    V, T = P.sphere(2)
    o = oracle_lib.Oracle(V, T, P.WL, P.EPS_METAL, ngp=7)
    Z = o.dense()
    k, E = incidence(0.0, 0.0, "TM", 2)
    b = o.rhs(k, E)
    x_direct = np.linalg.solve(Z, b)
    g = Sie(V, T, P.WL, P.EPS_METAL, ngp=7, dense=True).setup()
    x, st = g.solve(b, restart=50, max_iterations=2000, tolerance=1e-10, raise_on_noconv=False)
    assert st["backward_error_true"] < 1e-8
    assert rel(x, x_direct) < 1e-6, rel(x, x_direct)
    g.close()


def test_direct_dense_solve_matches_oracle(oracle_lib, gpu_lib):
    """Dense LU path (the reference's normal solver) against numpy on the oracle's matrix,
    two right-hand sides, the factors reused by a second call."""
    from specklesim_b200 import Sie, incidence
    V, T = P.sphere(2)
    o = oracle_lib.Oracle(V, T, P.WL, P.EPS_METAL, ngp=7)
    Z = o.dense()
    B = np.stack([o.rhs(*incidence(0.0, 0.0, "TM", 2)), o.rhs(*incidence(0.3, 0.4, "TE", 2))], axis=1)
    X = np.linalg.solve(Z, B)
    g = Sie(V, T, P.WL, P.EPS_METAL, ngp=7, dense=True).setup()
    # matrix entries agree to ~1e-12 (block tests); the solve scales that by cond(Z) ~ 1e3
    Xg = g.solve_direct(B)
    assert rel(Xg, X) < 1e-8, rel(Xg, X)
    x1 = g.solve_direct(B[:, 1])
    assert rel(x1, X[:, 1]) < 1e-8
    g.close()


def test_autotune_keeps_the_product(gpu_lib):
    """The autotuner only picks among variants that compute the same product."""
    from specklesim_b200 import Sie
    V, T = P.slab(cells=24, length_wl=6.0, seed=3)
    g = Sie(V, T, P.WL, P.EPS_METAL, tree_s_opt=100).setup()
    x = P.random_x(g.n, seed=11)
    y0 = g.matvec(x)
    before, after, modes = g.autotune("fp64")
    assert after <= before and 1 <= modes["sr"] <= 5 and 0 <= modes["overlap"] <= 3
    assert rel(g.matvec(x), y0) < 1e-13
    g.autotune("mixed")
    assert rel(g.matvec(x, precision="mixed"), y0) < 2e-4
    g.close()

"""Parity at the bench's own configuration (needs a B200, a few minutes): the 10 lambda
rough metal slab (seed 0, 19,456 triangles, 29,184 RWG edges) with the reference's
tree_s_opt = 250 (0.625 lambda leaf boxes, levels 2..4), against the oracle built the same
way, and the MLFMM products against the dense product of the same fill.

Tolerances: the K = 19 translation on 0.625 lambda boxes loses digits to cancellation
(sum of (2n + 1) h_n(2 k d) terms, kappa ~ 1e6), so the two implementations, whose h2 and
summation orders differ in the last bits, agree to kappa * 1e-16 rather than to 1e-12.

The dense comparison documents why the bench's converged solve is a direct one: with
K = 19 on every level (the reference's setting, lib_sie_mlfmm.f90:694-699) the product is
several per cent off the dense one, because the 2.5 lambda boxes of level 2 need K of
about 30; with 34 / 23 / 19 on levels 2 / 3 / 4 it is accurate to ~1e-4."""
import numpy as np
import pytest

from tests import problems as P

pytestmark = pytest.mark.gpu

LEVEL_K = {2: 34, 3: 23, 4: 19}


def _rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.fixture(scope="module")
def slab10(oracle_lib, gpu_lib):
    from specklesim_b200 import Sie, mesh
    V, T = mesh.slab_config(10.0, P.WL, 0.5, 1.0, 0, cells=64, thickness_wl=1.0)
    assert T.shape[0] == 19456
    o = oracle_lib.Oracle(V, T, P.WL, P.EPS_METAL, tree_s_opt=250, threads=0)
    info = o.tree()
    o.setup_fmm()
    g = Sie(V, T, P.WL, P.EPS_METAL, tree_s_opt=250).setup()
    yield V, T, o, info, g
    g.close()
    o.close()


def test_mesh_tree_and_near_entries(slab10):
    V, T, o, info, g = slab10
    assert g.n_edges == o.M == 29184
    assert (g.l_min, g.l_max) == (info["l_min"], info["l_max"]) == (2, 4)
    e_o, c_o = o.edges()
    e_g, c_g = g.edges()
    assert np.array_equal(e_o, e_g) and np.array_equal(c_o, c_g)
    _, _, leaf = g.tree()
    assert np.array_equal(leaf, info["leaf"])
    ia, ja, v = o.near_csr()
    assert g.near_nnz == len(ja)
    rows = np.arange(0, o.M, 97)
    mm = np.concatenate([np.full(ia[r + 1] - ia[r], r) for r in rows])
    nn = np.concatenate([ja[ia[r]:ia[r + 1]] for r in rows])
    vv = np.concatenate([v[ia[r]:ia[r + 1]] for r in rows])
    got = g.near_entries(mm, nn)
    scale = np.abs(vv).max(axis=1, keepdims=True)
    assert (np.abs(got - vv) / scale).max() < 1e-9


def test_products_match_oracle(slab10, oracle_lib):
    from specklesim_b200 import Sie
    V, T, o, info, g = slab10
    x = P.random_x(g.n, seed=3)
    err19 = _rel(g.matvec(x), o.matvec(x))
    print(f"K = 19 product, GPU vs oracle: {err19:.3e}")
    assert err19 < 1e-8
    ol = oracle_lib.Oracle(V, T, P.WL, P.EPS_METAL, tree_s_opt=250, threads=0)
    ol.tree()
    ol.set_level_truncation(LEVEL_K)
    ol.setup_fmm()
    gl = Sie(V, T, P.WL, P.EPS_METAL, tree_s_opt=250, level_truncation=LEVEL_K).setup()
    errl = _rel(gl.matvec(x), ol.matvec(x))
    print(f"per-level K product, GPU vs oracle: {errl:.3e}")
    assert errl < 1e-8
    gl.close()
    ol.close()


def test_budgeted_gmres_matches_oracle_zgmres(slab10, oracle_lib):
    from specklesim_b200 import incidence
    V, T, o, info, g = slab10
    k, E = incidence(0.0, 0.0, "TM", 2)
    b = g.rhs_planewave(k, E)
    assert _rel(b, o.rhs(k, E)) < 1e-12
    x_g, st = g.solve(b, restart=20, max_iterations=20, tolerance=1e-12, raise_on_noconv=False)
    x_o, info_o = oracle_lib.zgmres(o.matvec, b, 20, 1e-12, 20)
    print(f"20 GMRES steps: GPU {st['backward_error_true']:.6e}, oracle {info_o['be']:.6e}, "
          f"iterates {_rel(x_g, x_o):.3e}")
    assert abs(st["backward_error_true"] - info_o["be"]) < 1e-6 * info_o["be"]
    assert _rel(x_g, x_o) < 1e-6


def test_mlfmm_products_against_the_dense_product(slab10):
    from specklesim_b200 import Sie
    V, T, o, info, g = slab10
    d = Sie(V, T, P.WL, P.EPS_METAL, dense=True).setup()
    gl = Sie(V, T, P.WL, P.EPS_METAL, tree_s_opt=250, level_truncation=LEVEL_K).setup()
    errs19, errsl = [], []
    for seed in (5, 6):
        x = P.random_x(g.n, seed=seed)
        yd = d.matvec(x)
        errs19.append(_rel(g.matvec(x), yd))
        errsl.append(_rel(gl.matvec(x), yd))
    print(f"MLFMM vs dense: K = 19 {max(errs19):.3e}, per-level K {max(errsl):.3e}")
    assert min(errs19) > 1e-2          # measured 6.7e-2
    assert max(errsl) < 1e-3
    gl.close()
    d.close()

"""The oracle's local Lagrange interpolation between k-space samplings (the level-dependent
truncation path of the SS and RR passes, lib_sie_mlfmm.f90:268-610), checked on CPU.

The reference has no test of this routine and cannot be run here, so these checks pin the
restatement by its mathematics: it reproduces samples when both samplings are the same,
it is linear, and it reconstructs band-limited far-field patterns, including the constant
Cartesian field, which is the case where the rows reflected through the poles carry the
result (a reflection with the wrong sign or phi shift would give O(1) errors there).

The second half checks the whole product with a truncation number per level against the
product with K = 19 on every level: interpolation up in SS, anterpolation (the transpose)
down in RR, and the khat x f rotation at the -z pole in the receive."""
import numpy as np
import pytest


def _grid(oracle_lib, K):
    """Directions, theta-hat and phi-hat of the K sampling (theta-major, the order of the
    reference's Khat_and_TRF_ExtendedK), without the two poles."""
    x, _ = oracle_lib.gauss_legendre(K)
    T, P = np.meshgrid(np.arccos(x), np.arange(2 * K) * np.pi / K, indexing="ij")
    T, P = T.ravel(), P.ravel()
    kh = np.stack([np.sin(T) * np.cos(P), np.sin(T) * np.sin(P), np.cos(T)], 1)
    tth = np.stack([np.cos(T) * np.cos(P), np.cos(T) * np.sin(P), -np.sin(T)], 1)
    tph = np.stack([-np.sin(P), np.cos(P), 0 * P], 1)
    return kh, tth, tph


def _pattern(oracle_lib, K, V):
    """theta and phi components of the tangential field V(khat) on the K sampling; the
    +z and -z poles hold the Cartesian x and y components."""
    kh, tth, tph = _grid(oracle_lib, K)
    v = V(kh)
    vp = V(np.array([[0.0, 0.0, 1.0], [0.0, 0.0, -1.0]]))
    fa = np.concatenate([np.einsum("ij,ij->i", tth, v), vp[:, 0]])
    fb = np.concatenate([np.einsum("ij,ij->i", tph, v), vp[:, 1]])
    return fa, fb


def _sources(seed):
    """Far field of six point currents in a box of side 0.5 lambda (k r up to 2.7)."""
    rng = np.random.default_rng(seed)
    rs = rng.uniform(-0.25, 0.25, (6, 3))
    js = rng.standard_normal((6, 3)) + 1j * rng.standard_normal((6, 3))
    k = 2 * np.pi
    return lambda kh: np.exp(1j * k * kh @ rs.T) @ js


def _constant(kh):
    return np.tile(np.array([1.0, 0.5 - 0.2j, 0.3]), (len(kh), 1))


@pytest.mark.parametrize("K", [8, 12, 19])
def test_same_sampling_reproduces_the_samples(oracle_lib, K):
    q = 2 * K * K + 2
    rng = np.random.default_rng(K)
    fa = rng.standard_normal(q) + 1j * rng.standard_normal(q)
    fb = rng.standard_normal(q) + 1j * rng.standard_normal(q)
    ga, gb = oracle_lib.lagrange_interp(3, K, K, fa, fb)
    assert np.abs(ga - fa).max() < 1e-13 and np.abs(gb - fb).max() < 1e-13
    # the poles are copied, not interpolated
    assert np.array_equal(ga[-2:], fa[-2:]) and np.array_equal(gb[-2:], fb[-2:])


def test_interpolation_is_linear(oracle_lib):
    f1 = _pattern(oracle_lib, 12, _sources(1))
    f2 = _pattern(oracle_lib, 12, _sources(2))
    a, b = 0.7 - 0.4j, -1.3 + 0.2j
    g1 = oracle_lib.lagrange_interp(3, 12, 19, *f1)
    g2 = oracle_lib.lagrange_interp(3, 12, 19, *f2)
    g = oracle_lib.lagrange_interp(3, 12, 19, a * f1[0] + b * f2[0], a * f1[1] + b * f2[1])
    for c in range(2):
        ref = a * g1[c] + b * g2[c]
        assert np.abs(g[c] - ref).max() <= 1e-13 * np.abs(ref).max()


# (from K, to K, bound): measured errors are 4.5e-4, 2.7e-5 and 4.8e-4 for the sources,
# 1.8e-6, 1.1e-7 and 2.2e-6 for the constant field
@pytest.mark.parametrize("km,kn,bound_src,bound_const", [(12, 19, 1e-3, 1e-5), (19, 12, 1e-4, 1e-6),
                                                         (12, 24, 1e-3, 1e-5)])
def test_band_limited_patterns_are_reconstructed(oracle_lib, km, kn, bound_src, bound_const):
    for V, bound in ((_sources(3), bound_src), (_constant, bound_const)):
        ga, gb = oracle_lib.lagrange_interp(3, km, kn, *_pattern(oracle_lib, km, V))
        ea, eb = _pattern(oracle_lib, kn, V)
        scale = max(np.abs(ea).max(), np.abs(eb).max())
        err = max(np.abs(ga - ea).max(), np.abs(gb - eb).max()) / scale
        assert err < bound, (km, kn, err)


def test_rows_next_to_the_poles(oracle_lib):
    """The first and last theta rows of the target sampling lie between the outermost
    source nodes and the poles, so their stencils reach through the poles into the
    reflected rows.  For the constant Cartesian field both components there depend on phi
    at order one; the interpolated values must still match to the bulk accuracy."""
    km, kn = 12, 19
    ga, gb = oracle_lib.lagrange_interp(3, km, kn, *_pattern(oracle_lib, km, _constant))
    ea, eb = _pattern(oracle_lib, kn, _constant)
    rows = np.r_[0:2 * kn, (kn - 1) * 2 * kn:kn * 2 * kn]
    assert np.abs(ea[rows]).max() > 0.5
    assert max(np.abs(ga[rows] - ea[rows]).max(), np.abs(gb[rows] - eb[rows]).max()) < 1e-5


# ---------------------------------------------------------------------------
# The product with a truncation number per level (SS interpolation up, RR anterpolation
# down) against the product with K = 19 on every level.

def _slab_oracle(oracle_lib, k_by_level=None, K=19):
    from tests import problems as P
    V, T = P.slab(cells=16, length_wl=4.0, seed=3)
    o = oracle_lib.Oracle(V, T, P.WL, P.EPS_DIELECTRIC, tree_s_opt=60, threads=8, truncation_number=K)
    info = o.tree()
    if k_by_level:
        o.set_level_truncation(k_by_level)
    o.setup_fmm()
    return o, info


@pytest.fixture(scope="module")
def slab_k19(oracle_lib):
    from tests import problems as P
    o, info = _slab_oracle(oracle_lib)
    assert (info["l_min"], info["l_max"]) == (2, 3)  # one SS and one RR step between the levels
    x = P.random_x(o.N, seed=1)
    return x, o.matvec(x)


def _rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def test_equal_level_truncation_is_the_uniform_product(oracle_lib, slab_k19):
    x, y19 = slab_k19
    o, _ = _slab_oracle(oracle_lib, {2: 19, 3: 19})
    assert np.array_equal(o.matvec(x), y19)


# measured: 1.7e-3, 8.1e-4 and 4.5e-4; K = 12 and 14 on every level give 4.2e-3 and 1.1e-3
@pytest.mark.parametrize("k_by_level,bound", [({3: 12, 2: 14}, 3e-3), ({3: 14, 2: 16}, 1.5e-3),
                                              ({3: 16, 2: 19}, 1e-3)])
def test_level_truncation_product(oracle_lib, slab_k19, k_by_level, bound):
    x, y19 = slab_k19
    o, _ = _slab_oracle(oracle_lib, k_by_level)
    assert _rel(o.matvec(x), y19) < bound


def test_larger_upper_truncation_helps(oracle_lib, slab_k19):
    """Raising K on the upper level only (interpolated up, anterpolated down) makes the
    product more accurate than the leaf's K on every level."""
    x, y19 = slab_k19
    err_uniform = _rel(_slab_oracle(oracle_lib, K=12)[0].matvec(x), y19)
    err_level = _rel(_slab_oracle(oracle_lib, {3: 12, 2: 14})[0].matvec(x), y19)
    assert err_level < 0.6 * err_uniform


def test_truncation_growing_toward_the_leaf_is_refused(oracle_lib):
    with pytest.raises(ValueError):
        _slab_oracle(oracle_lib, {3: 16, 2: 14})

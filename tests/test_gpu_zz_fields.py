"""Fields inside the body and near-field maps through the surface (needs a B200):
sie_field_interior against the oracle's restatement of
Integration_scattered_field_tri_within_medium (src/lib_sie_tri_calculation_mod.f90:
2829-2877), and Sie.near_field against the same composition of the oracle's routines."""
import numpy as np
import pytest

from tests import problems as P

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.linalg.norm(np.ravel(a - b)) / np.linalg.norm(np.ravel(b))


@pytest.fixture(scope="module")
def slab_pair(oracle_lib, gpu_lib):
    from specklesim_b200 import Sie
    V, T = P.slab(cells=24, length_wl=6.0, seed=3)
    o = oracle_lib.Oracle(V, T, P.WL, P.EPS_DIELECTRIC, tree_s_opt=100, threads=8)
    g = Sie(V, T, P.WL, P.EPS_DIELECTRIC, tree_s_opt=100).setup()
    yield o, None, g
    g.close()
    o.close()


@pytest.fixture(scope="module")
def metal_pair(oracle_lib, gpu_lib):
    from specklesim_b200 import Sie
    V, T = P.slab(cells=24, length_wl=6.0, seed=3)
    o = oracle_lib.Oracle(V, T, P.WL, P.EPS_METAL, tree_s_opt=100, threads=8)
    g = Sie(V, T, P.WL, P.EPS_METAL, tree_s_opt=100).setup()
    yield o, None, g
    g.close()
    o.close()


@pytest.mark.parametrize("which,eps_r", [("slab_pair", None), ("metal_pair", None), ("slab_pair", 4.0 - 0.5j)])
def test_interior_field_matches_oracle(request, which, eps_r):
    """sie_field_interior (two passes of the exterior field kernel) against the oracle's
    restatement of Integration_scattered_field_tri_within_medium
    (lib_sie_tri_calculation_mod.f90:2829-2877), at points spread through the slab's
    bounding box, in the body's medium and in another one."""
    o, _, g = request.getfixturevalue(which)
    x = P.random_x(o.N, seed=11)
    rng = np.random.default_rng(12)
    pts = rng.uniform(-1.5, 1.5, size=(12, 3)) * P.WL
    pts[:, 2] = rng.uniform(-0.4, 0.4, size=12) * P.WL
    er = (P.EPS_DIELECTRIC if which == "slab_pair" else P.EPS_METAL) if eps_r is None else eps_r
    E1, H1 = g.field_interior(x, pts, eps_r)
    E2, H2 = o.field_interior(x, pts, er)
    assert rel(E1, E2) < 1e-8 and rel(H1, H2) < 1e-8


def test_near_field_map_matches_oracle(oracle_lib, gpu_lib):
    """A near-field map through the surface of the small sphere (the plane-wave branch of
    lib_sie_tri_observation_field_calculation, lib_sie_tri_solver_normal.f90:385-420):
    interior points from the interior routine, exterior ones scattered plus incident
    field, against the same composition of the oracle's routines."""
    from specklesim_b200 import Sie, incidence
    V, T = P.sphere(2)
    o = oracle_lib.Oracle(V, T, P.WL, P.EPS_DIELECTRIC, threads=8)
    g = Sie(V, T, P.WL, P.EPS_DIELECTRIC, dense=True).setup()
    k, E = incidence(0.0, 0.0, "TM", 2)
    x = P.random_x(o.N, seed=5)
    u = np.linspace(-1.0, 1.0, 9) * P.WL
    pts = np.stack(np.meshgrid(u, [0.0], u, indexing="ij"), -1).reshape(-1, 3) + np.array([0.013, 0, 0.007]) * P.WL
    r = np.linalg.norm(pts, axis=1)
    inside = r < 0.45 * P.WL
    keep = inside | (r > 0.55 * P.WL)  # away from the surface itself
    pts, inside = pts[keep], inside[keep]
    Eg, Hg = g.near_field(x, pts, inside, k, E)
    Eo, Ho = np.zeros_like(Eg), np.zeros_like(Hg)
    Eo[inside], Ho[inside] = o.field_interior(x, pts[inside], P.EPS_DIELECTRIC)
    Es, Hs, _ = o.field(x, pts[~inside])
    k1 = 2 * np.pi / P.WL
    omega = 2 * np.pi * float(np.float32(2.99792458e8)) / P.WL
    Einc = np.asarray(E)[None, :] * np.exp(-1j * k1 * (pts[~inside] @ np.asarray(k)))[:, None]
    Hinc = np.cross(k1 * np.asarray(k)[None, :], Einc) / (float(np.float32(1.2566370614e-6)) * omega)
    Eo[~inside], Ho[~inside] = Es + Einc, Hs + Hinc
    assert inside.sum() >= 4 and (~inside).sum() >= 20
    assert rel(Eg, Eo) < 1e-8 and rel(Hg, Ho) < 1e-8
    g.close()
    o.close()

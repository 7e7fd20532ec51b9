"""Host logic of Sie.near_field (the plane-wave branch of the reference's
lib_sie_tri_observation_field_calculation, src/lib_sie_tri_solver_normal.f90:385-420), on
the CPU: the library's two field entry points are replaced by the oracle's routines, so
the test checks the composition (which points take which routine, the 1e-20 zeroing of
interior components, the incident plane wave added outside) and not the kernels."""
import numpy as np

from specklesim_b200 import Sie
from specklesim_b200._lib import SieConfig
from tests import problems as P


def _host_only(o, eps_r2):
    """A Sie whose farfield / field_interior are the oracle's (no device)."""
    g = Sie.__new__(Sie)
    cfg = SieConfig()
    cfg.lambda_ = P.WL
    cfg.eps_r1_re, cfg.eps_r1_im = 1.0, 0.0
    cfg.eps_r2_re, cfg.eps_r2_im = eps_r2.real, eps_r2.imag
    g.cfg = cfg
    g.farfield = lambda x, pts: o.field(x, pts)
    g.field_interior = lambda x, pts, eps_r=None: o.field_interior(x, pts, eps_r2 if eps_r is None else eps_r)
    return g


def test_near_field_map_composition(oracle_lib):
    V, T = P.sphere(1)
    eps = complex(P.EPS_DIELECTRIC)
    o = oracle_lib.Oracle(V, T, P.WL, eps, threads=4)
    g = _host_only(o, eps)
    x = P.random_x(o.N, seed=6)
    u = np.linspace(-1.0, 1.0, 7) * P.WL
    pts = np.stack(np.meshgrid(u, u, [0.011 * P.WL], indexing="ij"), -1).reshape(-1, 3)
    inside = np.linalg.norm(pts, axis=1) < 0.4 * P.WL
    k = np.array([0.0, 0.0, -1.0])
    E0 = np.array([1.0, 0.0, 0.0])
    E, H = g.near_field(x, pts, inside, k, E0)
    Ei, Hi = o.field_interior(x, pts[inside], eps)
    assert np.array_equal(E[inside], Ei) and np.array_equal(H[inside], Hi)
    Es, Hs, _ = o.field(x, pts[~inside])
    k1 = 2 * np.pi / P.WL
    omega = 2 * np.pi * float(np.float32(2.99792458e8)) / P.WL
    Einc = E0[None, :] * np.exp(-1j * k1 * (pts[~inside] @ k))[:, None]
    Hinc = np.cross(k1 * k[None, :], Einc) / (float(np.float32(1.2566370614e-6)) * omega)
    assert np.allclose(E[~inside], Es + Einc, rtol=1e-14, atol=0)
    assert np.allclose(H[~inside], Hs + Hinc, rtol=1e-14, atol=0)
    # scattered field only without an incident wave
    E2, _ = g.near_field(x, pts, inside)
    assert np.array_equal(E2[~inside], Es)
    o.close()


def test_near_field_zeroes_vanishing_interior_components(oracle_lib):
    """A component of the interior E below 1e-20 is set to zero together with the same
    component of H (lib_sie_tri_solver_normal.f90:391-405)."""
    V, T = P.sphere(1)
    eps = complex(P.EPS_DIELECTRIC)
    o = oracle_lib.Oracle(V, T, P.WL, eps, threads=4)
    g = _host_only(o, eps)
    Ein = np.array([[1e-25, 1.0, 1e-21j], [2.0, 1e-19, 0.0]])
    Hin = np.array([[5.0, 6.0, 7.0], [8.0, 9.0, 10.0]], complex)
    g.field_interior = lambda x, pts, eps_r=None: (Ein.copy(), Hin.copy())
    E, H = g.near_field(np.zeros(o.N, complex), np.zeros((2, 3)), np.array([True, True]))
    assert np.array_equal(E, [[0, 1.0, 0], [2.0, 1e-19, 0]])
    assert np.array_equal(H, [[0, 6.0, 0], [8.0, 9.0, 0]])
    o.close()


def test_default_media_from_the_mesh(oracle_lib):
    """Without an inside mask, the map's medium-2 points are those inside the closed mesh
    (generalised winding number): the same result as the explicit mask."""
    V, T = P.sphere(1)
    eps = complex(P.EPS_DIELECTRIC)
    o = oracle_lib.Oracle(V, T, P.WL, eps, threads=4)
    g = _host_only(o, eps)
    g.verts, g.tris = np.asarray(V), np.asarray(T)
    x = P.random_x(o.N, seed=7)
    d = np.random.default_rng(3).normal(size=(20, 3))
    d /= np.linalg.norm(d, axis=1)[:, None]
    pts = np.concatenate([d * 0.3 * P.WL, d * 0.8 * P.WL])
    mask = np.arange(40) < 20
    E1, H1 = g.near_field(x, pts)
    E2, H2 = g.near_field(x, pts, mask)
    assert np.array_equal(E1, E2) and np.array_equal(H1, H2)
    o.close()


def test_winding_number_of_closed_meshes():
    from specklesim_b200 import mesh
    for V, T in (P.sphere(2), P.slab(cells=10, length_wl=2.0, seed=3)):
        c = np.asarray(V).mean(axis=0)
        far = c + np.array([0.0, 0.0, 10.0 * P.WL])
        w = mesh.winding_number(V, T, np.stack([c, far]))
        assert abs(abs(w[0]) - 1) < 1e-9 and abs(w[1]) < 1e-9

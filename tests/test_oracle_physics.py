"""Physics pin of the oracle: the ICTF and PMCHWT solutions for the small-sphere
configuration (radius 0.5 lambda, icosphere subdivision 3: 1280 triangles, 1920 RWG
edges) against the Mie series (intensity L2 errors 0.6-1.1 %, bound 5 %).  The reference has no golden vectors for its SIE blocks, so this and the
Hänninen probes are what pin the restated formulation.

Mie series: Bohren & Huffman, "Absorption and Scattering of Light by Small Particles"
(1983), eqs. 4.53 (a_n, b_n with Riccati-Bessel functions) and 4.74 (S1, S2 with the
angular functions pi_n, tau_n), in the exp(-i w t) convention; the SIE code uses
exp(+i w t), so the refractive index is conj(sqrt(eps))."""
import numpy as np
import pytest
from scipy.special import spherical_jn, spherical_yn

from tests import problems as P


def mie_s12(m, x, mu):
    nmax = int(x + 4 * x ** (1 / 3) + 2) + 10
    n = np.arange(1, nmax + 1)
    mx = m * x

    def psi(z):
        return z * spherical_jn(n, z)

    def dpsi(z):
        return spherical_jn(n, z) + z * spherical_jn(n, z, derivative=True)

    def xi(z):
        return z * (spherical_jn(n, z) + 1j * spherical_yn(n, z))

    def dxi(z):
        h = spherical_jn(n, z) + 1j * spherical_yn(n, z)
        dh = spherical_jn(n, z, derivative=True) + 1j * spherical_yn(n, z, derivative=True)
        return h + z * dh

    an = (m * psi(mx) * dpsi(x) - psi(x) * dpsi(mx)) / (m * psi(mx) * dxi(x) - xi(x) * dpsi(mx))
    bn = (psi(mx) * dpsi(x) - m * psi(x) * dpsi(mx)) / (psi(mx) * dxi(x) - m * xi(x) * dpsi(mx))
    c = (2 * n + 1) / (n * (n + 1))
    S1 = np.zeros(len(mu), complex)
    S2 = np.zeros(len(mu), complex)
    for i, u in enumerate(mu):
        pi = np.zeros(nmax + 1)
        tau = np.zeros(nmax + 1)
        pi[1], tau[1] = 1.0, u
        if nmax > 1:
            pi[2] = 3 * u
            tau[2] = 2 * u * pi[2] - 3 * pi[1]
        for j in range(3, nmax + 1):
            pi[j] = (2 * j - 1) / (j - 1) * u * pi[j - 1] - j / (j - 1) * pi[j - 2]
            tau[j] = j * u * pi[j] - (j + 1) * pi[j - 1]
        S1[i] = np.sum(c * (an * pi[1:] + bn * tau[1:]))
        S2[i] = np.sum(c * (an * tau[1:] + bn * pi[1:]))
    return S1, S2


_SOLVED = {}
K_IN = np.array([0.0, 0.0, -1.0])
E_IN = np.array([1.0, 0.0, 0.0])


def solved_sphere(oracle_lib, eps, formulation):
    """Oracle context and dense-LU currents of the small sphere under the x-polarised
    plane wave along -z, made once per (eps, formulation) for the tests below."""
    key = (eps, formulation)
    if key not in _SOLVED:
        V, T = P.sphere(3)
        o = oracle_lib.Oracle(V, T, P.WL, eps, formulation=formulation, threads=16)
        x = np.linalg.solve(o.dense(), o.rhs(K_IN, E_IN))
        _SOLVED[key] = (o, x)
    return _SOLVED[key]


@pytest.mark.parametrize("formulation", ["ICTF", "PMCHWT"])
@pytest.mark.parametrize("eps", [P.EPS_DIELECTRIC, P.EPS_METAL])
def test_small_sphere_matches_mie(oracle_lib, eps, formulation):
    o, x = solved_sphere(oracle_lib, eps, formulation)
    k = 2 * np.pi / P.WL
    a = 0.5 * P.WL
    R = 5.0
    th = np.linspace(0.2, np.pi - 0.2, 9)
    I_sie, I_mie = [], []
    for phi in (0.0, np.pi / 2):
        pts = R * np.stack([np.sin(th) * np.cos(phi), np.sin(th) * np.sin(phi), np.cos(th)], 1)
        E, _, _ = o.field(x, pts)
        rh = pts / R
        Er = np.einsum("ij,ij->i", E, rh)
        I_sie.append((np.sum(np.abs(E) ** 2, 1) - np.abs(Er) ** 2) * R ** 2)
        S1, S2 = mie_s12(np.sqrt(np.conj(eps)), k * a, np.cos(np.pi - th))
        I_mie.append((np.abs(S2) ** 2 * np.cos(phi) ** 2 + np.abs(S1) ** 2 * np.sin(phi) ** 2) / k ** 2)
    I_sie, I_mie = np.concatenate(I_sie), np.concatenate(I_mie)
    err = np.linalg.norm(I_sie - I_mie) / np.linalg.norm(I_mie)
    assert err < 0.05, err


@pytest.mark.parametrize("formulation", ["ICTF", "PMCHWT"])
@pytest.mark.parametrize("eps,bound", [(P.EPS_DIELECTRIC, 0.01), (P.EPS_METAL, 0.08)])
def test_extinction_theorem_inside_the_sphere(oracle_lib, eps, formulation, bound):
    """Extinction theorem: inside the body, the medium-1 field radiated by the exterior
    equivalent currents cancels the incident field.  Checked on H, which
    Integration_scattered_field_tri (lib_sie_tri_calculation_mod.f90:2782-2825) evaluates
    with every term; its E drops the scalar-potential term (the "*0" at :2815), which
    leaves only the far-zone transverse field right (the Mie test's quantity).
    H_inc = k_hat x E_inc / (mu_1 c0) with the reference's binary32 constants
    (incident_field_tri_general, :939-1002).  40 random directions at radii 0.1, 0.25
    and 0.35 lambda of the 0.5 lambda sphere.  Residuals are 0.2-0.7 % for the
    dielectric and 2-6 % for the metal, whose surface fields are strong; both shrink
    with mesh refinement (icosphere subdivision 2 gives 2 % and up to 97 %)."""
    o, x = solved_sphere(oracle_lib, eps, formulation)
    k1 = 2 * np.pi / P.WL
    mu0c0 = float(np.float32(1.2566370614e-6)) * float(np.float32(2.99792458e8))
    d = np.random.default_rng(0).normal(size=(40, 3))
    d /= np.linalg.norm(d, axis=1)[:, None]
    for r in (0.1, 0.25, 0.35):
        pts = d * r * P.WL
        _, Hs, _ = o.field(x, pts)
        Ei = E_IN[None, :] * np.exp(-1j * k1 * pts @ K_IN)[:, None]
        Hi = np.cross(K_IN, Ei) / mu0c0
        err = np.linalg.norm(Hs + Hi) / np.linalg.norm(Hi)
        assert err < bound, (r, err)


def mie_internal(m, x, k, pts):
    """The field inside the sphere (Bohren & Huffman eqs. 4.50 and 4.52, equal
    permeabilities): E1 = sum_n E_n (c_n M_o1n - i d_n N_e1n) with spherical Bessel radial
    functions of m k r, E_n = i^n (2n + 1) / (n (n + 1)), for their x-polarised unit wave
    along +z in the exp(-i w t) convention; pts (n, 3) in their frame."""
    nmax = int(x + 4 * x ** (1 / 3) + 2) + 10
    n = np.arange(1, nmax + 1)
    j = spherical_jn(n, x)
    h = j + 1j * spherical_yn(n, x)
    dxh = h + x * (spherical_jn(n, x, derivative=True) + 1j * spherical_yn(n, x, derivative=True))
    dxj = j + x * spherical_jn(n, x, derivative=True)
    mx = m * x
    jm = spherical_jn(n, mx)
    dmj = jm + mx * spherical_jn(n, mx, derivative=True)
    cn = (j * dxh - h * dxj) / (jm * dxh - h * dmj)
    dn = (m * j * dxh - m * h * dxj) / (m * m * jm * dxh - h * dmj)
    En = 1j ** n * (2 * n + 1) / (n * (n + 1))
    out = []
    for p in pts:
        r = np.linalg.norm(p)
        th, ph = np.arccos(p[2] / r), np.arctan2(p[1], p[0])
        u = np.cos(th)
        pi = np.zeros(nmax + 1)
        tau = np.zeros(nmax + 1)
        pi[1], tau[1] = 1.0, u
        pi[2] = 3 * u
        tau[2] = 2 * u * pi[2] - 3 * pi[1]
        for i in range(3, nmax + 1):
            pi[i] = (2 * i - 1) / (i - 1) * u * pi[i - 1] - i / (i - 1) * pi[i - 2]
            tau[i] = i * u * pi[i] - (i + 1) * pi[i - 1]
        pi, tau = pi[1:], tau[1:]
        rho = m * k * r
        z = spherical_jn(n, rho)
        dz = (z + rho * spherical_jn(n, rho, derivative=True)) / rho  # [rho z_n]' / rho
        Er = np.sum(En * -1j * dn * np.cos(ph) * n * (n + 1) * np.sin(th) * pi * z / rho)
        Et = np.sum(En * (cn * np.cos(ph) * pi * z - 1j * dn * np.cos(ph) * tau * dz))
        Ep = np.sum(En * (-cn * np.sin(ph) * tau * z + 1j * dn * np.sin(ph) * pi * dz))
        er = np.array([np.sin(th) * np.cos(ph), np.sin(th) * np.sin(ph), np.cos(th)])
        et = np.array([np.cos(th) * np.cos(ph), np.cos(th) * np.sin(ph), -np.sin(th)])
        ep = np.array([-np.sin(ph), np.cos(ph), 0.0])
        out.append(Er * er + Et * et + Ep * ep)
    return np.array(out)


@pytest.mark.parametrize("formulation", ["ICTF", "PMCHWT"])
def test_interior_field_matches_mie(oracle_lib, formulation):
    """Integration_scattered_field_tri_within_medium (lib_sie_tri_calculation_mod.f90:
    2829-2877) inside the dielectric sphere against the Mie internal field, amplitude and
    phase, at 12 random directions on radii 0.1-0.4 lambda (radius 0.5 lambda).  The SIE
    wave travels along -z in exp(+i w t): the Mie field at the point mirrored in z, its z
    component negated, complex-conjugated, with m = conj(sqrt(eps)).  Measured 0.6-1.1 %
    (ICTF) and 0.55-0.9 % (PMCHWT); at the centre the field is d_1 E0 x_hat (0.6 %)."""
    eps = P.EPS_DIELECTRIC
    o, x = solved_sphere(oracle_lib, eps, formulation)
    k = 2 * np.pi / P.WL
    a = 0.5 * P.WL
    m = np.sqrt(np.conj(eps))
    flip = np.array([1.0, 1.0, -1.0])
    d = np.random.default_rng(3).normal(size=(12, 3))
    d /= np.linalg.norm(d, axis=1)[:, None]
    for r in (0.1, 0.2, 0.3, 0.4):
        pts = d * r * P.WL
        E, _ = o.field_interior(x, pts, eps)
        ref = np.conj(mie_internal(m, k * a, k, pts * flip) * flip)
        err = np.linalg.norm(E - ref) / np.linalg.norm(ref)
        assert err < 0.02, (r, err)
    E0, _ = o.field_interior(x, np.zeros((1, 3)), eps)
    ref0 = np.conj(mie_internal(m, k * a, k, np.array([[0.0, 0.0, 1e-9 * P.WL]]))[0])
    assert np.linalg.norm(E0[0] - ref0) / np.linalg.norm(ref0) < 0.02


@pytest.mark.parametrize("formulation", ["ICTF", "PMCHWT"])
def test_interior_representation_vanishes_outside(oracle_lib, formulation):
    """Extinction theorem of the interior problem: the medium-2 field of the negated
    currents, which is the total field inside, vanishes outside the body.  Dielectric
    sphere, 40 random directions at 0.7, 0.85 and 1.0 lambda from the centre (radius
    0.5 lambda), relative to the incident field: measured 0.4-0.5 % (ICTF) and
    0.08-0.11 % (PMCHWT)."""
    eps = P.EPS_DIELECTRIC
    o, x = solved_sphere(oracle_lib, eps, formulation)
    d = np.random.default_rng(1).normal(size=(40, 3))
    d /= np.linalg.norm(d, axis=1)[:, None]
    for r in (0.7, 0.85, 1.0):
        E, H = o.field_interior(x, d * r * P.WL, eps)
        err = np.sqrt(np.mean(np.sum(np.abs(E) ** 2, axis=1)))  # |E_inc| = 1
        assert err < 0.01, (r, err)


@pytest.mark.parametrize("eps", [P.EPS_DIELECTRIC, P.EPS_METAL])
def test_interior_field_as_two_exterior_passes(oracle_lib, eps):
    """The library evaluates the interior field with its exterior field kernel run twice,
    in the interior medium: (i) on the negated currents with mu_0, eps_2 = eps_0 eps_r and
    km = k0 sqrt(eps_r), which gives H and E without its scalar-potential term; (ii) on
    the currents (J, M) = (0, -J / eps_2) with permeability 1 and permittivity 0, whose H
    is that term.  The decomposition reproduces the restated routine to rounding."""
    o, x = solved_sphere(oracle_lib, eps, "ICTF")
    eps0 = float(np.float32(8.854187817e-12))
    mu0 = float(np.float32(1.2566370614e-6))
    M = x.size // 2
    km = 2 * np.pi / P.WL * np.sqrt(complex(eps))
    pts = np.random.default_rng(2).normal(size=(16, 3)) * 0.15 * P.WL
    E, H = o.field_interior(x, pts, eps)
    E1, H1 = o.field_medium(-x, pts, km, mu0, eps0 * eps)
    x2 = np.concatenate([np.zeros(M, complex), -x[:M] / (eps0 * eps)])
    _, H2 = o.field_medium(x2, pts, km, 1.0, 0.0)
    assert np.linalg.norm(H1 - H) <= 1e-12 * np.linalg.norm(H)
    assert np.linalg.norm(E1 + H2 - E) <= 1e-12 * np.linalg.norm(E)

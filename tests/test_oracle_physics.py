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


@pytest.mark.parametrize("formulation", ["ICTF", "PMCHWT"])
@pytest.mark.parametrize("eps", [P.EPS_DIELECTRIC, P.EPS_METAL])
def test_small_sphere_matches_mie(oracle_lib, eps, formulation):
    V, T = P.sphere(3)
    o = oracle_lib.Oracle(V, T, P.WL, eps, formulation=formulation, threads=16)
    Z = o.dense()
    b = o.rhs(np.array([0.0, 0.0, -1.0]), np.array([1.0, 0.0, 0.0]))
    x = np.linalg.solve(Z, b)
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

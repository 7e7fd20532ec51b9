"""Conjugate-transpose product Z^H (needs a B200).

Z^H is checked three ways: against the oracle's dense matrix (dense mode), by the
dot-product identity <Z^H u, v> = <u, Z v> on MLFMM meshes (a size-independent property),
and entry by entry on sampled rows and columns of the MLFMM operator."""
import numpy as np
import pytest

from tests import problems as P

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.linalg.norm(np.ravel(a - b)) / np.linalg.norm(np.ravel(b))


def test_adjoint_matches_dense_oracle(oracle_lib, gpu_lib):
    from specklesim_b200 import Sie
    V, T = P.sphere(1)
    o = oracle_lib.Oracle(V, T, P.WL, P.EPS_METAL)
    Z = o.dense()
    g = Sie(V, T, P.WL, P.EPS_METAL, dense=True).setup()
    x = P.random_x(o.N, seed=5)
    assert rel(g.matvec_adjoint(x), Z.conj().T @ x) < 1e-10
    g.close()


@pytest.mark.parametrize("eps", [P.EPS_METAL, P.EPS_DIELECTRIC])
@pytest.mark.parametrize("formulation", ["ICTF", "PMCHWT"])
def test_adjoint_dot_product_identity(gpu_lib, eps, formulation):
    """<Z^H u, v> = <u, Z v> for random u, v: the far part is transposed exactly (up to
    the rounding of the khat -> -khat symmetry of the tables), not approximated."""
    from specklesim_b200 import Sie
    V, T = P.slab(cells=24, length_wl=6.0, seed=3)
    g = Sie(V, T, P.WL, eps, formulation=formulation, tree_s_opt=100).setup()
    for s in range(3):
        u = P.random_x(g.n, seed=10 + s)
        v = P.random_x(g.n, seed=20 + s)
        lhs = np.vdot(g.matvec_adjoint(u), v)
        rhs = np.vdot(u, g.matvec(v))
        scale = np.linalg.norm(u) * np.linalg.norm(g.matvec(v))
        assert abs(lhs - rhs) / scale < 1e-12, abs(lhs - rhs) / scale
    g.close()


def test_adjoint_entries(gpu_lib):
    """Z^H[i, j] = conj(Z[j, i]) on 6 x 6 sampled entries, near and far pairs alike."""
    from specklesim_b200 import Sie
    V, T = P.slab(cells=24, length_wl=6.0, seed=3)
    g = Sie(V, T, P.WL, P.EPS_METAL, tree_s_opt=100).setup()
    idx = np.array([0, 17, 1000, g.n // 2 + 3, g.n - 40, g.n - 1])
    E = np.zeros((g.n, len(idx)), np.complex128)
    E[idx, np.arange(len(idx))] = 1.0
    Zcols = g.matvec(E)             # Z[:, idx]
    ZHcols = g.matvec_adjoint(E)    # Z^H[:, idx]
    A = ZHcols[idx, :]              # Z^H[idx_i, idx_j]
    B = Zcols[idx, :].T.conj()      # conj(Z[idx_j, idx_i])
    assert np.abs(A - B).max() / np.abs(B).max() < 1e-10
    g.close()


def test_adjoint_several_columns(gpu_lib):
    from specklesim_b200 import Sie
    V, T = P.slab(cells=24, length_wl=6.0, seed=3)
    g = Sie(V, T, P.WL, P.EPS_METAL, tree_s_opt=100).setup()
    X = np.stack([P.random_x(g.n, seed=30 + j) for j in range(3)], axis=1)
    Y = g.matvec_adjoint(X)
    for j in range(3):
        assert rel(Y[:, j], g.matvec_adjoint(X[:, j])) < 1e-14
    g.close()

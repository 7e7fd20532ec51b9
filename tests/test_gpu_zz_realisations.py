"""One realisation of the batching form through batch.solve_realisation (needs a B200):
its plane waves solved as one batch, directly (dense tensor-core LU with FP64
refinement) and iteratively (batched mixed-precision FGMRES on the MLFMM product), against
one-at-a-time FP64 solves of the same systems."""
import numpy as np
import pytest

from specklesim_b200 import batch, mesh
from tests import problems as P

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.linalg.norm(np.ravel(a - b)) / np.linalg.norm(np.ravel(b))


def _pts():
    th = np.linspace(0.1, 1.2, 6)
    return 5.0 * np.stack([np.sin(th), 0.3 * np.sin(th), np.cos(th)], axis=1)


def test_direct_realisation_matches_fp64_lu(gpu_lib):
    from specklesim_b200 import Sie
    K, E, _ = batch.c4_incidences()
    r = {"seed": 3, "side_wl": 3.0, "rms_wl": 0.3, "corr_wl": 1.0}
    out = batch.solve_realisation(r, P.WL, P.EPS_METAL, K[:3], E[:3], _pts(), tolerance=1e-12)
    assert out["method"] == "direct" and all(out["converged"])
    assert out["intensity"].shape == (3, 6)
    V, T = mesh.slab_config(r["side_wl"], P.WL, r["rms_wl"], r["corr_wl"], r["seed"])
    g = Sie(V, T, P.WL, P.EPS_METAL, dense=True).setup()
    for j in range(3):
        x = g.solve_direct(g.rhs_planewave(K[j], E[j]))
        assert rel(out["intensity"][j], g.farfield(x, _pts())[2]) < 1e-7
    g.close()


def test_iterative_realisation_matches_fp64_gmres(gpu_lib):
    from specklesim_b200 import Sie
    K, E, _ = batch.c4_incidences()
    r = {"seed": 3, "side_wl": 6.0, "rms_wl": 0.3, "corr_wl": 1.0}
    out = batch.solve_realisation(r, P.WL, P.EPS_DIELECTRIC, K[:2], E[:2], _pts(), tolerance=1e-6,
                                  direct_max_unknowns=0, tree_s_opt=100)
    assert out["method"] == "fgmres" and all(out["converged"])
    V, T = mesh.slab_config(r["side_wl"], P.WL, r["rms_wl"], r["corr_wl"], r["seed"])
    g = Sie(V, T, P.WL, P.EPS_DIELECTRIC, tree_s_opt=100).setup()
    for j in range(2):
        x, st = g.solve(g.rhs_planewave(K[j], E[j]), tolerance=1e-7)
        assert st["converged"]
        assert rel(out["intensity"][j], g.farfield(x, _pts())[2]) < 1e-3
    g.close()

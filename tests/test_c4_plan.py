"""The batching form's realisation plan on the CPU: the 64 rough-slab realisations
(seeds 100-163, side, RMS height and correlation length drawn in the recipe's ranges),
their RWG edge counts without meshing, the 16 plane waves, and the rank plan over 8 GPUs."""
import numpy as np

from specklesim_b200 import batch, mesh

WL = 632.8e-9


def test_realisations_follow_the_recipe():
    R = batch.c4_realisations()
    assert [r["seed"] for r in R] == list(range(100, 164))
    for r in R:
        assert 8.0 <= r["side_wl"] <= 20.0
        assert 0.2 <= r["rms_wl"] <= 0.8
        assert 0.5 <= r["corr_wl"] <= 2.0
    assert R == batch.c4_realisations()  # every rank draws the same plan
    e = np.array([r["n_edges"] for r in R])
    assert e.min() < 30000 and e.max() > 90000  # uneven: 13k-70k triangles


def test_edge_count_without_meshing():
    for r in batch.c4_realisations(n=4, seed0=120):
        V, T = mesh.slab_config(r["side_wl"], WL, r["rms_wl"], r["corr_wl"], r["seed"])
        assert r["n_edges"] == 3 * len(T) // 2


def test_sixteen_plane_waves():
    K, E, labels = batch.c4_incidences()
    assert K.shape == (16, 3) and E.shape == (16, 3) and len(set(labels)) == 16
    assert np.allclose(np.linalg.norm(K, axis=1), 1) and np.allclose(np.linalg.norm(E, axis=1), 1)
    assert np.allclose(np.einsum("ij,ij->i", K, E), 0, atol=1e-12)
    assert np.all(K[:, 2] < 0)  # incident from above


def test_rank_plan_balance_on_eight_gpus():
    R = batch.c4_realisations()
    sizes = [r["n_edges"] for r in R]
    plan = batch.assign_realisations(sizes, 8)
    assert sorted(i for p in plan for i in p) == list(range(64))
    assert batch.balance(plan, sizes) < 1.01


class _FakeSie:
    """Stands in for the GPU context: records how solve_realisation drives it."""
    calls = []

    def __init__(self, V, T, wavelength, eps_r2, dense=False, **kw):
        self.n_edges = 3 * len(T) // 2
        self.n = 2 * self.n_edges
        self.dense, self.kw = dense, kw
        _FakeSie.calls.append(("init", dense, tuple(sorted(kw))))

    def setup(self):
        return self

    def rhs_planewave(self, k, E):
        k = np.atleast_2d(k)
        return np.ones((self.n, k.shape[0]), complex) * np.arange(1, k.shape[0] + 1)

    def _stats(self, B):
        return [{"converged": 1, "iterations": 3, "backward_error_true": 1e-12} for _ in range(B.shape[1])]

    def solve_direct_mixed(self, B, tolerance=1e-10, raise_on_noconv=True):
        _FakeSie.calls.append(("direct", B.shape, tolerance))
        return 2 * B, self._stats(B)

    def solve(self, B, **kw):
        _FakeSie.calls.append(("fgmres", B.shape, kw["precision"], kw["time_limit_s"]))
        return 3 * B, self._stats(B)

    def farfield(self, x, pts):
        I = np.full(len(pts), np.abs(x[0]) ** 2)
        return None, None, I

    def close(self):
        _FakeSie.calls.append(("close",))


def test_solve_realisation_drives_the_context(monkeypatch):
    """The host logic of batch.solve_realisation with a stand-in context: the direct path
    up to direct_max_unknowns, the batched mixed FGMRES above it (context arguments passed
    on), one intensity row per plane wave, and the context closed."""
    import specklesim_b200.sie as sie_mod
    monkeypatch.setattr(sie_mod, "Sie", _FakeSie)
    K, E, _ = batch.c4_incidences()
    pts = np.zeros((5, 3))
    r = {"seed": 3, "side_wl": 2.0, "rms_wl": 0.3, "corr_wl": 1.0}
    _FakeSie.calls = []
    out = batch.solve_realisation(r, WL, -11.7 - 1.26j, K[:4], E[:4], pts, tolerance=1e-9)
    assert out["method"] == "direct" and out["intensity"].shape == (4, 5)
    assert np.allclose(out["intensity"][:, 0], [(2 * j) ** 2 for j in range(1, 5)])
    assert out["converged"] == [True] * 4 and out["iterations"] == [3] * 4
    assert _FakeSie.calls[0] == ("init", True, ()) and _FakeSie.calls[1][0] == "direct"
    assert _FakeSie.calls[-1] == ("close",)
    _FakeSie.calls = []
    out = batch.solve_realisation(r, WL, 2.25, K[:2], E[:2], pts, direct_max_unknowns=0, tree_s_opt=100,
                                  time_limit_s=5.0)
    assert out["method"] == "fgmres" and out["intensity"].shape == (2, 5)
    assert _FakeSie.calls[0] == ("init", False, ("tree_s_opt",))
    assert _FakeSie.calls[1][2:] == ("mixed", 5.0) and _FakeSie.calls[-1] == ("close",)
    # a single plane wave as 1-D vectors
    out = batch.solve_realisation(r, WL, 2.25, K[0], E[0], pts)
    assert out["intensity"].shape == (1, 5)

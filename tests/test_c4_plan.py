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

"""Many independent solves across the GPUs of one node.

The solve path has no data exchange: realisations (independent meshes) and their
right-hand sides are the unit of parallel work.  One process per GPU takes a share of
the realisations; nothing crosses NVLink during a solve.  The only collective is the
final gather of the far-field intensities and statistics to rank 0.

Realisations of uneven size are shared by a greedy bin-pack on the edge count: the
largest realisation goes to the least-loaded rank (the cost of a solve grows with M).
"""
import heapq

import numpy as np


def assign_realisations(sizes, world):
    """Indices of the realisations each rank solves: greedy longest-first bin-packing on
    `sizes` (e.g. RWG edge counts).  Deterministic, so every rank computes the same plan."""
    heap = [(0.0, r) for r in range(world)]
    plan = [[] for _ in range(world)]
    for i in sorted(range(len(sizes)), key=lambda i: (-float(sizes[i]), i)):
        load, r = heapq.heappop(heap)
        plan[r].append(i)
        heapq.heappush(heap, (load + float(sizes[i]), r))
    return [sorted(p) for p in plan]


def gather_to_rank0(local, world, rank, group=None):
    """Gather one picklable object per rank to rank 0 (a list in rank order there, None
    elsewhere).  Uses torch.distributed when world > 1."""
    if world == 1:
        return [local]
    import torch.distributed as dist
    out = [None] * world if rank == 0 else None
    dist.gather_object(local, out, dst=0, group=group)
    return out


def run_batch(realisations, solve_one, world=1, rank=0, group=None):
    """Solve every realisation of `realisations` (a list of dicts holding at least
    "n_edges") on this node's ranks.  `solve_one(realisation)` runs on the rank's own GPU
    and returns a dict (intensities, statistics).  Returns, on rank 0, the results in
    realisation order; on the other ranks None."""
    plan = assign_realisations([r["n_edges"] for r in realisations], world)
    mine = {i: solve_one(realisations[i]) for i in plan[rank]}
    parts = gather_to_rank0(mine, world, rank, group)
    if rank != 0:
        return None
    merged = {}
    for p in parts:
        merged.update(p)
    return [merged[i] for i in range(len(realisations))]


def balance(plan, sizes):
    """Largest / mean per-rank load of a plan (1.0 = perfect)."""
    loads = np.array([sum(sizes[i] for i in p) for p in plan], dtype=float)
    return float(loads.max() / loads.mean()) if loads.mean() > 0 else 1.0


# The batching form's incidences: theta in {0, 10, 20, 30} deg x phi in {0, 90} deg x
# {TE, TM}, the 16 plane waves each realisation is solved for (the reference solves them
# one after another, main.f90:450-463 and lib_sie_solver_gmres_interface.f90:46-53).
C4_THETA_DEG = (0.0, 10.0, 20.0, 30.0)
C4_PHI_DEG = (0.0, 90.0)
C4_POLS = ("TE", "TM")


def c4_incidences():
    """(k_in (16, 3), E_in (16, 3), labels) of the batching form's plane waves."""
    from .sie import incidence
    ks, es, labels = [], [], []
    for th in C4_THETA_DEG:
        for ph in C4_PHI_DEG:
            for pol in C4_POLS:
                k, e = incidence(np.deg2rad(th), np.deg2rad(ph), pol, 2)
                ks.append(k)
                es.append(e)
                labels.append((th, ph, pol))
    return np.array(ks), np.array(es), labels


def slab_edges(length_wl, cells=None, thickness_wl=1.0):
    """RWG edges of mesh.slab_config's closed slab without building it: 2 n^2 triangles on
    the top and on the bottom, 2 per side-wall quad (4 n of them per layer, nz layers),
    3/2 edges per triangle."""
    n = int(round(length_wl * 6.4)) if cells is None else int(cells)
    nz = max(1, int(round(thickness_wl * n / length_wl)))
    return 3 * (4 * n * n + 8 * n * nz) // 2


def c4_realisations(n=64, seed0=100):
    """The batching form's realisations: seeds seed0 .. seed0 + n - 1, each drawing its
    square side uniformly in [8, 20] lambda, its RMS height in [0.2, 0.8] lambda and its
    correlation length in [0.5, 2] lambda from its own seed; "n_edges" (for the rank plan)
    from slab_edges.  The mesh itself is built by the rank that solves it."""
    out = []
    for i in range(n):
        seed = seed0 + i
        rng = np.random.default_rng(seed)
        side, rms, corr = rng.uniform(8.0, 20.0), rng.uniform(0.2, 0.8), rng.uniform(0.5, 2.0)
        out.append({"seed": seed, "side_wl": float(side), "rms_wl": float(rms), "corr_wl": float(corr),
                    "n_edges": slab_edges(side)})
    return out


def solve_realisation(r, wavelength, eps_r2, k_in, E_in, pts, tolerance=1e-6, direct_max_unknowns=60000,
                      time_limit_s=600.0, restart=50, max_iterations=650, **context):
    """One realisation on this rank's GPU: its rough slab (mesh.slab_config with the
    realisation's side, RMS height, correlation length and seed), every plane wave of
    (k_in, E_in) as one batch, and the far-field intensities at pts.

    Systems of up to direct_max_unknowns unknowns are solved directly (dense fill, the
    complex64 tensor-core LU and FP64 refinement to `tolerance`), which converges on the
    metal; larger ones with the batched mixed-precision FGMRES on the MLFMM product,
    bounded by time_limit_s (on the metal it stops unconverged, as the reference's does).
    Returns a dict: seed, n_edges, method, intensity (n_waves, n_pts), converged,
    iterations, backward_error per wave, seconds.  `context`: further Sie arguments
    (e.g. tree_s_opt) of the MLFMM context."""
    import time
    from . import mesh
    from .sie import Sie
    t0 = time.time()
    V, T = mesh.slab_config(r["side_wl"], wavelength, r["rms_wl"], r["corr_wl"], r["seed"])
    n_unknowns = 3 * len(T)  # 2 unknowns per edge, 3/2 edges per triangle
    direct = n_unknowns <= direct_max_unknowns
    g = Sie(V, T, wavelength, eps_r2, dense=True).setup() if direct else \
        Sie(V, T, wavelength, eps_r2, **context).setup()
    try:
        B = g.rhs_planewave(np.atleast_2d(k_in), np.atleast_2d(E_in))
        B = B.reshape(g.n, -1)
        if direct:
            X, st = g.solve_direct_mixed(B, tolerance=tolerance, raise_on_noconv=False)
        else:
            X, st = g.solve(B, restart=restart, max_iterations=max_iterations, tolerance=tolerance,
                            precision="mixed", time_limit_s=time_limit_s, raise_on_noconv=False)
        X = X.reshape(g.n, -1)
        st = st if isinstance(st, list) else [st]
        intensity = np.stack([g.farfield(X[:, j], pts)[2] for j in range(X.shape[1])])
        return {"seed": r["seed"], "n_edges": g.n_edges, "method": "direct" if direct else "fgmres",
                "intensity": intensity, "converged": [bool(s["converged"]) for s in st],
                "iterations": [int(s["iterations"]) for s in st],
                "backward_error": [float(s["backward_error_true"]) for s in st],
                "seconds": time.time() - t0}
    finally:
        g.close()

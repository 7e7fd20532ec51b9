"""The solver's limits and the reference's left Jacobi preconditioner (needs a B200).

- lib_sie_ml_fmm_preconditioner_left (src/lib_sie_tri_mlfmm_interface.f90:323-339) divides by
  the diagonal of the self blocks (precalculation_diagonal_element, :94-109): sie_precondition_left
  against the oracle's blocks (m, m).
- A host-side time limit ends a solve with SIE_ERR_TIMEOUT.
- The grid-wide waits of the Arnoldi kernel are bounded: with the limit set to one poll
  (SIE_GRID_SPIN_LIMIT) a solve returns SIE_ERR_CUDA instead of waiting, and the context
  solves normally afterwards.  No GPU fault is involved: the kernel records the failed wait
  and returns.
- A device allocation that cannot succeed (the dense matrix of a mesh whose near panels
  exceed the GPU's memory) ends the set-up with SIE_ERR_NOMEM, and the next context works."""
import numpy as np
import pytest

from tests import problems as P

pytestmark = pytest.mark.gpu


def test_left_jacobi_matches_oracle_self_blocks(oracle_lib, gpu_lib):
    from specklesim_b200 import Sie
    V, T = P.slab(cells=12, length_wl=3.0, seed=5)
    o = oracle_lib.Oracle(V, T, P.WL, P.EPS_METAL, tree_s_opt=60, threads=8)
    g = Sie(V, T, P.WL, P.EPS_METAL, tree_s_opt=60).setup()
    M = g.n_edges
    idx = np.arange(M, dtype=np.int32)
    blk = o.blocks(idx, idx)          # (D11, D12, D21, D22) of every self pair
    diag = np.concatenate([blk[:, 0], blk[:, 3]])
    v = P.random_x(g.n, seed=4)
    w = g.precondition_left(v)
    assert np.linalg.norm(w - v / diag) / np.linalg.norm(v / diag) < 1e-9
    g.close()
    o.close()


def test_time_limit_ends_the_solve(gpu_lib):
    from specklesim_b200 import Sie, SieError, _lib, incidence
    V, T = P.slab(cells=16, length_wl=4.0, seed=3)
    g = Sie(V, T, P.WL, P.EPS_METAL, tree_s_opt=60).setup()
    k, E = incidence(0.0, 0.0, "TM", 2)
    b = g.rhs_planewave(k, E)
    for prec in ("fp64", "mixed"):
        with pytest.raises(SieError) as e:
            g.solve(b, restart=50, max_iterations=2000, tolerance=1e-14, precision=prec, time_limit_s=1e-6)
        assert e.value.code == _lib.SIE_ERR_TIMEOUT
    # the context is still usable
    _, st = g.solve(b, restart=20, max_iterations=20, tolerance=1e-14, raise_on_noconv=False)
    assert st["iterations"] == 20
    g.close()


def test_bounded_grid_wait_reports_and_recovers(gpu_lib, monkeypatch):
    from specklesim_b200 import Sie, SieError, _lib, incidence
    V, T = P.slab(cells=24, length_wl=6.0, seed=1)
    monkeypatch.setenv("SIE_ARNOLDI_MODE", "0")  # the grid-barrier Arnoldi kernel
    g = Sie(V, T, P.WL, P.EPS_METAL, tree_s_opt=100).setup()
    k, E = incidence(0.0, 0.0, "TM", 2)
    b = g.rhs_planewave(k, E)
    x_ref, st_ref = g.solve(b, restart=10, max_iterations=10, tolerance=1e-14, raise_on_noconv=False)
    monkeypatch.setenv("SIE_GRID_SPIN_LIMIT", "1")
    with pytest.raises(SieError) as e:
        g.solve(b, restart=10, max_iterations=10, tolerance=1e-14, raise_on_noconv=False)
    assert e.value.code == _lib.SIE_ERR_CUDA and "grid barrier" in str(e.value)
    monkeypatch.delenv("SIE_GRID_SPIN_LIMIT")
    x, st = g.solve(b, restart=10, max_iterations=10, tolerance=1e-14, raise_on_noconv=False)
    assert st["iterations"] == 10
    assert np.linalg.norm(x - x_ref) <= 1e-12 * np.linalg.norm(x_ref)
    g.close()


def test_allocation_failure_reports_nomem(gpu_lib):
    import torch
    from specklesim_b200 import Sie, SieError, _lib, incidence, mesh
    total = torch.cuda.get_device_properties(0).total_memory
    # a dense context stores 48 bytes per pair of RWG edges: pick a slab whose pairs need more
    # than the whole device
    cells = 64
    while True:
        V, T = mesh.slab_config(cells / 6.4, P.WL, 0.3, 1.0, 4, cells=cells, thickness_wl=1.0)
        M = mesh.edge_count(T)
        if 48.0 * M * M > 1.05 * total:
            break
        cells += 8
    big = Sie(V, T, P.WL, P.EPS_METAL, dense=True)
    with pytest.raises(SieError) as e:
        big.setup()
    assert e.value.code == _lib.SIE_ERR_NOMEM
    big.close()  # frees whatever the failed set-up had allocated
    V, T = P.sphere(2)
    g = Sie(V, T, P.WL, P.EPS_METAL, dense=True).setup()
    x, st = g.solve_direct_mixed(g.rhs_planewave(*incidence(0.0, 0.0, "TM", 2)), tolerance=1e-12)
    assert st["converged"]
    g.close()


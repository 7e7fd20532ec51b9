"""Mixed-precision direct solve (sie_solve_direct_mixed: complex64 LU whose trailing
updates run on the tensor cores as split-FP16 products, 3xTF32 as the fallback, then FP64
iterative refinement) against the FP64 direct solve and the oracle's dense matrix (needs a
B200).

The reference's direct path is the dense fill plus ZGESV (lib_sie_tri_solver_normal_I,
src/lib_sie_tri_solver_normal.f90:64-217; solver_LU, src/lib_sie_math.f90:649-676)."""
import numpy as np
import pytest

from tests import problems as P

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.mark.parametrize("case", ["sphere320", "sphere1280", "slab_metal"])
def test_mixed_direct_solve_matches_fp64_and_oracle(oracle_lib, gpu_lib, case):
    from specklesim_b200 import Sie, incidence
    if case == "sphere320":
        V, T = P.sphere(2)          # N = 960: 8 panels, the last one ragged
    elif case == "sphere1280":
        V, T = P.sphere(3)          # N = 3840: 30 panels, tiles of the update ragged
    else:
        V, T = P.slab(cells=10, length_wl=2.0, seed=3)
    g = Sie(V, T, P.WL, P.EPS_METAL, dense=True).setup()
    k, E = incidence(0.3, 0.2, "TM", 2)
    b = g.rhs_planewave(k, E)
    x64 = g.solve_direct(b)
    xm, st = g.solve_direct_mixed(b, tolerance=1e-12, max_refinements=30)
    assert st["converged"] and st["backward_error_true"] <= 1e-12
    assert 1 <= st["iterations"] <= 30
    assert _rel(xm, x64) < 1e-9
    # these systems need no fallback: one factorisation, its updates in split-FP16
    tt = g.timings()
    assert tt["lu_f16"] == 1 and tt["lu_factorizations"] == 1, tt
    # the currents solve the oracle's own dense system (its blocks agree with the fill
    # kernels' to 1e-9 of the block scale; measured 1.2e-10 on the small sphere)
    o = oracle_lib.Oracle(V, T, P.WL, P.EPS_METAL, threads=8)
    Z = o.dense()
    assert _rel(Z @ xm, o.rhs(k, E)) < 1e-8
    o.close()
    # a second right-hand side reuses the factors
    k2, E2 = incidence(0.0, 0.0, "TE", 2)
    b2 = g.rhs_planewave(k2, E2)
    X, sts = g.solve_direct_mixed(np.stack([b, b2], axis=1), tolerance=1e-12)
    assert all(s["converged"] for s in sts)
    assert _rel(X[:, 0], x64) < 1e-9
    assert _rel(X[:, 1], g.solve_direct(b2)) < 1e-9
    assert g.timings()["lu_factor_ms"] > 0
    g.close()


def test_mixed_direct_solve_refuses_mlfmm_contexts(gpu_lib):
    from specklesim_b200 import Sie, SieError, _lib
    V, T = P.sphere(1)
    g = Sie(V, T, P.WL, P.EPS_METAL, tree_s_opt=20).setup()
    with pytest.raises(SieError) as e:
        g.solve_direct_mixed(np.ones(g.n, complex))
    assert e.value.code == _lib.SIE_ERR_STATE
    g.close()


def test_mixed_direct_solve_with_tf32_updates(gpu_lib, monkeypatch):
    """SIE_LU_GEMM=tf32 runs the trailing updates as 3xTF32 products: the same solution,
    in no more refinement steps."""
    from specklesim_b200 import Sie, incidence
    V, T = P.sphere(3)
    g = Sie(V, T, P.WL, P.EPS_METAL, dense=True).setup()
    b = g.rhs_planewave(*incidence(0.3, 0.2, "TM", 2))
    x_bf, st_bf = g.solve_direct_mixed(b, tolerance=1e-12)
    assert g.timings()["lu_f16"] == 1
    monkeypatch.setenv("SIE_LU_GEMM", "tf32")
    g.invalidate_factors()
    x_tf, st_tf = g.solve_direct_mixed(b, tolerance=1e-12)
    tt = g.timings()
    assert tt["lu_f16"] == 0 and tt["lu_factorizations"] == 1
    assert st_tf["converged"] and st_tf["iterations"] <= st_bf["iterations"]
    assert _rel(x_tf, x_bf) < 1e-10
    g.close()



@pytest.mark.parametrize("env", [
    {"SIE_LU_LOOKAHEAD": "0"},                              # 256 blocks, every multiprocessor
    {"SIE_LU_PANEL_BLOCKS": "1"},                           # a single block
    {"SIE_LU_PANEL_BLOCKS": "3", "SIE_LU_NB": "256", "SIE_LU_BLOCK": "256"},  # 3 blocks, whole-panel blocks
], ids=["all_sms", "one_block", "three_blocks"])
def test_panel_grids_agree(gpu_lib, monkeypatch, env):
    """The cooperative panel kernel with 256 blocks (no look-ahead), with 1 block and with
    3 blocks (256-column panels as one block each) factorises the same matrix to solutions
    that agree with the FP64 solve, in the same number of refinement steps (within one) as
    the default grid."""
    from specklesim_b200 import Sie, incidence
    V, T = P.slab(cells=10, length_wl=2.0, seed=3)
    g = Sie(V, T, P.WL, P.EPS_METAL, dense=True).setup()
    b = g.rhs_planewave(*incidence(0.3, 0.2, "TM", 2))
    x64 = g.solve_direct(b)
    x0, st0 = g.solve_direct_mixed(b, tolerance=1e-12, max_refinements=30)
    for key, val in env.items():
        monkeypatch.setenv(key, val)
    g.invalidate_factors()
    x1, st1 = g.solve_direct_mixed(b, tolerance=1e-12, max_refinements=30)
    assert st0["converged"] and st1["converged"]
    assert _rel(x0, x64) < 1e-9 and _rel(x1, x64) < 1e-9
    assert abs(st1["iterations"] - st0["iterations"]) <= 1
    assert g.timings()["lu_factorizations"] == 1
    g.close()

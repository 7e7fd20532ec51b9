"""Synthetic meshes and the pp_/tt_ file format (CPU)."""
import numpy as np
import pytest

from specklesim_b200 import mesh


def _signed_volume(V, T):
    a, b, c = V[T[:, 0]], V[T[:, 1]], V[T[:, 2]]
    return np.einsum("ij,ij->i", a, np.cross(b, c)).sum() / 6.0


def _closed(T):
    e = np.sort(np.concatenate([T[:, [0, 1]], T[:, [1, 2]], T[:, [2, 0]]]), axis=1)
    _, cnt = np.unique(e, axis=0, return_counts=True)
    return np.all(cnt == 2)


def test_icosphere_counts_and_orientation():
    V, T = mesh.icosphere(3, 1.0)
    assert T.shape == (1280, 3) and mesh.edge_count(T) == 1920
    assert _closed(T)
    # inward right-hand normals => negative signed volume
    assert _signed_volume(V, T) < 0
    assert np.allclose(np.linalg.norm(V, axis=1), 1.0)


def test_rough_slab_closed_and_counts():
    V, T = mesh.slab_config(10, 1.0, 0.5, 1.0, seed=0)
    assert _closed(T)
    assert _signed_volume(V, T) < 0
    assert T.shape[0] == 19456 and mesh.edge_count(T) == 29184


def test_rough_surface_statistics():
    h = mesh.gaussian_rough_surface(128, 10.0, 0.5, 1.0, seed=0)
    assert abs(h.mean()) < 1e-12 and abs(h.std() - 0.5) < 1e-12
    h2 = mesh.gaussian_rough_surface(128, 10.0, 0.5, 1.0, seed=0)
    assert np.array_equal(h, h2)


def test_pp_tt_roundtrip(tmp_path):
    V, T = mesh.icosphere(1, 2.0)
    pp, tt = tmp_path / "pp_s.txt", tmp_path / "tt_s.txt"
    mesh.write_pp_tt(pp, tt, V, T)
    V2, T2 = mesh.read_pp_tt(pp, tt)
    assert np.array_equal(T, T2) and np.allclose(V, V2, rtol=0, atol=0)
    assert open(tt).readline().split() == [str(i + 1) for i in T[0]]


def test_currents_file_format_and_roundtrip(tmp_path):
    from specklesim_b200 import io
    assert io.fortran_es(1.234567890123e-3) == " 1.234567890123E-03"
    assert io.fortran_es(-9.5e-104) == "-9.500000000000-104"
    assert io.fortran_es(0.0) == " 0.000000000000E+00"
    rng = np.random.default_rng(0)
    x = rng.standard_normal(12) * 1e-3 + 1j * rng.standard_normal(12)
    x[3] = 1e-120 - 2e-130j
    p = tmp_path / "Result_SEH_tri_ICTF.txt"
    io.write_currents(p, 80, x)
    lines = p.read_text().splitlines()
    assert len(lines) == 2 + 12 and len(lines[2]) == 2 * (19 + 5)
    n_el, m, y = io.read_currents(p)
    assert n_el == 80 and m == 6
    assert np.allclose(y, x, rtol=1e-12, atol=0)


def test_iteration_log_format(tmp_path):
    from specklesim_b200 import io
    p = tmp_path / "iteration_error.txt"
    io.write_iteration_log(p, [0.5, 1.25e-3])
    assert p.read_text().splitlines()[1] == "         2      1.250000000000E-03     "

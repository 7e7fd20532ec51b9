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


def test_run_parameters_file_roundtrip(tmp_path):
    """Calculation_parameters_* (output_file_GMRES, lib_sie_solver_gmres_interface.f90:
    214-241): the reference's labels in its order, one list-directed line each, and every
    value read back exactly."""
    from specklesim_b200 import io
    keys = io.parameter_keys("surface")
    assert keys[0] == "object_type" and keys[-1] == "m_pairs" and len(keys) == 25
    vals = {k: 0 for k in keys}
    vals.update({
        "object_type": "surface", "formulation_type": "ICTF", "illumination_type": "Plane",
        "beam_waist(nm) (Gaussian beam)": 0.0, "Wavelength (nm)": 632.8,
        "object dimension I (nm)": 6328.0, "object dimension II (nm)": 6328.0,
        "object centroid (m)": (0.0, 1.5e-9, -3.1640000000000001e-07),
        "N_el": 20480, "eps_r2": -11.7 - 1.26j, "evaluation_type": "BRDF_p",
        "evaluation_parameter%dim_a(nm)": (-1.5707963267948966, 1.5707963267948966),
        "GMRES_time (min.)": 0.0123456789, "convergence_tolerance": 1e-6, "l_max": 4,
        "dc at l_max": 7.91e-7, "tree_s_opt": 250, "m_pairs": 30720,
    })
    p = tmp_path / "Calculation_parameters_tri.txt"
    io.write_parameters(p, vals)
    lines = p.read_text().splitlines()
    assert [ln[1:].split("=")[0] + "=" for ln in lines] == \
        [lab.split("=")[0] + "=" for lab in io.PARAMETER_LABELS["surface"]]
    assert lines[0] == " object_type =                  surface"
    back = io.read_parameters(p)
    assert list(back) == keys
    for k in keys:
        v = io.parse_parameter(back[k])
        want = vals[k]
        if isinstance(want, tuple):
            assert v == want, k
        elif isinstance(want, str):
            assert v == want, k
        else:
            assert v == want and type(v) is type(want), k
    with pytest.raises(KeyError):
        io.write_parameters(tmp_path / "x.txt", {"object_type": "surface"})


def test_evaluation_points_follow_the_reference_layout():
    """get_evaluation_points (lib_sie_math.f90:295-359): point (i, j) at index (i - 1) n_a + j with
    the dim_b step outer; 'xy' counts down from the maxima, 'xz' up from the minima; the
    rcs and BRDF cuts sweep theta over dim_a at phi = dim_b(1) on a sphere of radius
    dim_c."""
    from specklesim_b200.observation import evaluation_points
    p = evaluation_points("xy", (-1.0, 1.0), (-2.0, 2.0), 0.5, 3, 2)
    assert p.shape == (6, 3)
    assert np.allclose(p[:3], [[1, 2, 0.5], [0, 2, 0.5], [-1, 2, 0.5]])
    assert np.allclose(p[3:], [[1, -2, 0.5], [0, -2, 0.5], [-1, -2, 0.5]])
    p = evaluation_points("yz", (-1.0, 1.0), (0.0, 4.0), 0.25, 2, 3)
    assert np.allclose(p, [[0.25, 1, 4], [0.25, -1, 4], [0.25, 1, 2], [0.25, -1, 2],
                           [0.25, 1, 0], [0.25, -1, 0]])
    p = evaluation_points("xz", (-1.0, 1.0), (0.0, 4.0), -0.3, 3, 2)
    assert np.allclose(p, [[-1, -0.3, 0], [0, -0.3, 0], [1, -0.3, 0],
                           [-1, -0.3, 4], [0, -0.3, 4], [1, -0.3, 4]])
    p = evaluation_points("BRDF_p", (0.0, np.pi / 2), (np.pi / 4, 0.0), 5.0, 5, 64)
    assert p.shape == (5, 3)
    assert np.allclose(np.linalg.norm(p, axis=1), 5.0)
    assert np.allclose(p[0], [0, 0, 5]) and np.allclose(p[-1], [5 / np.sqrt(2), 5 / np.sqrt(2), 0])
    assert np.allclose(np.arccos(p[:, 2] / 5.0), np.linspace(0, np.pi / 2, 5))
    with pytest.raises(ValueError):
        evaluation_points("zz", (0, 1), (0, 1), 0.0, 3, 3)


def test_energy_scat_follows_the_reference_formulas():
    """rcs: |E|^2 4 pi |r|^2; BRDF: |E|^2 |r|^2 / (cos theta_in cos theta_s) on the cut's
    angles (lib_sie_tri_solver_normal.f90:316-360), from fields on the cut's points."""
    from specklesim_b200.observation import energy_scat, evaluation_points
    rng = np.random.default_rng(4)
    pts = evaluation_points("BRDF_p", (0.0, 1.2), (0.3, 0.0), 5.0, 7)
    E = rng.normal(size=(7, 3)) + 1j * rng.normal(size=(7, 3))
    e2 = np.array([np.vdot(e, e).real for e in E])
    assert np.allclose(energy_scat("rcs_p", E, pts), e2 * 4 * np.pi * 25.0)
    th = np.linspace(0.0, 1.2, 7)
    assert np.allclose(energy_scat("BRDF_n", E, pts, theta_in=0.2, dim_a=(0.0, 1.2), n_a=7),
                       e2 * 25.0 / (np.cos(0.2) * np.cos(th)))
    with pytest.raises(ValueError):
        energy_scat("xy", E, pts)

"""Observation points in the reference's layouts, for sie_farfield.

get_evaluation_points (src/lib_sie_math.f90:295-359) builds the points at which the
reference evaluates the scattered field: a plane grid for the 'xy', 'yz' and 'xz' maps,
and a theta cut on a sphere for 'rcs_p'/'rcs_n' and 'BRDF_p'/'BRDF_n'.  The same
parameters (evaluation_parameter%dim_a, dim_b, dim_c, N_dim) give the same points in
the same order here.
"""
import numpy as np

PLANES = ("xy", "yz", "xz")
CUTS = ("rcs_p", "rcs_n", "BRDF_p", "BRDF_n")


def evaluation_points(evaluation_type, dim_a, dim_b, dim_c, n_a, n_b=1):
    """Points (n, 3) of get_evaluation_points.

    Planes: dim_a and dim_b are the (min, max) ranges of the two in-plane coordinates
    and dim_c is the fixed third one; n_a x n_b points, dim_a fastest.  'xy' and 'yz'
    run down from the maxima, 'xz' up from the minima, as the reference does.
    Cuts: theta runs over dim_a in n_a steps at phi = dim_b[0] on the sphere of radius
    dim_c.  The reference allocates n_a x n_b points for a cut but fills only these
    n_a (the rest stay at the origin); only the filled ones are returned.
    """
    a0, a1 = float(dim_a[0]), float(dim_a[1])
    if n_a < 2:
        raise ValueError("evaluation_points: n_a must be at least 2")
    dx_a = (a1 - a0) / (n_a - 1)
    j = np.arange(n_a, dtype=np.float64)
    c = float(dim_c)
    if evaluation_type in CUTS:
        phi = float(dim_b[0])
        theta = a0 + dx_a * j
        return np.stack([np.sin(theta) * np.cos(phi), np.sin(theta) * np.sin(phi),
                         np.cos(theta)], axis=1) * c
    if evaluation_type not in PLANES:
        raise ValueError(f"evaluation_points: unknown evaluation type {evaluation_type!r}")
    if n_b < 2:
        raise ValueError("evaluation_points: n_b must be at least 2 for a plane")
    b0, b1 = float(dim_b[0]), float(dim_b[1])
    dx_b = (b1 - b0) / (n_b - 1)
    # index (i - 1) * n_a + j: the dim_b step is the outer loop
    jj = np.tile(j, n_b)
    ii = np.repeat(np.arange(n_b, dtype=np.float64), n_a)
    out = np.empty((n_a * n_b, 3))
    if evaluation_type == "xy":
        out[:, 0], out[:, 1], out[:, 2] = a1 - dx_a * jj, b1 - dx_b * ii, c
    elif evaluation_type == "yz":
        out[:, 0], out[:, 1], out[:, 2] = c, a1 - dx_a * jj, b1 - dx_b * ii
    else:
        out[:, 0], out[:, 1], out[:, 2] = a0 + dx_a * jj, c, b0 + dx_b * ii
    return out


def energy_scat(evaluation_type, E, pts, theta_in=0.0, dim_a=None, n_a=None):
    """The scattered energy the reference reports beside E_out
    (lib_sie_tri_observation_field_calculation, src/lib_sie_tri_solver_normal.f90:325-360):
    for 'rcs_p'/'rcs_n', |E|^2 4 pi |r|^2 (the intensity of sie_farfield); for
    'BRDF_p'/'BRDF_n', |E|^2 |r|^2 / (cos theta_in cos theta_s), with theta_s the cut's
    angles dim_a[0] + j (dim_a[1] - dim_a[0]) / (n_a - 1) (:316-322).  E: (n, 3) complex
    fields at the points pts (n, 3)."""
    E = np.asarray(E)
    p = np.asarray(pts, dtype=np.float64).reshape(-1, 3)
    e2 = np.sum(np.abs(E) ** 2, axis=1)
    r2 = np.sum(p * p, axis=1)
    if evaluation_type in ("rcs_p", "rcs_n"):
        return e2 * 4 * np.pi * r2
    if evaluation_type in ("BRDF_p", "BRDF_n"):
        if dim_a is None or n_a is None:
            raise ValueError("energy_scat: BRDF needs the cut's dim_a and n_a")
        a0, a1 = float(dim_a[0]), float(dim_a[1])
        theta_s = a0 + (a1 - a0) / (n_a - 1) * np.arange(n_a)
        if theta_s.size != e2.size:
            raise ValueError("energy_scat: one field per angle of the cut")
        return e2 * r2 / (np.cos(theta_in) * np.cos(theta_s))
    raise ValueError(f"energy_scat: no energy for evaluation type {evaluation_type!r}")

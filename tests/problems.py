"""Small seeded SIE problems shared by the CPU and GPU tests."""
import numpy as np

from specklesim_b200 import mesh

WL = 632.8e-9
EPS_METAL = -11.7 - 1.26j      # reference convention exp(+iwt): lossy => Im < 0
EPS_DIELECTRIC = 2.25 - 0.01j


def sphere(sub=2, radius_wl=0.5):
    V, T = mesh.icosphere(sub, radius_wl * WL)
    return V, T


def slab(cells=24, length_wl=4.0, seed=3, rms_wl=0.3, corr_wl=1.0, thickness_wl=1.0):
    return mesh.rough_slab(cells, length_wl * WL, thickness_wl * WL, rms_wl * WL, corr_wl * WL, seed,
                           nz=max(1, int(round(thickness_wl * cells / length_wl))))


def random_x(n, seed=0):
    rng = np.random.default_rng(seed)
    return rng.standard_normal(n) + 1j * rng.standard_normal(n)

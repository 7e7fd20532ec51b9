"""B200-native SIE hot path of SpeckleSim: RWG near-field fill with Hänninen
singularity subtraction + MLFMM matvec + GMRES, behind the reference's matvec
callback interface (C-ABI in include/sie_gpu.h, loaded from libsiegpu.so)."""
from ._lib import SieError, load  # noqa: F401
from .sie import Sie, incidence  # noqa: F401

__all__ = ["Sie", "SieError", "incidence", "load"]

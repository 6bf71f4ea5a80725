"""B200-native implementation of ParMooN's scalar convection-diffusion hot path.

The work runs in ``libcdgpu.so`` (CUDA for sm_100a, C ABI in ``include/cdgpu.h``);
this package holds its ctypes binding (:mod:`._lib`), the host mirror of the
reference's ``TSystemCD2D`` / ``TSystemCD3D`` facade (:mod:`.system`), structured
mesh and DOF-map generation (:mod:`.mesh`) and the in-tree build (:mod:`._build`).
"""
from .system import (GALERKIN, GMG, SUPG, Context, TSystemCD2D, TSystemCD3D, coeffs,  # noqa: F401
                     solver_params)

"""em3d_b200 — B200-native operator-and-Krylov path of em3d.

A drop-in for the reference's hot path: ``Backend.b200()`` plays the role of a
new ``em3d.Backend``; ``Grid``, ``Problem``, ``PreparedEMKernel``,
``Operator``, ``AcousticOperator`` and the solvers keep the reference's names,
signatures and error behaviour.  All operator and solver arithmetic runs in
the sm_100a kernels of ``_native/libem3d_b200.so`` (C ABI in
``include/em3d_b200.h``); there is no CPU fallback.
"""
from __future__ import annotations

from .backend import Backend, Precision
from .problem import (AxisAlignedBox, Ellipsoid, FullDomain, Grid, Problem, cylinder_refraction,
                      ellipsis_refraction, flat_wave_vec, sample_contrast_tensor)
from .operator import Operator, PreparedEMKernel, prep_coeffs_em3d, prep_conj_coeffs_em3d
from . import acoustics, gamma0

__version__ = "0.1.0"
REFERENCE_VERSION = "0.8.0"

__all__ = [
    "Backend", "Precision", "Grid", "Problem", "Operator", "PreparedEMKernel", "prep_coeffs_em3d",
    "prep_conj_coeffs_em3d", "flat_wave_vec", "sample_contrast_tensor", "cylinder_refraction",
    "ellipsis_refraction", "Ellipsoid", "AxisAlignedBox", "FullDomain", "acoustics", "gamma0",
]

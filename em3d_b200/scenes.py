"""Scenes of (rotated) ellipsoids and plane waves, built on the device
(``em3d_sample_ellipsoids`` / ``em3d_plane_wave`` in ``csrc/materials.cu``).

These replace the host-side builders when many inputs are needed (training
data for the warm start, large multi-sphere acoustic scenes): the contrast is
sampled at cell centres exactly as the reference's ``center_mask`` +
``sample_contrast_tensor`` do it (``src/em3d/geometry.py:67-93, 203-252``),
with the ellipsoid's offset rotated into its body frame first; shapes are
painted in order (the last shape containing a cell wins).
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Sequence

import numpy as np

from . import _lib
from .problem import Grid

SHAPE_DOUBLES = 33


@dataclass(frozen=True)
class EllipsoidShape:
    """Ellipsoid ``{c + R p : sum (p_i / a_i)^2 <= 1}`` with material ``eps``
    (scalar or 3x3 complex; the acoustic builder reads the scalar / [0][0])."""

    center: tuple
    radii: tuple
    rotation: object = None
    eps: object = 1.0

    def packed(self) -> np.ndarray:
        R = np.eye(3) if self.rotation is None else np.asarray(self.rotation, dtype=np.float64)
        if R.shape != (3, 3):
            raise ValueError(f"rotation must be 3x3, got {R.shape}")
        if len(self.center) != 3 or len(self.radii) != 3:
            raise ValueError("center and radii must have three values")
        if any(float(a) <= 0.0 for a in self.radii):
            raise ValueError(f"ellipsoid radii must be positive, got {self.radii!r}")
        e = np.asarray(self.eps, dtype=np.complex128)
        if e.ndim == 0:
            e = complex(e) * np.eye(3, dtype=np.complex128)
        if e.shape != (3, 3):
            raise ValueError(f"eps must be a scalar or 3x3, got {e.shape}")
        ev = np.stack([e.real.reshape(-1), e.imag.reshape(-1)], axis=1).reshape(-1)
        return np.concatenate([np.asarray(self.center, np.float64), np.asarray(self.radii, np.float64),
                               R.reshape(-1), ev])


def pack_shapes(shapes: Sequence[EllipsoidShape]) -> np.ndarray:
    if not shapes:
        return np.zeros((0, SHAPE_DOUBLES))
    return np.stack([s.packed() for s in shapes])


_AXES = {}


def device_axes(grid: Grid):
    """Float64 cell-centre coordinates of ``grid`` on its device (cached)."""
    import torch

    key = (grid.N, tuple(grid.L), tuple(grid.center), grid.backend.precision.value, str(grid.backend.torch_device))
    hit = _AXES.get(key)
    if hit is None:
        hit = tuple(torch.as_tensor(np.asarray(a, dtype=np.float64), device=grid.backend.torch_device)
                    for a in grid.host_axes)
        _AXES[key] = hit
    return hit


def _upload_shapes(grid, shapes):
    import torch

    packed = shapes if isinstance(shapes, np.ndarray) else pack_shapes(shapes)
    packed = np.ascontiguousarray(packed, dtype=np.float64).reshape(-1, SHAPE_DOUBLES)
    dev = torch.as_tensor(packed, device=grid.backend.torch_device) if len(packed) else None
    return packed.shape[0], dev


def reference_tol(grid: Grid) -> float:
    """The EM builder's tolerance, 64 eps_f64 max(1, |L|) (``geometry.py:79``)."""
    return 64.0 * float(np.finfo(np.float64).eps) * max(1.0, *(abs(float(v)) for v in grid.L))


def sample_scene(grid: Grid, shapes, *, background_eps_r=1.0, tol: float | None = None, out=None):
    """EM contrast ``chi = eps - I`` (3, 3, Nx, Ny, Nz) of the scene, in the
    grid's complex dtype, written into ``out`` when given."""
    import torch

    be = grid.backend
    if out is None:
        out = torch.empty((3, 3) + grid.N, dtype=be.precision.torch_complex, device=be.torch_device)
    bg = np.asarray(background_eps_r, dtype=np.complex128)
    if bg.ndim == 0:
        bg = complex(bg) * np.eye(3, dtype=np.complex128)
    bgv = np.ascontiguousarray(np.stack([bg.real.reshape(-1), bg.imag.reshape(-1)], axis=1).reshape(-1))
    count, dev = _upload_shapes(grid, shapes)
    x, y, z = device_axes(grid)
    _lib.call("em3d_sample_ellipsoids", _lib.EM3D_EM, be.precision.native_dtype, *grid.N, x.data_ptr(), y.data_ptr(),
              z.data_ptr(), count, None if dev is None else dev.data_ptr(),
              float(reference_tol(grid) if tol is None else tol), bgv.ctypes.data, out.data_ptr(),
              _lib.stream_handle())
    return out


def sample_scene_eta(grid: Grid, shapes, *, eta_outside=1.0, tol: float = 0.0, out=None):
    """Acoustic material ``eta`` (Nx, Ny, Nz): each shape's scalar ``eps``
    inside it, ``eta_outside`` elsewhere (``eta_sphere`` semantics, tol 0)."""
    import torch

    be = grid.backend
    if out is None:
        out = torch.empty(grid.N, dtype=be.precision.torch_complex, device=be.torch_device)
    e = complex(eta_outside)
    bgv = np.array([e.real, e.imag], dtype=np.float64)
    count, dev = _upload_shapes(grid, shapes)
    x, y, z = device_axes(grid)
    _lib.call("em3d_sample_ellipsoids", _lib.EM3D_ACOUSTIC, be.precision.native_dtype, *grid.N, x.data_ptr(),
              y.data_ptr(), z.data_ptr(), count, None if dev is None else dev.data_ptr(), float(tol),
              bgv.ctypes.data, out.data_ptr(), _lib.stream_handle())
    return out


def plane_wave(grid: Grid, *, k: float, orient, amplitude, phi0: float = 0.0, sign: int = 1, out=None):
    """``amplitude exp(i sign (k orient.r + phi0))``, (3, Nx, Ny, Nz) on the
    device (the arithmetic of ``flat_wave_vec``, ``src/em3d/wave.py:9-37``)."""
    import torch

    norm2 = float(orient[0]) ** 2 + float(orient[1]) ** 2 + float(orient[2]) ** 2
    if abs(norm2 - 1.0) > 1e-9:
        raise ValueError(f"orient must be a unit vector, got norm² = {norm2}")
    be = grid.backend
    if out is None:
        out = torch.empty((3,) + grid.N, dtype=be.precision.torch_complex, device=be.torch_device)
    o = np.ascontiguousarray(np.asarray(orient, dtype=np.float64))
    a = np.asarray(amplitude, dtype=np.complex128)
    av = np.ascontiguousarray(np.stack([a.real, a.imag], axis=1).reshape(-1))
    x, y, z = device_axes(grid)
    _lib.call("em3d_plane_wave", be.precision.native_dtype, *grid.N, x.data_ptr(), y.data_ptr(), z.data_ptr(),
              float(k), o.ctypes.data, av.ctypes.data, float(phi0), int(sign), out.data_ptr(), _lib.stream_handle())
    return out

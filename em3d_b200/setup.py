"""Host-side problem inputs: grid axes, incident waves and material tensors.

These are the one-off input builders that sit below the operator (they are
not on the hot path).  They run on the host in NumPy, reproduce the
reference's arithmetic operation by operation so that the device operator is
fed the same bits the reference would see, and are uploaded once.

Reference counterparts (qwerty29544/em3d v0.8.0):
``src/em3d/grid.py:10-52``, ``src/em3d/wave.py:9-37``,
``src/em3d/geometry.py:18-93,203-252``, ``src/em3d/refraction.py:11-138``,
``src/em3d/acoustics/materials.py:11-83``, ``src/em3d/acoustics/problem.py:10-40``.
"""
from __future__ import annotations

from dataclasses import dataclass
from enum import Enum
from math import pi

import numpy as np


def real_dtype_of(precision: str):
    return np.float32 if precision == "single" else np.float64


def complex_dtype_of(precision: str):
    return np.complex64 if precision == "single" else np.complex128


# ---------------------------------------------------------------------------
# grid (reference src/em3d/grid.py:10-13)
# ---------------------------------------------------------------------------

def axis_host(n: int, length: float, centre: float, real_dtype) -> np.ndarray:
    step = length / n
    start = centre - length / 2 + step / 2
    return np.linspace(start, start + step * (n - 1), n, dtype=real_dtype)


def grid_axes_host(N, L, center, precision: str = "double"):
    rd = real_dtype_of(precision)
    return tuple(axis_host(int(N[i]), float(L[i]), float(center[i]), rd) for i in range(3))


def _mesh(axes):
    return np.meshgrid(axes[0], axes[1], axes[2], indexing="ij")


# ---------------------------------------------------------------------------
# incident waves
# ---------------------------------------------------------------------------

def flat_wave_vec_host(axes, *, k, orient, amplitude, phi0=0.0, sign=1, dtype=np.complex128):
    """``A exp(i sign (k orient.r + phi0))``, shape (3,Nx,Ny,Nz) (reference ``src/em3d/wave.py:9-37``)."""
    if sign not in (1, -1):
        raise ValueError(f"sign must be 1 or -1, got {sign!r}")
    norm2 = float(orient[0]) ** 2 + float(orient[1]) ** 2 + float(orient[2]) ** 2
    if abs(norm2 - 1.0) > 1e-9:
        raise ValueError(f"orient must be a unit vector, got norm² = {norm2}")
    X, Y, Z = _mesh(axes)
    phase = sign * (k * (orient[0] * X + orient[1] * Y + orient[2] * Z) + phi0)
    carrier = np.exp(1j * phase).astype(dtype, copy=False)
    out = np.zeros((3,) + X.shape, dtype=dtype)
    for i, a in enumerate(amplitude):
        if a != 0.0:
            out[i] = dtype(a) * carrier
    return out


def plane_wave_scalar_host(axes, *, k, direction=(0.0, 0.0, 1.0), amplitude=1.0, dtype=np.complex128):
    """``amplitude exp(i k d.x)`` (reference ``src/em3d/acoustics/problem.py:10-40``)."""
    d = tuple(float(x) for x in direction)
    if len(d) != 3:
        raise ValueError(f"direction must have length 3, got {direction!r}")
    rd = np.float32 if dtype == np.complex64 else np.float64
    dv = np.asarray(d, dtype=rd)
    norm = float(np.linalg.norm(dv))
    if norm == 0.0:
        raise ValueError("direction must be non-zero")
    dv = dv / norm
    X, Y, Z = _mesh(axes)
    phase = dv[0] * X + dv[1] * Y + dv[2] * Z
    ik = dtype(1j * float(k))
    return (dtype(amplitude) * np.exp(ik * phase)).astype(dtype, copy=False)


# ---------------------------------------------------------------------------
# EM geometry and contrast (reference src/em3d/geometry.py)
# ---------------------------------------------------------------------------

class SamplingMode(str, Enum):
    CELL_CENTER = "cell_center"


@dataclass(frozen=True)
class FullDomain:
    pass


@dataclass(frozen=True)
class AxisAlignedBox:
    center: tuple
    size: tuple

    def __post_init__(self):
        if any(float(v) <= 0.0 for v in self.size):
            raise ValueError(f"box sizes must be positive, got {self.size!r}")


@dataclass(frozen=True)
class Ellipsoid:
    center: tuple
    radii: tuple

    def __post_init__(self):
        if any(float(v) <= 0.0 for v in self.radii):
            raise ValueError(f"ellipsoid radii must be positive, got {self.radii!r}")


def center_mask(geometry, axes, L) -> np.ndarray:
    """Cell centres inside ``geometry`` (reference ``src/em3d/geometry.py:62-93``)."""
    shape = tuple(len(a) for a in axes)
    if isinstance(geometry, FullDomain):
        return np.ones(shape, dtype=bool)
    x, y, z = (np.asarray(a, dtype=np.float64) for a in axes)
    X, Y, Z = np.meshgrid(x, y, z, indexing="ij")
    tol = 64.0 * np.finfo(np.float64).eps * max(1.0, *(abs(float(v)) for v in L))
    if isinstance(geometry, AxisAlignedBox):
        res = np.ones(shape, dtype=bool)
        for cc, c0, sz in zip((X, Y, Z), geometry.center, geometry.size):
            res &= np.abs(cc - float(c0)) <= float(sz) / 2.0 + tol
        return res
    if isinstance(geometry, Ellipsoid):
        val = np.zeros(shape, dtype=np.float64)
        for cc, c0, rr in zip((X, Y, Z), geometry.center, geometry.radii):
            val += ((cc - float(c0)) / float(rr)) ** 2
        return val <= 1.0 + tol
    raise TypeError(f"unsupported geometry {type(geometry)!r}")


def _material_tensor(value, name):
    arr = np.asarray(value, dtype=np.complex128)
    if arr.ndim == 0:
        return complex(arr) * np.eye(3, dtype=np.complex128)
    if arr.shape != (3, 3):
        raise ValueError(f"{name} must be a scalar or a (3, 3) tensor, got {arr.shape}")
    return arr


def sample_contrast_tensor(axes, L, *, background_eps_r, feature_eps_r, geometry, dtype=np.complex128):
    """``chi = eps_r - I`` sampled at cell centres (reference ``src/em3d/geometry.py:203-252``)."""
    bg = _material_tensor(background_eps_r, "background_eps_r")
    ft = _material_tensor(feature_eps_r, "feature_eps_r")
    w = center_mask(geometry, axes, L).astype(np.float64)
    eps = bg[:, :, None, None, None] + (ft - bg)[:, :, None, None, None] * w[None, None, ...]
    eps = np.asarray(eps, dtype=dtype)
    eye = np.asarray(np.eye(3, dtype=np.complex128)[:, :, None, None, None], dtype=dtype)
    return (eps - eye).astype(dtype, copy=False)


def _eta_matrix(eps_real, eps_imag):
    """(3,3) contrast from permittivity parts (reference ``src/em3d/refraction.py:11-49``)."""
    if (np.ndim(eps_real) == 0) != (np.ndim(eps_imag) == 0):
        raise TypeError("eps_real and eps_imag must both be scalars or both be (3,3) arrays")
    if np.ndim(eps_real) == 0:
        if np.iscomplex(eps_real) or np.iscomplex(eps_imag):
            raise TypeError("eps_real / eps_imag must be real scalars")
        return (float(eps_real) - 1.0 + 1j * float(eps_imag)) * np.eye(3, dtype=np.complex128)
    E = np.asarray(eps_real, dtype=np.float64)
    F = np.asarray(eps_imag, dtype=np.float64)
    if E.shape != (3, 3) or F.shape != (3, 3):
        raise ValueError("eps_real and eps_imag must have shape (3,3)")
    return (E - np.eye(3)) + 1j * F


def _masked_tensor(mask, eta, dtype):
    out = np.zeros((3, 3) + mask.shape, dtype=dtype)
    for i in range(3):
        for j in range(3):
            out[i, j] = np.where(mask, eta[i, j], out[i, j])
    return out


def cylinder_refraction(axes, *, eps_real, eps_imag, radius, axis="z", dtype=np.complex128):
    """Infinite cylinder contrast (reference ``src/em3d/refraction.py:52-83``)."""
    X, Y, Z = _mesh(axes)
    if axis == "z":
        r2 = X * X + Y * Y
    elif axis == "y":
        r2 = X * X + Z * Z
    elif axis == "x":
        r2 = Y * Y + Z * Z
    else:
        raise ValueError(f"axis must be 'x'|'y'|'z', got {axis!r}")
    return _masked_tensor(r2 <= radius * radius, _eta_matrix(eps_real, eps_imag), dtype)


def ellipsis_refraction(axes, *, eps_real, eps_imag, center, radius, dtype=np.complex128):
    """Axis-aligned ellipsoid contrast (reference ``src/em3d/refraction.py:112-138``)."""
    X, Y, Z = _mesh(axes)
    metric = ((X - center[0]) / radius[0]) ** 2 + ((Y - center[1]) / radius[1]) ** 2 + ((Z - center[2]) / radius[2]) ** 2
    return _masked_tensor(metric <= 1.0, _eta_matrix(eps_real, eps_imag), dtype)


# ---------------------------------------------------------------------------
# acoustic materials (reference src/em3d/acoustics/materials.py)
# ---------------------------------------------------------------------------

def eta_homogeneous(shape, eta_value, dtype=np.complex128):
    out = np.zeros(tuple(shape), dtype=dtype)
    out[...] = dtype(eta_value)
    return out


def eta_ellipsoid(axes, *, center, radii, eta_inside, eta_outside=1.0, dtype=np.complex128):
    if len(center) != 3:
        raise ValueError(f"center must have length 3, got {center!r}")
    if len(radii) != 3 or any(float(r) <= 0.0 for r in radii):
        raise ValueError(f"radii must contain three positive values, got {radii!r}")
    X, Y, Z = _mesh(axes)
    cx, cy, cz = (float(v) for v in center)
    rx, ry, rz = (float(v) for v in radii)
    metric = ((X - cx) / rx) ** 2 + ((Y - cy) / ry) ** 2 + ((Z - cz) / rz) ** 2
    return np.where(metric <= 1.0, dtype(eta_inside), dtype(eta_outside)).astype(dtype, copy=False)


def eta_sphere(axes, *, center, radius, eta_inside, eta_outside=1.0, dtype=np.complex128):
    return eta_ellipsoid(axes, center=center, radii=(float(radius),) * 3, eta_inside=eta_inside,
                         eta_outside=eta_outside, dtype=dtype)


def eta_slab(axes, L, center, *, eta_inside, eta_outside=1.0, axis=0, width_fraction=0.5, dtype=np.complex128):
    if axis not in (0, 1, 2):
        raise ValueError(f"axis must be 0, 1, or 2, got {axis!r}")
    if not (0.0 < float(width_fraction) <= 1.0):
        raise ValueError(f"width_fraction must be in (0, 1], got {width_fraction!r}")
    coords = _mesh(axes)
    half = 0.5 * float(L[axis]) * float(width_fraction)
    mask = np.abs(coords[axis] - float(center[axis])) <= half
    return np.where(mask, dtype(eta_inside), dtype(eta_outside)).astype(dtype, copy=False)


def exact_ellipsoid_volume(radii) -> float:
    return float(4.0 * pi * np.prod(radii) / 3.0)

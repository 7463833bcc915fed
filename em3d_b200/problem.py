"""Grid, Problem and the input builders of the public API.

Mirror of the reference ``Grid`` (``src/em3d/grid.py:16-52``), ``Problem``
(``src/em3d/problem.py:7-46``), ``flat_wave_vec`` (``src/em3d/wave.py:9-37``),
``sample_contrast_tensor`` (``src/em3d/geometry.py:233-252``) and the legacy
refraction profiles (``src/em3d/refraction.py``).  Inputs are computed on the
host with the reference's arithmetic (``em3d_b200.setup``) and uploaded once.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Tuple

import numpy as np

from . import setup as _setup
from .backend import Backend


def _to_device(be: Backend, arr, dtype=None):
    import torch

    if isinstance(arr, torch.Tensor):
        t = arr.to(device=be.torch_device)
        return t if dtype is None else t.to(dtype)
    a = np.ascontiguousarray(arr)
    t = torch.from_numpy(a).to(be.torch_device)
    return t if dtype is None else t.to(dtype)


@dataclass(frozen=True)
class Grid:
    """Uniform cell-centred grid; ``x, y, z`` are device tensors of the precision's real dtype."""

    N: Tuple[int, int, int]
    L: Tuple[float, float, float]
    center: Tuple[float, float, float]
    backend: Backend
    _x: object = field(init=False, repr=False)
    _y: object = field(init=False, repr=False)
    _z: object = field(init=False, repr=False)
    _host_axes: object = field(init=False, repr=False)

    def __post_init__(self) -> None:
        if any(n <= 0 for n in self.N):
            raise ValueError(f"Grid.N must be strictly positive, got {self.N}")
        if any(v <= 0 for v in self.L):
            raise ValueError(f"Grid.L must be strictly positive, got {self.L}")
        object.__setattr__(self, "N", tuple(int(n) for n in self.N))
        host = _setup.grid_axes_host(self.N, self.L, self.center, self.backend.precision.value)
        object.__setattr__(self, "_host_axes", host)
        object.__setattr__(self, "_x", _to_device(self.backend, host[0]))
        object.__setattr__(self, "_y", _to_device(self.backend, host[1]))
        object.__setattr__(self, "_z", _to_device(self.backend, host[2]))

    @property
    def dv(self) -> float:
        return (self.L[0] / self.N[0]) * (self.L[1] / self.N[1]) * (self.L[2] / self.N[2])

    @property
    def x(self):
        return self._x

    @property
    def y(self):
        return self._y

    @property
    def z(self):
        return self._z

    @property
    def host_axes(self):
        """The axes as NumPy arrays (what the host input builders use)."""
        return self._host_axes

    def coords(self):
        import torch

        return torch.meshgrid(self._x, self._y, self._z, indexing="ij")


@dataclass(frozen=True)
class Problem:
    """``Problem(grid, eps_tensor, wave, k0, volume)``; ``eps_tensor`` is ``chi = eps_r - I``."""

    grid: Grid
    eps_tensor: object
    wave: object
    k0: float
    volume: float

    def __post_init__(self) -> None:
        be = self.grid.backend
        expected_eta = (3, 3) + tuple(self.grid.N)
        expected_wave = (3,) + tuple(self.grid.N)
        if tuple(self.eps_tensor.shape) != expected_eta:
            raise ValueError(f"eps_tensor.shape {tuple(self.eps_tensor.shape)} != expected {expected_eta}")
        if tuple(self.wave.shape) != expected_wave:
            raise ValueError(f"wave.shape {tuple(self.wave.shape)} != expected {expected_wave}")
        tc = be.precision.torch_complex
        for name in ("eps_tensor", "wave"):
            val = getattr(self, name)
            dt = val.dtype
            ok = (dt == tc) if not isinstance(dt, np.dtype) else (dt == np.dtype(be.complex_dtype))
            if not ok:
                raise TypeError(f"{name}.dtype {dt} != {be.complex_dtype}")
            object.__setattr__(self, name, _to_device(be, val).contiguous())

    @property
    def backend(self):
        return self.grid.backend

    @property
    def contrast_tensor(self):
        return self.eps_tensor


def flat_wave_vec(grid: Grid, *, k: float, orient, amplitude, phi0: float = 0.0, sign: int = 1):
    """Plane wave ``A exp(i sign (k orient.r + phi0))`` as a (3,Nx,Ny,Nz) device tensor."""
    host = _setup.flat_wave_vec_host(grid.host_axes, k=k, orient=orient, amplitude=amplitude, phi0=phi0,
                                     sign=sign, dtype=grid.backend.complex_dtype)
    return _to_device(grid.backend, host)


def sample_contrast_tensor(grid: Grid, *, background_eps_r, feature_eps_r, geometry,
                           mode=_setup.SamplingMode.CELL_CENTER):
    """``chi = eps_r - I`` sampled at cell centres, as a (3,3,Nx,Ny,Nz) device tensor."""
    if _setup.SamplingMode(mode) is not _setup.SamplingMode.CELL_CENTER:
        raise NotImplementedError("only cell-centre sampling is provided")
    host = _setup.sample_contrast_tensor(grid.host_axes, grid.L, background_eps_r=background_eps_r,
                                         feature_eps_r=feature_eps_r, geometry=geometry,
                                         dtype=grid.backend.complex_dtype)
    return _to_device(grid.backend, host)


def cylinder_refraction(grid: Grid, *, eps_real, eps_imag, radius: float, axis: str = "z"):
    host = _setup.cylinder_refraction(grid.host_axes, eps_real=eps_real, eps_imag=eps_imag, radius=radius,
                                      axis=axis, dtype=grid.backend.complex_dtype)
    return _to_device(grid.backend, host)


def ellipsis_refraction(grid: Grid, *, eps_real, eps_imag, center, radius):
    host = _setup.ellipsis_refraction(grid.host_axes, eps_real=eps_real, eps_imag=eps_imag, center=center,
                                      radius=radius, dtype=grid.backend.complex_dtype)
    return _to_device(grid.backend, host)


Ellipsoid = _setup.Ellipsoid
AxisAlignedBox = _setup.AxisAlignedBox
FullDomain = _setup.FullDomain
SamplingMode = _setup.SamplingMode

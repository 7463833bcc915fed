"""Scalar acoustic operator ``H u = u - B((eta - 1) u)`` on the B200.

Mirror of the reference ``src/em3d/acoustics/{problem,materials,kernel,operator}.py``:
``AcousticProblem``, ``make_acoustic_problem``, ``plane_wave_scalar``,
``eta_homogeneous/slab/sphere/ellipsoid``, ``self_cell_coefficient`` and
``AcousticOperator``.  The kernel spectrum (with the equivalent-sphere self
cell) is built in FP64 on the device and stored as one even octant; the
adjoint uses its conjugate, which equals the reference's separately built
``fftn(conj K)``.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import _lib
from . import setup as _setup
from .operator import _Applier, _build_workspace, _uint8, ctypes_ref
from .problem import Grid, _to_device


def self_cell_coefficient(*, k0: float, dv: float) -> complex:
    """``e^{ika}(1 - ika) - 1``, ``a = (3 dv / 4 pi)^(1/3)`` (reference ``acoustics/kernel.py:7-18``)."""
    k = float(k0)
    if k <= 0.0:
        raise ValueError(f"k0 must be positive, got {k0}")
    if float(dv) <= 0.0:
        raise ValueError(f"dv must be positive, got {dv}")
    a = (3.0 * float(dv) / (4.0 * np.pi)) ** (1.0 / 3.0)
    return complex(np.exp(1j * k * a) * (1.0 - 1j * k * a) - 1.0)


def plane_wave_scalar(grid: Grid, *, k: float, direction=(0.0, 0.0, 1.0), amplitude: complex = 1.0):
    host = _setup.plane_wave_scalar_host(grid.host_axes, k=k, direction=direction, amplitude=amplitude,
                                         dtype=grid.backend.complex_dtype)
    return _to_device(grid.backend, host)


def eta_homogeneous(grid: Grid, eta_value):
    return _to_device(grid.backend, _setup.eta_homogeneous(grid.N, eta_value, dtype=grid.backend.complex_dtype))


def eta_slab(grid: Grid, *, eta_inside, eta_outside=1.0, axis: int = 0, width_fraction: float = 0.5):
    host = _setup.eta_slab(grid.host_axes, grid.L, grid.center, eta_inside=eta_inside, eta_outside=eta_outside,
                           axis=axis, width_fraction=width_fraction, dtype=grid.backend.complex_dtype)
    return _to_device(grid.backend, host)


def eta_ellipsoid(grid: Grid, *, center, radii, eta_inside, eta_outside=1.0):
    host = _setup.eta_ellipsoid(grid.host_axes, center=center, radii=radii, eta_inside=eta_inside,
                                eta_outside=eta_outside, dtype=grid.backend.complex_dtype)
    return _to_device(grid.backend, host)


def eta_sphere(grid: Grid, *, center, radius: float, eta_inside, eta_outside=1.0):
    return eta_ellipsoid(grid, center=center, radii=(float(radius),) * 3, eta_inside=eta_inside,
                         eta_outside=eta_outside)


@dataclass(frozen=True)
class AcousticProblem:
    """Grid, scalar eta, incident wave and wave number (reference ``acoustics/problem.py:43-79``)."""

    grid: Grid
    eta: object
    wave: object
    k0: float
    volume: float

    def __post_init__(self) -> None:
        be = self.grid.backend
        expected = tuple(self.grid.N)
        if tuple(getattr(self.eta, "shape", ())) != expected:
            raise ValueError(f"eta.shape {tuple(getattr(self.eta, 'shape', ()))} != expected {expected}")
        if tuple(getattr(self.wave, "shape", ())) != expected:
            raise ValueError(f"wave.shape {tuple(getattr(self.wave, 'shape', ()))} != expected {expected}")
        tc = be.precision.torch_complex
        for name in ("eta", "wave"):
            val = getattr(self, name)
            dt = val.dtype
            ok = (dt == tc) if not isinstance(dt, np.dtype) else (dt == np.dtype(be.complex_dtype))
            if not ok:
                raise TypeError(f"{name}.dtype {dt} != {be.complex_dtype}")
            object.__setattr__(self, name, _to_device(be, val).contiguous())
        if float(self.k0) <= 0.0:
            raise ValueError(f"k0 must be positive, got {self.k0}")
        if float(self.volume) <= 0.0:
            raise ValueError(f"volume must be positive, got {self.volume}")

    @property
    def backend(self):
        return self.grid.backend

    @property
    def chi(self):
        """Acoustic contrast ``eta - 1``."""
        return self.eta - 1.0


def make_acoustic_problem(grid: Grid, eta, *, k0: float, direction=(0.0, 0.0, 1.0), amplitude: complex = 1.0):
    be = grid.backend
    eta_arr = _to_device(be, eta if not isinstance(eta, np.ndarray) else eta.astype(be.complex_dtype),
                         be.precision.torch_complex)
    wave = plane_wave_scalar(grid, k=float(k0), direction=direction, amplitude=amplitude)
    n_cells = int(grid.N[0] * grid.N[1] * grid.N[2])
    return AcousticProblem(grid=grid, eta=eta_arr, wave=wave, k0=float(k0), volume=grid.dv * n_cells)


class AcousticOperator(_Applier):
    """``H u = u - B(chi u)`` and its adjoint (reference ``acoustics/operator.py:25-73``)."""

    _kind = _lib.EM3D_ACOUSTIC
    _native_names = ("em3d_acoustic_matvec", "em3d_acoustic_rmatvec")

    def __init__(self, problem: AcousticProblem, *, _spectrum=None):
        self.problem = problem
        grid = problem.grid
        self._be = grid.backend
        self._N = tuple(grid.N)
        spec = _spectrum
        if spec is None:
            g, ws = _build_workspace(grid)
            dt = self._be.precision.native_dtype
            nbytes = _lib.load().em3d_spectrum_bytes(ctypes_ref(g), _lib.EM3D_ACOUSTIC, dt)
            spec = _uint8(nbytes, self._be.torch_device).zero_()  # alignment padding is deterministic
            _lib.call("em3d_acoustic_spectrum_build", ctypes_ref(g), float(problem.k0), dt, spec.data_ptr(),
                      ws.data_ptr(), ws.numel(), _lib.stream_handle())
            del ws
        self._setup_native(grid, spec, problem.chi)

    @property
    def backend(self):
        return self._be

    @property
    def persistent_nbytes(self) -> int:
        return int(self._spectrum.numel())

    def _field_shape(self):
        return self._N

    def matvec(self, u):
        import torch

        x = self._as_field(u, "u")
        return self._apply_checked(x, torch.empty_like(x))

    def rmatvec(self, v):
        import torch

        x = self._as_field(v, "v")
        return self._apply_checked(x, torch.empty_like(x), adjoint=True)

    def with_precision(self, precision) -> "AcousticOperator":
        """The same operator at another precision (FP32 twin for inner solves);
        its spectrum is this operator's, converted on the device."""
        from .backend import Backend
        from .operator import convert_spectrum

        if precision == self._be.precision:
            return self
        be = Backend.b200(precision, device_index=self._be.device_index)
        g = self.problem.grid
        grid = Grid(N=g.N, L=g.L, center=g.center, backend=be)
        tc = precision.torch_complex
        prob = AcousticProblem(grid=grid, eta=self.problem.eta.to(tc), wave=self.problem.wave.to(tc),
                               k0=self.problem.k0, volume=self.problem.volume)
        spec = convert_spectrum(self._spectrum, grid, _lib.EM3D_ACOUSTIC, self._be.precision, precision)
        return AcousticOperator(prob, _spectrum=spec)

    def kernel_hat(self, adjoint: bool = False):
        """Reference-layout spectrum ``fftn(K)`` (or ``fftn(conj K)``), (2Nx,2Ny,2Nz)."""
        import torch

        grid = self.problem.grid
        g, ws = _build_workspace(grid)
        out = torch.empty(tuple(2 * n for n in grid.N), dtype=self._tc, device=self._be.torch_device)
        _lib.call("em3d_acoustic_kernel_hat_full", ctypes_ref(g), float(self.problem.k0), self._dt, int(adjoint),
                  out.data_ptr(), ws.data_ptr(), ws.numel(), _lib.stream_handle())
        return out

    def to_dense(self):
        raise RuntimeError("AcousticOperator.to_dense requires numpy backend")

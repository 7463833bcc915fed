"""Far field on the B200: the scatter integral and RCS of an EM solution, and
the scalar acoustic far-field amplitude and pattern.

Mirror of the reference ``em3d.farfield`` (``src/em3d/farfield/__init__.py``,
``_core.py``) and ``em3d.acoustics.farfield`` (``src/em3d/acoustics/farfield.py``):
same names, arguments, validation messages and (host NumPy) return values.
The integral runs in one kernel (``em3d_em_farfield`` /
``em3d_acoustic_farfield``) with FP64 phases and sums.  ``method="fft"``
(the reference's oversampled-FFT approximation, accurate to ~1e-4) returns
the exact direct sum here, which is at least as accurate.
"""
from __future__ import annotations

import numpy as np

from . import _lib
from .operator import _uint8, ctypes_ref
from .scenes import device_axes


def _run(kind, chi, u, grid, k0, dirs):
    import torch

    dirs = np.ascontiguousarray(np.asarray(dirs, dtype=np.float64).reshape(-1, 3))
    M = dirs.shape[0]
    be = grid.backend
    dev = be.torch_device
    tc = be.precision.torch_complex
    chi = chi.to(device=dev, dtype=tc).contiguous()
    u = torch.as_tensor(u).to(device=dev, dtype=tc).contiguous()
    g = _lib.make_grid(grid.N, grid.L)
    nb = _lib.load().em3d_farfield_workspace_bytes(ctypes_ref(g), M)
    ws = _uint8(nb, dev)
    d = torch.as_tensor(dirs, device=dev)
    C = 3 if kind == _lib.EM3D_EM else 1
    F = torch.empty((M, C), dtype=torch.complex128, device=dev)
    x, y, z = device_axes(grid)
    name = "em3d_em_farfield" if kind == _lib.EM3D_EM else "em3d_acoustic_farfield"
    _lib.call(name, ctypes_ref(g), be.precision.native_dtype, chi.data_ptr(), u.data_ptr(), x.data_ptr(), y.data_ptr(),
              z.data_ptr(), float(k0), float(grid.dv), M, d.data_ptr(), F.data_ptr(), ws.data_ptr(), ws.numel(),
              _lib.stream_handle())
    out = F.cpu().numpy()
    return out if C == 3 else out[:, 0]


# ----------------------------------------------------------------------- EM
def scatter_integral_direct(u, problem, directions, *, batch_size: int = 64) -> np.ndarray:
    """``F[m] = dV sum_q (chi u)_q exp(-i k0 e_m . r_q)``, (M, 3) complex128 on
    the host (reference ``farfield/_core.py:8-71``; ``batch_size`` is checked
    but the kernel handles all directions together)."""
    directions = np.asarray(directions, dtype=np.float64)
    if directions.ndim != 2 or directions.shape[1] != 3:
        raise ValueError(f"directions must have shape (M, 3), got {directions.shape}")
    if batch_size <= 0:
        raise ValueError(f"batch_size must be positive, got {batch_size}")
    expected = (3,) + tuple(problem.grid.N)
    u_shape = tuple(getattr(u, "shape", ()))
    if u_shape != expected:
        raise ValueError(f"u must have shape {expected}, got {u_shape}")
    if directions.shape[0] == 0:
        return np.zeros((0, 3), dtype=np.complex128)
    return _run(_lib.EM3D_EM, problem.eps_tensor, u, problem.grid, problem.k0, directions)


def scatter_integral(u, problem, directions, *, method: str = "direct", batch_size: int = 64) -> np.ndarray:
    directions = np.asarray(directions, dtype=np.float64)
    if directions.ndim == 1:
        directions = directions[np.newaxis, :]
    if method not in ("direct", "fft"):
        raise ValueError(f"method must be 'direct' or 'fft', got {method!r}")
    return scatter_integral_direct(u, problem, directions, batch_size=batch_size)


def rcs(u, problem, direction) -> float:
    """``k0^4 / (16 pi^2) |e x F(e)|^2`` for one (normalised) direction."""
    direction = np.asarray(direction, dtype=np.float64)
    direction = direction / np.linalg.norm(direction)
    F = scatter_integral(u, problem, direction[np.newaxis, :])[0]
    cross = np.cross(direction, F)
    return problem.k0 ** 4 / (16.0 * np.pi ** 2) * float(np.real(np.dot(cross, cross.conj())))


def plane_directions(n_phi: int, plane: str) -> tuple:
    phi = np.linspace(0.0, 2.0 * np.pi, n_phi, endpoint=False)
    c, s, z = np.cos(phi), np.sin(phi), np.zeros_like(phi)
    if plane == "xy":
        dirs = np.stack([c, s, z], axis=-1)
    elif plane == "yz":
        dirs = np.stack([z, c, s], axis=-1)
    elif plane == "xz":
        dirs = np.stack([c, z, s], axis=-1)
    else:
        raise ValueError(f"plane must be 'xy'|'yz'|'xz', got {plane!r}")
    return phi, dirs


def rcs_plane(u, problem, n_phi: int = 80, plane: str = "xy", method: str = "direct", batch_size: int = 64) -> tuple:
    """RCS over ``n_phi`` directions in a coordinate plane (reference
    ``farfield/__init__.py:86-125``): ``(phi, sigma)``."""
    phi, dirs = plane_directions(n_phi, plane)
    F = scatter_integral(u, problem, dirs, method=method, batch_size=batch_size)
    cross = np.cross(dirs, F)
    sigma = problem.k0 ** 4 / (16.0 * np.pi ** 2) * np.real(np.einsum("mi,mi->m", cross, cross.conj()))
    return phi, sigma


# ----------------------------------------------------------------- acoustic
def _acoustic_directions(directions) -> np.ndarray:
    dirs = np.asarray(directions, dtype=np.float64)
    if dirs.ndim != 2 or dirs.shape[1] != 3:
        raise ValueError(f"directions must have shape (M, 3), got {dirs.shape}")
    norms = np.linalg.norm(dirs, axis=1)
    if np.any(norms == 0.0):
        raise ValueError("directions must be non-zero")
    return dirs / norms[:, None]


def farfield_amplitude(u, problem, directions, *, batch_size: int = 64) -> np.ndarray:
    """``k0^2 dV / (4 pi) sum_q exp(-i k0 s . r_q) chi_q u_q`` for unit ``s``
    (reference ``acoustics/farfield.py:29-60``), (M,) complex128 on the host."""
    dirs = _acoustic_directions(directions)
    if tuple(getattr(u, "shape", ())) != tuple(problem.grid.N):
        raise ValueError(f"u.shape {tuple(getattr(u, 'shape', ()))} != expected {problem.grid.N}")
    if int(batch_size) <= 0:
        raise ValueError(f"batch_size must be positive, got {batch_size!r}")
    if len(dirs) == 0:
        return np.zeros(0, dtype=np.complex128)
    return _run(_lib.EM3D_ACOUSTIC, problem.chi, u, problem.grid, problem.k0, dirs)


def scattering_pattern(u, problem, directions, *, normalize: str | None = "max") -> np.ndarray:
    sigma = np.abs(farfield_amplitude(u, problem, directions)) ** 2
    if normalize is None:
        return sigma.astype(np.float64, copy=False)
    if normalize != "max":
        raise ValueError(f"normalize must be None or 'max', got {normalize!r}")
    peak = float(np.max(sigma)) if sigma.size else 0.0
    if peak > 0.0:
        sigma = sigma / peak
    return sigma.astype(np.float64, copy=False)


def pattern_plane(u, problem, *, plane: str = "xy", n_angles: int = 360, normalize: str | None = "max") -> tuple:
    if int(n_angles) <= 0:
        raise ValueError(f"n_angles must be positive, got {n_angles!r}")
    phi = np.linspace(0.0, 2.0 * np.pi, int(n_angles), endpoint=False)
    if plane == "xy":
        dirs = np.column_stack([np.cos(phi), np.sin(phi), np.zeros_like(phi)])
    elif plane == "xz":
        dirs = np.column_stack([np.cos(phi), np.zeros_like(phi), np.sin(phi)])
    elif plane == "yz":
        dirs = np.column_stack([np.zeros_like(phi), np.cos(phi), np.sin(phi)])
    else:
        raise ValueError(f"plane must be 'xy', 'xz', or 'yz', got {plane!r}")
    return phi, scattering_pattern(u, problem, dirs, normalize=normalize)

"""NumPy restatement of the reference scalar acoustic operator ``H u = u - B(chi u)``.

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).
"""
from __future__ import annotations

import numpy as np

from .em import cell_volume, doubled_offsets, precision_dtypes


def self_cell_coefficient(k0: float, dv: float) -> complex:
    """Equivalent-sphere self term ``e^{ika}(1 - ika) - 1``, ``a = (3 dv / 4 pi)^(1/3)``.

    Restates reference ``src/em3d/acoustics/kernel.py:7-18``.
    """
    k = float(k0)
    if k <= 0.0:
        raise ValueError(f"k0 must be positive, got {k0}")
    if dv <= 0.0:
        raise ValueError(f"dv must be positive, got {dv}")
    a = (3.0 * dv / (4.0 * np.pi)) ** (1.0 / 3.0)
    return complex(np.exp(1j * k * a) * (1.0 - 1j * k * a) - 1.0)


def kernel_on_doubled_grid(N, L, k0: float, precision="double"):
    """``k0^2 dv e^{ikR}/(4 pi R)`` on the doubled grid, self cell replaced.

    Restates reference ``src/em3d/acoustics/kernel.py:21-40``.
    """
    _, cdt = precision_dtypes(precision)
    sx, sy, sz = doubled_offsets(N, L)
    SX, SY, SZ = np.meshgrid(sx, sy, sz, indexing="ij")
    R = np.sqrt(SX * SX + SY * SY + SZ * SZ)
    is_self = R < 1e-15
    Rs = np.where(is_self, np.ones_like(R), R)
    ik = cdt(1j * float(k0))
    dv = cell_volume(N, L)
    g = (float(k0) ** 2) * dv * np.exp(ik * Rs) / (4.0 * np.pi * Rs)
    sv = cdt(self_cell_coefficient(float(k0), dv))
    return np.where(is_self, sv, g).astype(cdt, copy=False)


def kernel_hat(N, L, k0: float, precision="double", adjoint: bool = False):
    """``fftn`` of the (optionally conjugated) kernel.

    Restates ``prep_coeffs_acoustic`` / ``prep_conj_coeffs_acoustic``
    (reference ``src/em3d/acoustics/kernel.py:43-58``).
    """
    _, cdt = precision_dtypes(precision)
    K = kernel_on_doubled_grid(N, L, k0, precision)
    if adjoint:
        K = np.conj(K)
    return np.fft.fftn(K, axes=(-3, -2, -1)).astype(cdt, copy=False)


def _pad(u, N):
    nx, ny, nz = N
    out = np.zeros((2 * nx, 2 * ny, 2 * nz), dtype=u.dtype)
    out[:nx, :ny, :nz] = u
    return out


def matvec(chi, u, khat, N):
    """Restates ``AcousticOperator.matvec`` (reference ``src/em3d/acoustics/operator.py:40-54``)."""
    cdt = khat.dtype
    u = np.asarray(u, dtype=cdt)
    big = np.fft.ifftn(khat * np.fft.fftn(_pad(chi * u, N), axes=(-3, -2, -1)), axes=(-3, -2, -1))
    nx, ny, nz = N
    return (u - big[:nx, :ny, :nz]).astype(cdt, copy=False)


def matvec_streamed(chi, u, N, L, k0: float, adjoint: bool = False, precision: str = "double"):
    """``AcousticOperator.matvec`` / ``rmatvec`` for large grids (256^3: a
    512^3 doubled grid), one spectrum at a time and without the three
    meshgrid coordinate arrays: the same kernel values as
    :func:`kernel_on_doubled_grid` (``R`` from per-axis squares added in the
    same order), its ``fftn`` (of ``conj K`` for the adjoint), one forward
    and one inverse transform of the field.  Restates reference
    ``src/em3d/acoustics/operator.py:40-67`` with ``acoustics/kernel.py:21-58``."""
    from .em import _fftn

    _, cdt = precision_dtypes(precision)
    sx, sy, sz = doubled_offsets(N, L)
    R = np.sqrt(sx[:, None, None] * sx[:, None, None] + sy[None, :, None] * sy[None, :, None]
                + sz[None, None, :] * sz[None, None, :])
    is_self = R < 1e-15
    R[is_self] = 1.0
    ik = cdt(1j * float(k0))
    dv = cell_volume(N, L)
    K = (float(k0) ** 2) * dv * np.exp(ik * R) / (4.0 * np.pi * R)
    del R
    K[is_self] = cdt(self_cell_coefficient(float(k0), dv))
    K = K.astype(cdt, copy=False)
    if adjoint:
        K = np.conj(K)
    khat = _fftn(K).astype(cdt, copy=False)
    del K
    u = np.asarray(u, dtype=cdt)
    src = u if adjoint else chi * u
    big = _fftn(khat * _fftn(_pad(src, N)), inverse=True)
    nx, ny, nz = N
    y = big[:nx, :ny, :nz]
    if adjoint:
        y = np.conj(chi) * y
    return (u - y).astype(cdt, copy=False)


def rmatvec(chi, v, khat_conj, N):
    """Restates ``AcousticOperator.rmatvec`` (reference ``src/em3d/acoustics/operator.py:56-67``)."""
    cdt = khat_conj.dtype
    v = np.asarray(v, dtype=cdt)
    big = np.fft.ifftn(khat_conj * np.fft.fftn(_pad(v, N), axes=(-3, -2, -1)), axes=(-3, -2, -1))
    nx, ny, nz = N
    return (v - np.conj(chi) * big[:nx, :ny, :nz]).astype(cdt, copy=False)


def dense_operator_matrix(chi, N, L, center, k0: float):
    """Dense ``H = I - B diag(chi)`` (reference ``src/em3d/acoustics/dense.py:31-51``)."""
    from .em import grid_axes

    x, y, z = grid_axes(N, L, center, "double")
    X, Y, Z = np.meshgrid(x, y, z, indexing="ij")
    cen = np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=-1)
    dv = cell_volume(N, L)
    R = np.linalg.norm(cen[:, None, :] - cen[None, :, :], axis=-1)
    is_self = R < 1e-15
    Rs = np.where(is_self, 1.0, R)
    k = float(k0)
    B = (k * k) * dv * np.exp(1j * k * Rs) / (4.0 * np.pi * Rs)
    B = np.where(is_self, self_cell_coefficient(k, dv), B)
    c = np.asarray(chi, dtype=np.complex128).reshape(-1)
    return np.eye(B.shape[0], dtype=np.complex128) - B * c[None, :]

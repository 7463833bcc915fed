"""NumPy restatement of the reference EM operator ``A = I - B chi``.

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).

Every function names the reference lines it restates.  Arithmetic follows the
reference operation by operation, including its dtype promotions, so the
SINGLE-precision restatement reproduces the reference's complex64 results and
not merely an FP64 result rounded to FP32.
"""
from __future__ import annotations

import numpy as np


def precision_dtypes(precision: str):
    """``Precision`` -> (real, complex) dtypes (reference ``src/em3d/dtypes.py:9-19``)."""
    if precision == "single":
        return np.float32, np.complex64
    if precision == "double":
        return np.float64, np.complex128
    raise ValueError(f"precision must be 'single' or 'double', got {precision!r}")


def axis(n: int, length: float, centre: float, real_dtype) -> np.ndarray:
    """Cell-centre coordinates along one axis (reference ``src/em3d/grid.py:10-13``)."""
    step = length / n
    start = centre - length / 2 + step / 2
    return np.linspace(start, start + step * (n - 1), n, dtype=real_dtype)


def grid_axes(N, L, center, precision="double"):
    real, _ = precision_dtypes(precision)
    return tuple(axis(int(N[i]), float(L[i]), float(center[i]), real) for i in range(3))


def cell_volume(N, L) -> float:
    """``Grid.dv`` (reference ``src/em3d/grid.py:36-38``)."""
    return (L[0] / N[0]) * (L[1] / N[1]) * (L[2] / N[2])


def doubled_offsets(N, L):
    """Signed cell offsets on the doubled grid in FFT order.

    Restates ``_doubled_offsets`` (reference ``src/em3d/operator.py:16-25``):
    ``[0, d, ..., (n-1) d, -n d, ..., -d]`` per axis.
    """
    out = []
    for n, length in zip(N, L):
        d = length / n
        out.append(np.concatenate([np.arange(n) * d, -(np.arange(n, 0, -1)) * d]))
    return tuple(out)


def kernel_blocks(N, L, k: float, precision="double"):
    """The nine dyadic Green blocks on the doubled grid, shape (3,3,2Nx,2Ny,2Nz).

    Restates ``_kernel_geometry`` + ``_kernel_block_from_geometry`` +
    ``_kernel_tensor_on_doubled_grid`` (reference ``src/em3d/operator.py:28-107``):
    block(r, c) = dv e^{ikr}/(4 pi r) [C1 a_r a_c + C2 delta_rc], with
    C1 = 3/r^2 - 3ik/r - k^2, C2 = k^2 + ik/r - 1/r^2, and the self cell
    replaced by -1/3 on the diagonal and 0 off it.
    """
    geo = kernel_geometry(N, L, k, precision)
    out = np.empty((3, 3) + geo["radius"].shape, dtype=geo["cdt"])
    for r in range(3):
        for c in range(3):
            out[r, c] = kernel_block(geo, r, c)
    return out


def kernel_geometry(N, L, k: float, precision="double"):
    """Distances, self-cell mask and the factors shared by the nine blocks.

    Restates ``_kernel_geometry`` (reference ``src/em3d/operator.py:28-58``)."""
    _, cdt = precision_dtypes(precision)
    sx, sy, sz = doubled_offsets(N, L)
    dv = cell_volume(N, L)
    r2 = sx[:, None, None] ** 2
    r2 = r2 + sy[None, :, None] ** 2
    r2 = r2 + sz[None, None, :] ** 2
    radius = np.sqrt(r2)
    is_self = radius < 1e-15
    radius = np.where(is_self, np.ones_like(radius), radius)
    inv_r = 1.0 / radius
    ik = cdt(1j * k)
    wg = (np.exp(ik * radius) / (4.0 * np.pi * radius) * dv).astype(cdt, copy=False)
    c1 = (3.0 * inv_r * inv_r - 3.0 * ik * inv_r - k * k).astype(cdt, copy=False)
    c2 = (k * k + ik * inv_r - inv_r * inv_r).astype(cdt, copy=False)
    return dict(cdt=cdt, offsets=(sx, sy, sz), radius=radius, is_self=is_self, inv_r=inv_r, wg=wg, c1=c1, c2=c2)


def kernel_block(geo, r: int, c: int):
    """One dyadic block (r, c) on the doubled grid.

    Restates ``_kernel_block_from_geometry`` (reference ``src/em3d/operator.py:61-84``)."""
    shapes = ((-1, 1, 1), (1, -1, 1), (1, 1, -1))
    offsets, inv_r, wg, is_self = geo["offsets"], geo["inv_r"], geo["wg"], geo["is_self"]
    a_r = offsets[r].reshape(shapes[r]) * inv_r
    a_c = offsets[c].reshape(shapes[c]) * inv_r
    blk = wg * geo["c1"] * a_r * a_c
    if r == c:
        blk = blk + wg * geo["c2"]
        blk = np.where(is_self, -1.0 / 3.0, blk)
    else:
        blk = np.where(is_self, 0.0, blk)
    return blk.astype(geo["cdt"], copy=False)


def _fftn(x, inverse: bool = False):
    """``numpy.fft.fftn`` / ``ifftn`` over the last three axes, computed by the
    same pocketfft library through ``scipy.fft`` on every host core (the
    results agree with NumPy's to round-off), so that checks at 128^3 and
    256^3 finish in seconds."""
    import os

    import scipy.fft as sfft

    fn = sfft.ifftn if inverse else sfft.fftn
    return fn(x, axes=(-3, -2, -1), workers=os.cpu_count() or 1)


def matvec_streamed(chi, u, N, L, k: float, adjoint: bool = False, precision: str = "double"):
    """``Operator.matvec`` (``adjoint=False``) or ``Operator.rmatvec`` with the
    explicit adjoint spectrum (``adjoint=True``), with the block spectra built
    one at a time as in ``_build_kernel_hat_streamed`` (reference
    ``src/em3d/operator.py:110-138``) and applied as soon as they exist, so
    that the full (3,3,2N,2N,2N) spectrum is never held (2.4 GB at 128^3).

    matvec (reference ``operator.py:353-363``): ``u - crop(ifftn(sum_c K_rc fftn(pad(chi u)_c)))``;
    rmatvec (``:365-398``): ``v - chi^H crop(ifftn(sum_c fftn(conj K_rc) fftn(pad v)_c))``."""
    _, cdt = precision_dtypes(precision)
    u = np.asarray(u)
    src = u if adjoint else np.einsum("ab...,b...->a...", chi, u)
    spec = [_fftn(_pad(src[c:c + 1], N)[0]) for c in range(3)]
    geo = kernel_geometry(N, L, k, precision)
    acc = [None, None, None]
    for r in range(3):
        for c in range(3):
            blk = kernel_block(geo, r, c)
            if adjoint:
                blk = np.conj(blk)
            term = _fftn(blk).astype(cdt, copy=False) * spec[c]
            acc[r] = term if acc[r] is None else acc[r] + term
            del blk, term
    del geo, spec
    nx, ny, nz = N
    y = np.stack([_fftn(acc[r], inverse=True)[:nx, :ny, :nz] for r in range(3)])
    if adjoint:
        y = np.einsum("ab...,b...->a...", np.conj(chi).swapaxes(0, 1), y)
    return (u - y).astype(cdt, copy=False)


def kernel_hat(N, L, k: float, precision="double", adjoint: bool = False):
    """Spectrum of the dyadic kernel, (3,3,2Nx,2Ny,2Nz).

    Restates ``PreparedEMKernel.build`` with ``build_strategy='standard'``
    (reference ``src/em3d/operator.py:202-211``); ``adjoint=True`` gives the
    explicit adjoint spectrum ``fftn(conj(K))``.
    """
    _, cdt = precision_dtypes(precision)
    blocks = kernel_blocks(N, L, k, precision)
    if adjoint:
        blocks = np.conj(blocks)
    return np.fft.fftn(blocks, axes=(-3, -2, -1)).astype(cdt, copy=False)


def reverse_frequency_axes(block):
    """``F(k) -> F(-k)`` in FFT index order (reference ``src/em3d/operator.py:141-148``)."""
    return np.roll(np.flip(block, axis=(-3, -2, -1)), shift=(1, 1, 1), axis=(-3, -2, -1))


def _pad(field, N):
    """Zero-pad (C,Nx,Ny,Nz) into (C,2Nx,2Ny,2Nz) (reference ``src/em3d/operator.py:282-286``)."""
    nx, ny, nz = N
    out = np.zeros((field.shape[0], 2 * nx, 2 * ny, 2 * nz), dtype=field.dtype)
    out[:, :nx, :ny, :nz] = field
    return out


def _block_apply(khat, xhat):
    """``y_r = sum_c K_rc x_c`` (reference ``src/em3d/operator.py:294-302``)."""
    out = np.zeros_like(xhat)
    for r in range(3):
        acc = None
        for c in range(3):
            term = khat[r, c] * xhat[c]
            acc = term if acc is None else acc + term
        out[r] = acc
    return out


def matvec(chi, u, khat, N):
    """``u - crop(ifftn(K_hat * fftn(pad(chi u))))``.

    Restates ``Operator.matvec`` (reference ``src/em3d/operator.py:353-363``).
    """
    cdt = khat.dtype
    cu = np.einsum("ab...,b...->a...", chi, u)
    spec = np.fft.fftn(_pad(cu, N), axes=(-3, -2, -1))
    big = np.fft.ifftn(_block_apply(khat, spec), axes=(-3, -2, -1))
    nx, ny, nz = N
    return (u - big[:, :nx, :ny, :nz]).astype(cdt, copy=False)


def rmatvec(chi, v, N, *, khat_adjoint=None, khat=None):
    """``v - chi^H crop(ifftn(K_adj * fftn(pad v)))``.

    Restates ``Operator.rmatvec`` (reference ``src/em3d/operator.py:365-398``):
    with ``khat_adjoint`` the explicit adjoint spectrum is used (``:376-380``);
    with ``khat`` the derived adjoint ``conj(K_hat[-k])`` (``:305-317``).
    """
    if khat_adjoint is None and khat is None:
        raise ValueError("need khat_adjoint or khat")
    cdt = (khat_adjoint if khat_adjoint is not None else khat).dtype
    spec = np.fft.fftn(_pad(v, N), axes=(-3, -2, -1))
    if khat_adjoint is not None:
        applied = _block_apply(khat_adjoint, spec)
    else:
        applied = np.zeros_like(spec)
        for r in range(3):
            acc = None
            for c in range(3):
                term = np.conj(reverse_frequency_axes(khat[r, c])) * spec[c]
                acc = term if acc is None else acc + term
            applied[r] = acc
    big = np.fft.ifftn(applied, axes=(-3, -2, -1))
    nx, ny, nz = N
    chi_h = np.conj(chi).swapaxes(0, 1)
    out = v - np.einsum("ab...,b...->a...", chi_h, big[:, :nx, :ny, :nz])
    return out.astype(cdt, copy=False)


# --------------------------------------------------------------------------
# Dense known answers (small grids only)
# --------------------------------------------------------------------------

def flatten_field(field):
    """(3,Nx,Ny,Nz) -> cell-major/component-minor vector (reference ``src/em3d/layout.py:14-28``)."""
    return np.transpose(field, (1, 2, 3, 0)).reshape(-1)


def unflatten_field(vec, N):
    """Inverse of :func:`flatten_field` (reference ``src/em3d/layout.py:31-39``)."""
    return np.transpose(vec.reshape(N[0], N[1], N[2], 3), (3, 0, 1, 2))


def dense_kernel_matrix(N, L, center, k: float):
    """Dense ``B`` in cell-major/component-minor order.

    Restates ``dense_kernel_blocks_backend`` / ``dense_kernel_matrix``
    (reference ``src/em3d/dense.py:35-97``) in complex128.
    """
    x, y, z = grid_axes(N, L, center, "double")
    X, Y, Z = np.meshgrid(x, y, z, indexing="ij")
    cen = np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=-1)
    diff = cen[:, None, :] - cen[None, :, :]
    r = np.linalg.norm(diff, axis=-1)
    is_self = r < 1e-15
    rs = np.where(is_self, 1.0, r)
    a = diff / rs[..., None]
    aa = a[..., :, None] * a[..., None, :]
    ir = 1.0 / rs
    ik = 1j * float(k)
    c1 = 3.0 * ir * ir - 3.0 * ik * ir - k * k
    c2 = k * k + ik * ir - ir * ir
    g = np.exp(ik * rs) / (4.0 * np.pi * rs)
    eye = np.eye(3, dtype=np.complex128)
    blocks = g[..., None, None] * cell_volume(N, L) * (c1[..., None, None] * aa + c2[..., None, None] * eye)
    blocks = np.where(is_self[..., None, None], (-1.0 / 3.0) * eye, blocks)
    cells = cen.shape[0]
    return blocks.transpose(0, 2, 1, 3).reshape(3 * cells, 3 * cells)


def dense_operator_matrix(chi, N, L, center, k: float):
    """Dense ``A = I - B chi`` (reference ``src/em3d/dense.py:180-200``)."""
    B = dense_kernel_matrix(N, L, center, k)
    cells = int(np.prod(N))
    blocks = np.asarray(chi, dtype=np.complex128).transpose(2, 3, 4, 0, 1).reshape(cells, 3, 3)
    C = np.zeros((3 * cells, 3 * cells), dtype=np.complex128)
    idx = np.arange(cells)
    for r in range(3):
        for c in range(3):
            C[3 * idx + r, 3 * idx + c] = blocks[:, r, c]
    return np.eye(3 * cells, dtype=np.complex128) - B @ C


# --------------------------------------------------------------------------
# Crop-equivalence of the symmetric (octant) spectrum used by the GPU path
# --------------------------------------------------------------------------

def kernel_blocks_crop_equivalent(N, L, k: float):
    """Kernel blocks with the index-N plane zeroed along every odd axis.

    Not a reference function: it states the identity the GPU path relies on.
    A cropped circular convolution on the doubled grid only reads kernel
    offsets in (-N, N), never the index-N plane, so zeroing that plane along
    the axes where an off-diagonal block is odd leaves ``matvec`` unchanged
    while making every block exactly even or odd per axis.  Its spectrum is
    then fully described by the octant ``[0..Nx] x [0..Ny] x [0..Nz]``.
    """
    K = kernel_blocks(N, L, k, "double").copy()
    for r in range(3):
        for c in range(3):
            if r == c:
                continue
            for ax in {r, c}:
                sl = [slice(None)] * 3
                sl[ax] = N[ax]
                K[(r, c) + tuple(sl)] = 0.0
    return K

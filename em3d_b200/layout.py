"""Flat vector layout of EM fields: cell-major, component-minor.

The public names and ``ValueError`` texts are the reference's contract
(``src/em3d/layout.py:14-45``); the bodies work on torch tensors (device) and
NumPy arrays (host) alike.  Flat entry ``((ix * Ny + iy) * Nz + iz) * 3 + c``
holds component ``c`` of cell ``(ix, iy, iz)``, the order of the dense block
matrices.
"""
from __future__ import annotations

from math import prod
from typing import Any, Sequence


def _cells(shape: Sequence[int]) -> tuple:
    """``shape`` as three positive ints, else the contract's ``ValueError``."""
    dims = [int(v) for v in shape]
    if len(dims) == 3 and min(dims) > 0:
        return tuple(dims)
    raise ValueError(f"shape must be a positive 3-tuple, got {shape!r}")


def _moved(x: Any, order: tuple) -> Any:
    """Axis permutation for torch (``permute``) or NumPy (``transpose``)."""
    return x.permute(*order) if hasattr(x, "permute") else x.transpose(*order)


def flatten_field(field: Any) -> Any:
    """(3, Nx, Ny, Nz) -> flat vector in (ix, iy, iz, component) order."""
    shape = getattr(field, "shape", None)
    if getattr(field, "ndim", None) == 4 and shape[0] == 3:
        return _moved(field, (1, 2, 3, 0)).reshape(-1)
    raise ValueError(f"field must have shape (3, Nx, Ny, Nz), got {shape!r}")


def unflatten_field(vector: Any, shape: Sequence[int]) -> Any:
    """Inverse of :func:`flatten_field` on a grid of ``shape`` cells."""
    nx, ny, nz = _cells(shape)
    want = 3 * nx * ny * nz
    count = int(vector.numel()) if hasattr(vector, "numel") else int(getattr(vector, "size", -1))
    if getattr(vector, "ndim", None) != 1 or count != want:
        raise ValueError(f"vector must be one-dimensional with {want} entries, got shape "
                         f"{getattr(vector, 'shape', None)!r}")
    field = _moved(vector.reshape(nx, ny, nz, 3), (3, 0, 1, 2))
    return field.contiguous() if hasattr(field, "contiguous") else field


def field_size(shape: Sequence[int]) -> int:
    """Complex unknowns of an EM field on ``shape`` cells."""
    return 3 * prod(_cells(shape))

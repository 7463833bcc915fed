"""Flat (cell-major, component-minor) vector layout (reference ``src/em3d/layout.py:14-45``)."""
from __future__ import annotations

from math import prod
from typing import Any, Sequence


def _normalize_shape(shape: Sequence[int]) -> tuple:
    n = tuple(int(v) for v in shape)
    if len(n) != 3 or any(v <= 0 for v in n):
        raise ValueError(f"shape must be a positive 3-tuple, got {shape!r}")
    return n


def flatten_field(field: Any) -> Any:
    if getattr(field, "ndim", None) != 4 or field.shape[0] != 3:
        raise ValueError(f"field must have shape (3, Nx, Ny, Nz), got {getattr(field, 'shape', None)!r}")
    return field.permute(1, 2, 3, 0).reshape(-1) if hasattr(field, "permute") else field.transpose(1, 2, 3, 0).reshape(-1)


def unflatten_field(vector: Any, shape: Sequence[int]) -> Any:
    Nx, Ny, Nz = _normalize_shape(shape)
    expected = 3 * prod((Nx, Ny, Nz))
    if getattr(vector, "ndim", None) != 1 or int(vector.numel() if hasattr(vector, "numel") else vector.size) != expected:
        raise ValueError(f"vector must be one-dimensional with {expected} entries, got shape "
                         f"{getattr(vector, 'shape', None)!r}")
    v = vector.reshape(Nx, Ny, Nz, 3)
    return v.permute(3, 0, 1, 2).contiguous() if hasattr(v, "permute") else v.transpose(3, 0, 1, 2)


def field_size(shape: Sequence[int]) -> int:
    return 3 * prod(_normalize_shape(shape))

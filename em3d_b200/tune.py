"""Autotuner for the operator passes.

The native library offers equivalent implementations of the x pass (see
``EM3D_TUNE_XPASS_VARIANT`` in ``include/em3d_b200.h``).  ``autotune(op)``
times each on the operator's own grid with CUDA events and keeps the
fastest for the process; results are cached per (grid, dtype, kind).
"""
from __future__ import annotations

from . import _lib

_cache: dict = {}


def set_xpass_variant(v: int) -> None:
    _lib.call("em3d_set_tuning", _lib.EM3D_TUNE_XPASS_VARIANT, int(v))


def get_xpass_variant() -> int:
    return int(_lib.load().em3d_get_tuning(_lib.EM3D_TUNE_XPASS_VARIANT))


def autotune(op, *, reps: int = 10, variants=(0, 1, 2, 3, 4, 5, 6)) -> dict:
    """Time every x-pass variant on ``op`` (an ``Operator`` or
    ``AcousticOperator``) and select the fastest.  Returns {variant: ms}."""
    import torch

    key = (tuple(op.problem.grid.N), op._dt, op._kind)
    if key in _cache:
        set_xpass_variant(_cache[key][0])
        return _cache[key][1]
    x = op._as_field(op.problem.wave)
    out = torch.empty_like(x)
    times = {}
    for v in variants:
        if v == 2 and op._kind != _lib.EM3D_EM:
            continue
        set_xpass_variant(v)
        for _ in range(2):
            op.apply_into(x, out)
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(reps):
            op.apply_into(x, out)
        b.record()
        torch.cuda.synchronize()
        times[v] = a.elapsed_time(b) / reps
    best = min(times, key=times.get)
    set_xpass_variant(best)
    _cache[key] = (best, times)
    return times

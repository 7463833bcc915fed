"""Autotuner for the operator passes.

The native library offers equivalent implementations of the x pass, the pass
that holds the spectrum multiply (``EM3D_TUNE_XPASS_VARIANT`` in
``include/em3d_b200.h``): tile widths (8 or 16 kz columns per CTA), threads
per CTA (128 or 256), radix plans (16 x 16 or 8 x 8 x 4 points on a
256-point axis: 16 or 8 elements per thread), the pipelining of the field and
spectrum slabs (none, cp.async, TMA) and the placement of the stage twiddles;
``"generic"`` is the shared-memory mixed-radix Stockham plan for every axis.
``autotune(op)`` times each on the operator itself with CUDA events and keeps
the fastest on that operator (``op.xpass_variant``); the operator applies it
on every launch, so operators of different grids or precisions keep their
own choice in one process.  Results are cached per (grid, dtype, kind,
batch).
"""
from __future__ import annotations

from . import _lib

_cache: dict = {}

VARIANTS = (0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, "generic")


def set_xpass_variant(v: int) -> None:
    """Process-wide x-pass variant (-1: the library's default per operator)."""
    _lib.call("em3d_set_tuning", _lib.EM3D_TUNE_XPASS_VARIANT, int(v))


def get_xpass_variant() -> int:
    return int(_lib.load().em3d_get_tuning(_lib.EM3D_TUNE_XPASS_VARIANT))


def apply_choice(choice) -> None:
    """Select ``choice`` (a variant number, -1, or ``"generic"``) for the
    launches that follow."""
    generic = choice == "generic"
    lib = _lib.load()
    if int(lib.em3d_get_tuning(_lib.EM3D_TUNE_FFT_GENERIC)) != int(generic):
        _lib.call("em3d_set_tuning", _lib.EM3D_TUNE_FFT_GENERIC, int(generic))
    v = -1 if generic else int(choice)
    if int(lib.em3d_get_tuning(_lib.EM3D_TUNE_XPASS_VARIANT)) != v:
        _lib.call("em3d_set_tuning", _lib.EM3D_TUNE_XPASS_VARIANT, v)


def autotune(op, *, reps: int = 10, variants=VARIANTS, batch: int = 1, rounds: int = 2) -> dict:
    """Time each x-pass choice on ``op`` (an ``Operator``, ``AcousticOperator``
    or operator group) over ``batch`` right-hand sides, store the fastest as
    ``op.xpass_variant`` and return {choice: ms per application}.  The
    choices are timed ``rounds`` times in turn and each keeps its best time,
    so one disturbed measurement does not decide."""
    import torch

    fs = tuple(op._field_shape())
    if hasattr(op, "problems"):  # a group applies to one field per problem
        batch = len(op)
    key = (tuple(op._grid_key()), op._dt, op._kind, batch)
    if key in _cache:
        op.xpass_variant = _cache[key][0]
        return _cache[key][1]
    x = torch.randn((batch,) + fs if batch > 1 else fs, dtype=op._tc, device=op.backend.torch_device)
    out = torch.empty_like(x)
    times = {}
    previous = getattr(op, "xpass_variant", None)
    try:
        for _ in range(max(1, int(rounds))):
            for v in variants:
                if v == 2 and op._kind != _lib.EM3D_EM:
                    continue
                op.xpass_variant = v
                for _ in range(2):
                    op.apply_into(x, out)
                a = torch.cuda.Event(enable_timing=True)
                b = torch.cuda.Event(enable_timing=True)
                a.record()
                for _ in range(reps):
                    op.apply_into(x, out)
                b.record()
                torch.cuda.synchronize()
                ms = a.elapsed_time(b) / reps
                times[v] = min(ms, times.get(v, ms))
    finally:
        op.xpass_variant = previous
        apply_choice(-1)
    best = min(times, key=times.get)
    op.xpass_variant = best
    _cache[key] = (best, times)
    return times

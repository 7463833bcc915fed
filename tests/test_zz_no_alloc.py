"""The allocation-free EM matvec entry point, called through the C ABI.

``em3d_em_matvec_static_scratch`` serves callers that cannot allocate device
memory (for example a host framework that owns every device allocation and
only hands the library its input and output buffers): it keeps its workspace
in a fixed 64 MiB array inside the library.  These tests check that it gives
the same result as the regular ``em3d_em_matvec`` path on two calls in a row
(the shared array keeps the previous call's contents), and that grids too
large for the array are refused before anything is launched.

This file is named so that pytest collects it last.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu


def _operator(N, prec, seed):
    import torch

    import em3d_b200 as e

    be = e.Backend.b200(e.Precision.DOUBLE if prec == "double" else e.Precision.SINGLE)
    grid = e.Grid(N=N, L=(1.0, 0.9, 1.1), center=(0.0, 0.0, 0.0), backend=be)
    gen = torch.Generator(device="cuda").manual_seed(seed)
    tc = be.precision.torch_complex
    chi = (torch.randn((3, 3) + N, dtype=tc, device="cuda", generator=gen) * 0.3).contiguous()
    u = torch.randn((3,) + N, dtype=tc, device="cuda", generator=gen).contiguous()
    op = e.Operator(e.Problem(grid=grid, eps_tensor=chi, wave=u, k0=6.0, volume=1.0))
    return be, op


def _static_call(op, u, out):
    from em3d_b200 import _lib

    g = _lib.make_grid(op.problem.grid.N, op.problem.grid.L)
    chi = op.problem.eps_tensor.contiguous()  # the full (3,3,Nx,Ny,Nz) contrast this entry point takes
    _lib.call("em3d_em_matvec_static_scratch", ctypes.byref(g), op._dt, op._spectrum.data_ptr(),
              chi.data_ptr(), u.data_ptr(), out.data_ptr(), None, _lib.stream_handle())
    return out


@pytest.mark.parametrize("prec,N", [("double", (32, 32, 32)), ("single", (64, 64, 64)), ("double", (24, 20, 16))])
def test_static_scratch_matvec_matches_regular_path_twice(prec, N):
    import torch

    be, op = _operator(N, prec, seed=5)
    tol = 1e-13 if prec == "double" else 1e-6
    for seed in (11, 12):  # two calls in a row on different inputs
        gen = torch.Generator(device="cuda").manual_seed(seed)
        u = torch.randn((3,) + N, dtype=be.precision.torch_complex, device="cuda", generator=gen).contiguous()
        ref = op.matvec(u)
        got = _static_call(op, u, torch.empty_like(u))
        torch.cuda.synchronize()
        assert rel_err(be.to_host(got), be.to_host(ref)) < tol


def test_static_scratch_rejects_grids_beyond_its_size():
    from em3d_b200 import _lib

    lib = _lib.load()
    assert lib.em3d_static_scratch_bytes() == 64 << 20
    g = _lib.make_grid((128, 128, 128), (1.0, 1.0, 1.0))
    with pytest.raises(ValueError, match="64 MiB static scratch"):
        _lib.call("em3d_em_matvec_static_scratch", ctypes.byref(g), _lib.EM3D_C64, 1, 1, 1, 1, None, None)

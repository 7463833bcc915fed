"""Groups of problems on one grid, applied together.

Many independent problems of the same grid size (each with its own contrast
and wave number, hence its own kernel spectrum) are stacked into one operator
whose batch entry ``b`` is problem ``b``: every pass of an application is one
launch for the whole group (``em3d_*_matvec_grouped``).  Any batched solver
takes a group as its operator and the stacked right-hand sides as ``rhs``;
entries whose solve has stopped skip their share of the operator work::

    group = OperatorGroup(problems)                     # same N and L
    results = BiCGStab(cfg).solve_batch(group, group.waves())
    results = DefectCorrection(cfg).solve_batch(group, group.waves())   # FP32 inside FP64

Problems of different grid sizes form one group per size (``group_by_grid``).
The reference solves such sets one problem after another.
"""
from __future__ import annotations

from collections import OrderedDict
from typing import Sequence

import numpy as np

from . import _lib
from .operator import _build_workspace, _uint8, ctypes_ref, raise_on_failed_waits, status_word, tuned


def _align(n: int, a: int = 256) -> int:
    return (n + a - 1) // a * a


class _Group:
    _kind = _lib.EM3D_EM
    _names = ("", "")
    # batched solvers may pass their per-entry status words (entry_done)
    accepts_entry_skip = True

    def __init__(self, problems: Sequence):
        import torch

        problems = list(problems)
        if not problems:
            raise ValueError("a group needs at least one problem")
        g0 = problems[0].grid
        for p in problems[1:]:
            if tuple(p.grid.N) != tuple(g0.N) or tuple(p.grid.L) != tuple(g0.L):
                raise ValueError(f"all problems of a group need the same grid: {p.grid.N}, {p.grid.L} != "
                                 f"{g0.N}, {g0.L}")
            if p.grid.backend.precision != g0.backend.precision or p.grid.backend.device != g0.backend.device:
                raise ValueError("all problems of a group need the same backend (precision and device)")
        self.problems = problems
        self._be = g0.backend
        self._N = tuple(g0.N)
        self._grid_c = _lib.make_grid(g0.N, g0.L)
        self._dt = self._be.precision.native_dtype
        self._tc = self._be.precision.torch_complex
        nbytes = _lib.load().em3d_spectrum_bytes(ctypes_ref(self._grid_c), self._kind, self._dt)
        self._stride = _align(int(nbytes))
        self._spectra = _uint8(self._stride * len(problems), self._be.torch_device)
        g, ws = _build_workspace(g0)
        name = "em3d_em_spectrum_build" if self._kind == _lib.EM3D_EM else "em3d_acoustic_spectrum_build"
        for b, p in enumerate(problems):
            _lib.call(name, ctypes_ref(g), float(p.k0), self._dt, self._spectra.data_ptr() + b * self._stride,
                      ws.data_ptr(), ws.numel(), _lib.stream_handle())
        del ws
        self._chis = torch.stack([self._contrast(p).to(self._tc) for p in problems]).contiguous()
        self._workspaces = {}

    @property
    def backend(self):
        return self._be

    def __len__(self) -> int:
        return len(self.problems)

    def waves(self):
        """The problems' incident fields stacked (the right-hand sides)."""
        import torch

        return torch.stack([p.wave.to(self._tc) for p in self.problems]).contiguous()

    def workspace(self, batch: int):
        ws = self._workspaces.get(batch)
        if ws is None:
            nb = _lib.load().em3d_apply_workspace_bytes(ctypes_ref(self._grid_c), self._kind, self._dt, int(batch))
            if nb == 0:
                _lib.check(_lib.EM3D_ERR_INVALID, "em3d_apply_workspace_bytes")
            ws = _uint8(nb, self._be.torch_device).zero_()  # the status words at its end start at zero
            self._workspaces[batch] = ws
        return ws

    def apply_into(self, x, out, *, adjoint: bool = False, skip_ptr=None, stream=None, entry_done=None):
        """``out[b] = A_b x[b]`` (or ``A_b* x[b]``) for every problem ``b``.
        ``entry_done = (address, stride)``: device ints, entry b's at
        ``address + b * stride``; entries whose int is non-zero are skipped
        (their ``out`` is left as it was)."""
        n = int(np.prod(self._field_shape()))
        if x.numel() != len(self) * n:
            raise ValueError(f"a group of {len(self)} problems applies to {len(self)} fields of shape "
                             f"{self._field_shape()}, got shape {tuple(x.shape)}")
        ws = self.workspace(len(self))
        with tuned(self.xpass_variant):
            _lib.call(self._names[1 if adjoint else 0], ctypes_ref(self._grid_c), self._dt, len(self),
                      self._spectra.data_ptr(), self._stride, self._chis.data_ptr(), x.data_ptr(), out.data_ptr(),
                      ws.data_ptr(), ws.numel(), skip_ptr, entry_done[0] if entry_done else None,
                      int(entry_done[1]) if entry_done else 0, _lib.stream_handle(stream))
        return out

    # x-pass choice of ``em3d_b200.tune.autotune`` (None: the process-wide setting)
    xpass_variant = None

    def _grid_key(self):
        g = self._grid_c
        return (g.nx, g.ny, g.nz, g.lx, g.ly, g.lz)

    def status_word(self, batch: int = 0):
        """Device int32 counting the failed bounded waits of this group's
        applications (every application covers the whole group)."""
        return status_word(self.workspace(len(self)))

    def check_status(self) -> None:
        """Raise ``NativeError`` if an application since the last check lost a transfer."""
        raise_on_failed_waits(list(self._workspaces.values()), type(self).__name__)

    def matvec(self, fields):
        import torch

        x = fields.to(device=self._be.torch_device, dtype=self._tc).contiguous()
        out = self.apply_into(x, torch.empty_like(x))
        self.check_status()
        return out

    def rmatvec(self, fields):
        import torch

        x = fields.to(device=self._be.torch_device, dtype=self._tc).contiguous()
        out = self.apply_into(x, torch.empty_like(x), adjoint=True)
        self.check_status()
        return out

    def true_relative_residuals(self, u, rhs) -> np.ndarray:
        """``||f_b - A_b u_b|| / ||f_b||`` per problem (FP64 norms)."""
        import torch

        r = rhs.to(self._tc) - self.matvec(u)
        num = torch.linalg.vector_norm(r.reshape(len(self), -1).to(torch.complex128), dim=1)
        den = torch.linalg.vector_norm(rhs.reshape(len(self), -1).to(torch.complex128), dim=1)
        return (num / den).cpu().numpy()

    def with_precision(self, precision):
        """The same group at another precision (spectra rebuilt from the FP64 sampling)."""
        if precision == self._be.precision:
            return self
        return type(self)([self._cast(p, precision) for p in self.problems])


class OperatorGroup(_Group):
    """EM operators ``A_b = I - B_b chi_b`` of problems on one grid."""

    _kind = _lib.EM3D_EM
    _names = ("em3d_em_matvec_grouped", "em3d_em_rmatvec_grouped")

    @staticmethod
    def _contrast(p):
        return p.eps_tensor

    def _field_shape(self):
        return (3,) + self._N

    @staticmethod
    def _cast(p, precision):
        from .backend import Backend
        from .problem import Grid, Problem

        be = Backend.b200(precision, device_index=p.grid.backend.device_index)
        grid = Grid(N=p.grid.N, L=p.grid.L, center=p.grid.center, backend=be)
        tc = precision.torch_complex
        return Problem(grid=grid, eps_tensor=p.eps_tensor.to(tc), wave=p.wave.to(tc), k0=p.k0, volume=p.volume)


class AcousticOperatorGroup(_Group):
    """Acoustic operators ``H_b = I - B_b chi_b`` of problems on one grid."""

    _kind = _lib.EM3D_ACOUSTIC
    _names = ("em3d_acoustic_matvec_grouped", "em3d_acoustic_rmatvec_grouped")

    @staticmethod
    def _contrast(p):
        return p.chi

    def _field_shape(self):
        return self._N

    @staticmethod
    def _cast(p, precision):
        from .acoustics import AcousticProblem
        from .backend import Backend
        from .problem import Grid

        be = Backend.b200(precision, device_index=p.grid.backend.device_index)
        grid = Grid(N=p.grid.N, L=p.grid.L, center=p.grid.center, backend=be)
        tc = precision.torch_complex
        return AcousticProblem(grid=grid, eta=p.eta.to(tc), wave=p.wave.to(tc), k0=p.k0, volume=p.volume)


def group_by_grid(problems: Sequence, acoustic: bool = False) -> "OrderedDict":
    """{(N, L): (indices, group)} for a list of problems of mixed grid sizes."""
    buckets = OrderedDict()
    for i, p in enumerate(problems):
        buckets.setdefault((tuple(p.grid.N), tuple(p.grid.L)), []).append(i)
    cls = AcousticOperatorGroup if acoustic else OperatorGroup
    return OrderedDict((k, (idx, cls([problems[i] for i in idx]))) for k, idx in buckets.items())


class GroupedSolver:
    """Solves a list of problems of mixed grid sizes: one group per size, each
    group solved as one batch by its own solver, the groups' solves on their
    own CUDA streams at the same time (one host thread each), so small grids
    run alongside large ones.  Results come back in the input order.

        gs = GroupedSolver(problems, lambda: MixedBiCGStab(cfg), low_precision=Precision.SINGLE)
        results = gs.solve()

    ``make_solver`` builds one solver per group (solvers keep per-operator
    caches and are not shared between threads); ``low_precision`` builds each
    group's twin for the mixed solvers' ``operator_low``.
    """

    def __init__(self, problems, make_solver, *, acoustic: bool = False, low_precision=None):
        import torch

        self.problems = list(problems)
        self.groups = group_by_grid(self.problems, acoustic=acoustic)
        self.solvers = {k: make_solver() for k in self.groups}
        self.lows = ({k: g.with_precision(low_precision) for k, (_, g) in self.groups.items()}
                     if low_precision is not None else {})
        self.streams = {k: torch.cuda.Stream(device=g.backend.torch_device) for k, (_, g) in self.groups.items()}

    def _solve_group(self, key):
        idx, group = self.groups[key]
        kw = {"operator_low": self.lows[key]} if key in self.lows else {}
        return idx, self.solvers[key].solve_batch(group, group.waves(), **kw)

    def solve(self, concurrent: bool = True) -> list:
        import threading

        import torch

        out = [None] * len(self.problems)
        if not concurrent or len(self.groups) == 1:
            for key in self.groups:
                idx, res = self._solve_group(key)
                for i, r in zip(idx, res):
                    out[i] = r
            return out
        caller = torch.cuda.current_stream()
        errors = []

        def work(key):
            try:
                stream = self.streams[key]
                stream.wait_stream(caller)
                with torch.cuda.stream(stream):
                    idx, res = self._solve_group(key)
                for r in res:
                    # the results are used on the caller's stream from here on
                    if isinstance(getattr(r, "u", None), torch.Tensor):
                        r.u.record_stream(caller)
                stream.synchronize()
                for i, r in zip(idx, res):
                    out[i] = r
            except BaseException as exc:  # re-raised in the calling thread
                errors.append(exc)

        threads = [threading.Thread(target=work, args=(key,)) for key in self.groups]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        if errors:
            raise errors[0]
        for stream in self.streams.values():
            caller.wait_stream(stream)
        return out

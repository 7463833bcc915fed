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

Problems of different grid sizes form one group per size (``group_by_grid``),
or all of them one :class:`UnevenGroup`, whose every pass is one launch over
all sizes.  The reference solves such sets one problem after another.
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


class UnevenGroup:
    """Problems of uneven grid sizes applied together: each of the five passes
    of an application is ONE launch over every problem (``em3d_*_uneven``); a
    CTA finds the segment (grid size) its index falls in and runs that size's
    register FFT.  Up to ``EM3D_MAX_SEGMENTS`` (8) sizes, each doubled axis a
    length ``em3d_uneven_supported`` accepts (32..256: powers of two, 96, 160,
    192).

    Entry ``b`` is problem ``order[b]`` of the list given (the problems sorted
    by grid, so that each size is one run of entries).  Fields are stacked
    as rows of one length ``n`` (the largest problem's field): problem b's
    field, flattened, at the start of row b, zeros after it.  The solvers
    read ``entry_lengths`` and leave that padding alone, so a batched solve
    works on this group like on a group of one grid::

        group = UnevenGroup(problems)
        low = group.with_precision(Precision.SINGLE)
        results = MixedBiCGStab(cfg).solve_batch(group, group.waves(), operator_low=low)
        results[b].u                  # problem order[b]'s solution, shape (3, *N_b)

    The reference solves such sets one problem after another (one ``Operator``
    per problem, ``src/em3d/operator.py:320-428``)."""

    accepts_entry_skip = True
    # x-pass autotuning does not apply (the uneven x pass has one implementation)
    xpass_variant = None

    def __init__(self, problems: Sequence, acoustic: bool = False, *, _spectra=None):
        import torch

        problems = list(problems)
        if not problems:
            raise ValueError("an uneven group needs at least one problem")
        self._acoustic = bool(acoustic)
        self._kind = _lib.EM3D_ACOUSTIC if acoustic else _lib.EM3D_EM
        self._C = 1 if acoustic else 3
        be = problems[0].grid.backend
        for p in problems[1:]:
            if p.grid.backend.precision != be.precision or p.grid.backend.device != be.device:
                raise ValueError("all problems of a group need the same backend (precision and device)")
        self._be = be
        self._dt = be.precision.native_dtype
        self._tc = be.precision.torch_complex
        lib = _lib.load()

        def key(i):
            g = problems[i].grid
            return tuple(g.N), tuple(g.L)

        self.order = sorted(range(len(problems)), key=key)
        self.problems = [problems[i] for i in self.order]
        runs = []  # [key, first entry, count]
        for b, i in enumerate(self.order):
            if runs and runs[-1][0] == key(i):
                runs[-1][2] += 1
            else:
                runs.append([key(i), b, 1])
        if len(runs) > _lib.EM3D_MAX_SEGMENTS:
            raise ValueError(f"an uneven group takes at most {_lib.EM3D_MAX_SEGMENTS} grid sizes, got {len(runs)}")
        self._sizes = [self._C * int(np.prod(p.grid.N)) for p in self.problems]
        self.n = max(self._sizes)
        self._esz = 8 if self._dt == _lib.EM3D_C64 else 16
        # contrast storage shared by all segments: the smallest exact one that
        # fits every problem (isotropic 1 < symmetric 6 < full 9 per cell)
        if acoustic:
            self._layout = 1
            chis = [p.chi.to(self._tc) for p in self.problems]
        else:
            from .operator import compact_contrast

            self._layout = max(compact_contrast(p.eps_tensor)[0] for p in self.problems)
            chis = [self._store_contrast(p.eps_tensor.to(self._tc), self._layout) for p in self.problems]
        self._segments = []
        for s, ((N, L), b0, count) in enumerate(runs):
            g = _lib.make_grid(N, L)
            if not lib.em3d_uneven_supported(ctypes_ref(g), self._kind, self._dt):
                raise ValueError(f"grid {N} cannot join an uneven application (see em3d_uneven_supported)")
            nbytes = int(lib.em3d_spectrum_bytes(ctypes_ref(g), self._kind, self._dt))
            stride = _align(nbytes)
            if _spectra is not None:
                spec = _spectra[s]
            else:
                spec = _uint8(stride * count, be.torch_device).zero_()
                gb, ws = _build_workspace(self.problems[b0].grid)
                name = "em3d_em_spectrum_build" if not acoustic else "em3d_acoustic_spectrum_build"
                for j in range(count):
                    _lib.call(name, ctypes_ref(gb), float(self.problems[b0 + j].k0), self._dt,
                              spec.data_ptr() + j * stride, ws.data_ptr(), ws.numel(), _lib.stream_handle())
                del ws
            chi = torch.stack(chis[b0:b0 + count]).contiguous()
            self._segments.append({"grid": g, "N": N, "L": L, "first": b0, "count": count, "spectra": spec,
                                   "stride": stride, "chi": chi, "chi_stride": chi[0].numel() * self._esz})
        self._workspace = None

    @staticmethod
    def _store_contrast(c, layout):
        if layout == _lib.EM3D_CHI_ISOTROPIC:
            return c[0, 0].contiguous()
        if layout == _lib.EM3D_CHI_SYMMETRIC:
            import torch

            return torch.stack([c[0, 0], c[1, 1], c[2, 2], c[0, 1], c[0, 2], c[1, 2]]).contiguous()
        return c.contiguous()

    @property
    def backend(self):
        return self._be

    @property
    def chi_layout(self) -> str:
        return {1: "isotropic", 6: "symmetric", 9: "full"}[self._layout]

    def __len__(self) -> int:
        return len(self.problems)

    def _field_shape(self):
        return (self.n,)

    @property
    def entry_lengths(self):
        """Elements of each entry's row in use (its problem's field)."""
        return list(self._sizes)

    def problem_shape(self, b: int):
        N = tuple(self.problems[b].grid.N)
        return N if self._acoustic else (3,) + N

    def entry_field(self, rows, b: int):
        """Problem ``order[b]``'s field inside row ``b`` of ``rows`` (a view)."""
        return rows[b, :self._sizes[b]].view(self.problem_shape(b))

    def pack(self, fields):
        """Rows (batch, n) holding ``fields[b]`` (entry order), zero-padded."""
        import torch

        out = torch.zeros((len(self), self.n), dtype=self._tc, device=self._be.torch_device)
        for b, f in enumerate(fields):
            out[b, :self._sizes[b]] = torch.as_tensor(f).to(device=out.device, dtype=self._tc).reshape(-1)
        return out

    def waves(self):
        """The problems' incident fields as zero-padded rows (the right-hand sides)."""
        return self.pack([p.wave for p in self.problems])

    def _segment_array(self, x, out, entry_done=None):
        segs = (_lib.Segment * len(self._segments))()
        row = self.n * self._esz
        for i, s in enumerate(self._segments):
            sg = segs[i]
            sg.grid = s["grid"]
            sg.count = s["count"]
            sg.chi_layout = self._layout
            sg.spectra = s["spectra"].data_ptr()
            sg.spectrum_stride = s["stride"]
            sg.chi = s["chi"].data_ptr()
            sg.chi_stride = s["chi_stride"]
            sg.u = x.data_ptr() + s["first"] * row if x is not None else None
            sg.out = out.data_ptr() + s["first"] * row if out is not None else None
            sg.field_stride = row
            if entry_done is not None:
                sg.entry_done = int(entry_done[0]) + s["first"] * int(entry_done[1])
                sg.entry_done_stride = int(entry_done[1])
        return segs

    def workspace(self, batch: int = 0):
        """The application workspace (one for every batch: the group is the batch)."""
        if self._workspace is None:
            segs = self._segment_array(None, None)
            nb = _lib.load().em3d_uneven_workspace_bytes(self._kind, self._dt, len(self._segments), segs)
            if nb == 0:
                _lib.check(_lib.EM3D_ERR_INVALID, "em3d_uneven_workspace_bytes")
            self._workspace = _uint8(nb, self._be.torch_device).zero_()
        return self._workspace

    def apply_into(self, x, out, *, adjoint: bool = False, skip_ptr=None, stream=None, entry_done=None):
        """``out[b] = A_b x[b]`` (or ``A_b* x[b]``) on every row's problem part;
        the padding of ``out`` is left as it was."""
        if x.numel() != len(self) * self.n or out.numel() != len(self) * self.n:
            raise ValueError(f"an uneven group of {len(self)} problems applies to rows ({len(self)}, {self.n}), "
                             f"got shape {tuple(x.shape)}")
        if not (x.is_contiguous() and out.is_contiguous()):
            raise ValueError("uneven group fields must be contiguous")
        ws = self.workspace()
        segs = self._segment_array(x, out, entry_done)
        name = ("em3d_acoustic_" if self._acoustic else "em3d_em_") + ("rmatvec_uneven" if adjoint else "matvec_uneven")
        _lib.call(name, self._dt, len(self._segments), segs, ws.data_ptr(), ws.numel(), skip_ptr,
                  _lib.stream_handle(stream))
        return out

    def _grid_key(self):
        return tuple((s["grid"].nx, s["grid"].ny, s["grid"].nz) for s in self._segments)

    def status_word(self, batch: int = 0):
        return status_word(self.workspace())

    def check_status(self) -> None:
        raise_on_failed_waits([self.workspace()], type(self).__name__)

    def _rows(self, fields):
        import torch

        x = torch.as_tensor(fields).to(device=self._be.torch_device, dtype=self._tc)
        return x.reshape(len(self), self.n).contiguous()

    def matvec(self, rows):
        import torch

        x = self._rows(rows)
        out = self.apply_into(x, torch.zeros_like(x))
        self.check_status()
        return out

    def rmatvec(self, rows):
        import torch

        x = self._rows(rows)
        out = self.apply_into(x, torch.zeros_like(x), adjoint=True)
        self.check_status()
        return out

    def true_relative_residuals(self, u, rhs) -> np.ndarray:
        """``||f_b - A_b u_b|| / ||f_b||`` per entry (FP64 norms; the padding is zero)."""
        import torch

        f = self._rows(rhs)
        r = f - self.matvec(u)
        num = torch.linalg.vector_norm(r.to(torch.complex128), dim=1)
        den = torch.linalg.vector_norm(f.to(torch.complex128), dim=1)
        return (num / den).cpu().numpy()

    def with_precision(self, precision):
        """The same group at another precision; the spectra are converted on the
        device (the bytes equal a build in that precision)."""
        from .operator import convert_spectrum

        if precision == self._be.precision:
            return self
        cast = OperatorGroup._cast if not self._acoustic else AcousticOperatorGroup._cast
        problems = [cast(p, precision) for p in self.problems]
        lib = _lib.load()
        spectra = []
        for s in self._segments:
            g = s["grid"]
            nb = int(lib.em3d_spectrum_bytes(ctypes_ref(g), self._kind, precision.native_dtype))
            stride = _align(nb)
            buf = _uint8(stride * s["count"], self._be.torch_device).zero_()
            grid = self.problems[s["first"]].grid
            for j in range(s["count"]):
                src = s["spectra"][j * s["stride"]:j * s["stride"] + s["stride"]]
                conv = convert_spectrum(src, grid, self._kind, self._be.precision, precision)
                buf[j * stride:j * stride + conv.numel()] = conv
            spectra.append(buf)
        twin = UnevenGroup(problems, self._acoustic, _spectra=spectra)
        return twin


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

    ``single_launch=True`` puts every problem into one :class:`UnevenGroup`
    instead: one batched solve whose every operator pass is one launch over
    all sizes (grids the uneven application supports, at most eight sizes).
    """

    def __init__(self, problems, make_solver, *, acoustic: bool = False, low_precision=None,
                 single_launch: bool = False):
        import torch

        self.problems = list(problems)
        if single_launch:
            uneven = UnevenGroup(self.problems, acoustic=acoustic)
            self.groups = OrderedDict([("uneven", (list(uneven.order), uneven))])
        else:
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

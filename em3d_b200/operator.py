"""EM operator ``A = I - B chi`` on the B200: ``PreparedEMKernel`` and ``Operator``.

Drop-in mirror of the reference ``src/em3d/operator.py:151-428``:

* ``PreparedEMKernel.build(grid, *, k, include_adjoint=True,
  adjoint_storage="explicit"|"derived", build_strategy="standard"|"streamed")``
  samples the dyadic Green kernel and transforms it in FP64 on the device
  (``em3d_em_spectrum_build``) and keeps one symmetric octant of the spectrum
  in the operator precision.  Because the stored blocks are exactly even or
  odd per axis, the adjoint spectrum ``conj(K_hat(-k))`` equals
  ``conj(K_hat(k))``: the explicit and the derived adjoint storages share the
  same bytes, and ``persistent_nbytes`` is about 1/12 of the reference's.
  ``kernel_hat`` / ``kernel_hat_adjoint`` materialise the reference's full
  (3,3,2Nx,2Ny,2Nz) spectra on demand.
* ``Operator(problem, *, prepared_kernel=None)`` applies ``matvec`` /
  ``rmatvec`` through the five fused passes of ``em3d_em_matvec`` /
  ``em3d_em_rmatvec``; fields may carry leading batch dimensions.
"""
from __future__ import annotations

import threading
from dataclasses import dataclass, field
from math import prod
from typing import Literal

import numpy as np

from . import _lib
from .problem import Grid, Problem

AdjointStorage = Literal["explicit", "derived", "none"]
KernelBuildStrategy = Literal["standard", "streamed"]


def _uint8(nbytes, device):
    import torch

    return torch.empty(max(int(nbytes), 1), dtype=torch.uint8, device=device)


def convert_spectrum(spectrum, grid: Grid, kind: int, src_precision, dst_precision):
    """A prepared spectrum buffer converted to ``dst_precision`` on the device."""
    g = _lib.make_grid(grid.N, grid.L)
    nbytes = _lib.load().em3d_spectrum_bytes(ctypes_ref(g), kind, dst_precision.native_dtype)
    if nbytes == 0:
        _lib.check(_lib.EM3D_ERR_INVALID, "em3d_spectrum_bytes")
    out = _uint8(nbytes, spectrum.device).zero_()  # alignment padding is deterministic
    _lib.call("em3d_spectrum_convert", ctypes_ref(g), kind, src_precision.native_dtype, spectrum.data_ptr(),
              dst_precision.native_dtype, out.data_ptr(), _lib.stream_handle())
    return out


def compact_contrast(chi):
    """``(layout, tensor)``: the EM contrast (3,3,Nx,Ny,Nz) in the smallest
    storage that holds it exactly: isotropic ``chi = s I`` as s (Nx,Ny,Nz),
    symmetric ``chi = chi^T`` as (6,Nx,Ny,Nz) (xx yy zz xy xz yz), otherwise
    the full tensor.  The passes that apply chi then read 1/9 or 6/9 of its
    bytes; the problem keeps the full tensor."""
    import torch

    c = chi
    symmetric = all(torch.equal(c[a, b], c[b, a]) for a, b in ((0, 1), (0, 2), (1, 2)))
    if not symmetric:
        return _lib.EM3D_CHI_FULL, c.contiguous()
    diagonal = not any(bool(torch.any(c[a, b] != 0)) for a, b in ((0, 1), (0, 2), (1, 2)))
    if diagonal and torch.equal(c[0, 0], c[1, 1]) and torch.equal(c[0, 0], c[2, 2]):
        return _lib.EM3D_CHI_ISOTROPIC, c[0, 0].contiguous()
    return _lib.EM3D_CHI_SYMMETRIC, torch.stack([c[0, 0], c[1, 1], c[2, 2], c[0, 1], c[0, 2], c[1, 2]]).contiguous()


class tuned:
    """Context that selects an operator's autotuned x-pass choice for the
    launches inside it and restores the process-wide setting afterwards
    (``None``: leave the setting alone)."""

    def __init__(self, choice):
        self.choice = choice
        self.saved = None

    def __enter__(self):
        if self.choice is not None:
            from .tune import apply_choice

            lib = _lib.load()
            self.saved = (int(lib.em3d_get_tuning(_lib.EM3D_TUNE_XPASS_VARIANT)),
                          int(lib.em3d_get_tuning(_lib.EM3D_TUNE_FFT_GENERIC)))
            apply_choice(self.choice)
        return self

    def __exit__(self, *exc):
        if self.saved is not None:
            _lib.call("em3d_set_tuning", _lib.EM3D_TUNE_XPASS_VARIANT, self.saved[0])
            _lib.call("em3d_set_tuning", _lib.EM3D_TUNE_FFT_GENERIC, self.saved[1])
        return False


def _build_workspace(grid: Grid):
    g = _lib.make_grid(grid.N, grid.L)
    nb = _lib.load().em3d_build_workspace_bytes(ctypes_ref(g))
    if nb == 0:
        _lib.check(_lib.EM3D_ERR_INVALID, "em3d_build_workspace_bytes")
    return g, _uint8(nb, grid.backend.torch_device)


def ctypes_ref(obj):
    import ctypes

    return ctypes.byref(obj)


# The last bytes of an apply workspace hold status words; the int32 at their
# start counts the bounded waits inside the passes that gave up (a transfer
# into shared memory that never completed; the application is then invalid).
STATUS_BYTES = 256


def status_word(ws):
    """int32 view (one element) of the give-up count of apply workspace ``ws``."""
    import torch

    n = ws.numel()
    return ws[n - STATUS_BYTES:n - STATUS_BYTES + 4].view(torch.int32)


_status_reads = threading.local()


def _read_int32(v) -> int:
    """The int32 at device view ``v``, read through a pinned word by a kernel
    on the current stream (``em3d_copy_small``) rather than a copy engine,
    where it could wait behind a large host transfer of another stream."""
    import torch

    buf = getattr(_status_reads, "buf", None)
    if buf is None:
        buf = torch.zeros(4, dtype=torch.int32).pin_memory()
        _status_reads.buf = buf
    stream = torch.cuda.current_stream(v.device)
    _lib.call("em3d_copy_small", buf.data_ptr(), v.data_ptr(), 4, stream.cuda_stream)
    stream.synchronize()
    return int(buf[0])


def raise_on_failed_waits(workspaces, what: str, counts=None) -> None:
    """Raise ``NativeError`` when a workspace's give-up count is non-zero.

    ``counts`` (optional) are values already read on the host, one per
    workspace, so callers that synchronise anyway need no further read.  The
    count is reset to zero before raising, so the operator stays usable."""
    for i, ws in enumerate(workspaces):
        v = status_word(ws)
        n = _read_int32(v) if counts is None else int(counts[i])
        if n:
            v.zero_()
            raise _lib.NativeError(
                f"{what}: {n} bounded wait(s) inside the operator passes gave up (a transfer into shared memory "
                f"did not complete); the result of this application is invalid")


@dataclass(frozen=True)
class PreparedEMKernel:
    """Reusable spectrum of the EM convolution kernel for one (grid, k, device, precision)."""

    grid_shape: tuple
    grid_lengths: tuple
    wave_number: float
    device: str
    precision: str
    spectrum: object = field(repr=False)
    adjoint_storage: AdjointStorage = "explicit"
    build_strategy: KernelBuildStrategy = "standard"
    _backend: object = field(default=None, repr=False, compare=False)
    _cache: dict = field(default_factory=dict, repr=False, compare=False)

    @classmethod
    def build(cls, grid: Grid, *, k: float, include_adjoint: bool = True,
              adjoint_storage: Literal["explicit", "derived"] = "explicit",
              build_strategy: KernelBuildStrategy = "standard") -> "PreparedEMKernel":
        if build_strategy not in {"standard", "streamed"}:
            raise ValueError(f"build_strategy must be 'standard' or 'streamed', got {build_strategy!r}")
        if adjoint_storage not in {"explicit", "derived"}:
            raise ValueError(f"adjoint_storage must be 'explicit' or 'derived', got {adjoint_storage!r}")
        storage = adjoint_storage if include_adjoint else "none"
        be = grid.backend
        g, ws = _build_workspace(grid)
        dt = be.precision.native_dtype
        nbytes = _lib.load().em3d_spectrum_bytes(ctypes_ref(g), _lib.EM3D_EM, dt)
        spec = _uint8(nbytes, be.torch_device).zero_()  # alignment padding is deterministic
        _lib.call("em3d_em_spectrum_build", ctypes_ref(g), float(k), dt, spec.data_ptr(), ws.data_ptr(),
                  ws.numel(), _lib.stream_handle())
        del ws
        return cls(grid_shape=tuple(int(n) for n in grid.N), grid_lengths=tuple(float(v) for v in grid.L),
                   wave_number=float(k), device=str(be.device), precision=str(be.precision.value),
                   spectrum=spec, adjoint_storage=storage, build_strategy=build_strategy, _backend=be)

    @property
    def supports_adjoint(self) -> bool:
        return self.adjoint_storage != "none"

    @property
    def persistent_nbytes(self) -> int:
        """Device bytes this kernel holds: the octant spectrum, plus the full
        reference-layout spectra once ``kernel_hat`` / ``kernel_hat_adjoint``
        have materialised them (see :meth:`release_full_spectra`)."""
        return int(self.spectrum.numel()) + sum(int(t.numel() * t.element_size()) for t in self._cache.values())

    def release_full_spectra(self) -> None:
        """Drop the cached full spectra (the operator never reads them)."""
        self._cache.clear()

    def _full(self, adjoint: bool):
        import torch

        key = "adjoint" if adjoint else "forward"
        if key not in self._cache:
            be = self._backend
            N = self.grid_shape
            g = _lib.make_grid(N, self.grid_lengths)
            nb = _lib.load().em3d_build_workspace_bytes(ctypes_ref(g))
            ws = _uint8(nb, be.torch_device)
            out = torch.empty((3, 3) + tuple(2 * n for n in N), dtype=be.precision.torch_complex,
                              device=be.torch_device)
            _lib.call("em3d_em_kernel_hat_full", ctypes_ref(g), self.wave_number, be.precision.native_dtype,
                      int(adjoint), out.data_ptr(), ws.data_ptr(), ws.numel(), _lib.stream_handle())
            self._cache[key] = out
        return self._cache[key]

    @property
    def kernel_hat(self):
        """Reference-layout spectrum ``fftn(K)``, (3,3,2Nx,2Ny,2Nz), built on first access."""
        return self._full(False)

    @property
    def kernel_hat_adjoint(self):
        """``fftn(conj K)`` when the kernel was built with the explicit adjoint storage, else None."""
        if self.adjoint_storage != "explicit":
            return None
        return self._full(True)

    def validate(self, grid: Grid, *, k: float) -> None:
        errors = []
        if tuple(grid.N) != self.grid_shape:
            errors.append(f"grid shape {grid.N!r} != {self.grid_shape!r}")
        if not np.allclose(grid.L, self.grid_lengths, rtol=0.0, atol=0.0):
            errors.append(f"grid lengths {grid.L!r} != {self.grid_lengths!r}")
        if not np.isclose(float(k), self.wave_number, rtol=1e-14, atol=1e-14):
            errors.append(f"wave number {k!r} != {self.wave_number!r}")
        if grid.backend.device != self.device:
            errors.append(f"device {grid.backend.device!r} != {self.device!r}")
        if grid.backend.precision.value != self.precision:
            errors.append(f"precision {grid.backend.precision.value!r} != {self.precision!r}")
        if errors:
            raise ValueError("incompatible PreparedEMKernel: " + "; ".join(errors))


def prep_coeffs_em3d(grid: Grid, *, k: float, volume=None):
    """``PreparedEMKernel.build(grid, k=k, include_adjoint=False).kernel_hat``."""
    return PreparedEMKernel.build(grid, k=k, include_adjoint=False).kernel_hat


def prep_conj_coeffs_em3d(grid: Grid, *, k: float, volume=None):
    return PreparedEMKernel.build(grid, k=k, include_adjoint=True, adjoint_storage="explicit").kernel_hat_adjoint


class _Applier:
    """Shared plumbing of the EM and acoustic operators: field checks,
    workspace per batch size, native calls."""

    _kind = _lib.EM3D_EM

    def _setup_native(self, grid: Grid, spectrum, chi, chi_layout: int = 9):
        self._grid_c = _lib.make_grid(grid.N, grid.L)
        self._spectrum = spectrum
        self._chi = chi.contiguous()
        self._chi_layout = int(chi_layout)
        self._workspaces = {}
        self._dt = self._be.precision.native_dtype
        self._tc = self._be.precision.torch_complex

    def _field_shape(self):
        raise NotImplementedError

    def status_word(self, batch: int = 1):
        """Device int32 counting the failed bounded waits of applications over
        ``batch`` right-hand sides (see :func:`raise_on_failed_waits`)."""
        return status_word(self.workspace(batch))

    def check_status(self) -> None:
        """Raise ``NativeError`` if an application since the last check lost a
        transfer (reads the status words on the host: one synchronisation)."""
        raise_on_failed_waits(list(self._workspaces.values()), type(self).__name__)

    def workspace(self, batch: int):
        ws = self._workspaces.get(batch)
        if ws is None:
            nb = _lib.load().em3d_apply_workspace_bytes(ctypes_ref(self._grid_c), self._kind, self._dt, int(batch))
            if nb == 0:
                _lib.check(_lib.EM3D_ERR_INVALID, "em3d_apply_workspace_bytes")
            ws = _uint8(nb, self._be.torch_device).zero_()  # the status words at its end start at zero
            self._workspaces[batch] = ws
        return ws

    def _as_field(self, x, name="field"):
        import torch

        fs = self._field_shape()
        if not isinstance(x, torch.Tensor):
            x = torch.as_tensor(np.asarray(x))
        if tuple(x.shape[-len(fs):]) != fs:
            raise ValueError(f"{name}.shape {tuple(x.shape)} != expected (..., {', '.join(map(str, fs))})")
        x = x.to(device=self._be.torch_device, dtype=self._tc)
        return x.contiguous()

    def _batch_of(self, x):
        fs = self._field_shape()
        lead = tuple(x.shape[: x.dim() - len(fs)])
        return int(prod(lead)) if lead else 1

    def apply_into(self, x, out, *, adjoint: bool = False, skip_ptr=None, stream=None):
        """Write ``A x`` (or ``A* x``) into ``out`` without allocating.  ``x`` and
        ``out`` are contiguous device tensors of the operator dtype; ``skip_ptr``
        is an optional device address of an int (non-zero: kernels return at once)."""
        b = self._batch_of(x)
        ws = self.workspace(b)
        name = self._native_names[1 if adjoint else 0]
        with tuned(self.xpass_variant):
            if self._chi_layout == _lib.EM3D_CHI_FULL:
                _lib.call(name, ctypes_ref(self._grid_c), self._dt, b, self._spectrum.data_ptr(),
                          self._chi.data_ptr(), x.data_ptr(), out.data_ptr(), ws.data_ptr(), ws.numel(), skip_ptr,
                          _lib.stream_handle(stream))
            else:
                _lib.call(name + "_chi", ctypes_ref(self._grid_c), self._dt, b, self._spectrum.data_ptr(),
                          self._chi_layout, self._chi.data_ptr(), x.data_ptr(), out.data_ptr(), ws.data_ptr(),
                          ws.numel(), skip_ptr, _lib.stream_handle(stream))
        return out

    def dot_parts(self) -> int:
        """CTAs of the last pass when it also forms BiCGStab's omega inner
        products (``apply_dots_into``); 0 where that is not available."""
        n = getattr(self, "_dot_parts", None)
        if n is None:
            n = int(_lib.load().em3d_matvec_dot_parts(self._kind, ctypes_ref(self._grid_c), self._dt))
            self._dot_parts = n
        return n

    def apply_dots_into(self, x, out, partials, *, dot_with=None, skip_ptr=None, stream=None):
        """``out = A x`` for one right-hand side, the last pass also writing, per
        CTA, |t|^2 and Re / Im of vdot(t, w) of t = out into ``partials``
        (float64, 3 x :meth:`dot_parts` values); w = ``dot_with`` (a vector
        shaped like ``x``), or ``x`` itself."""
        ws = self.workspace(1)
        w = None if dot_with is None else dot_with.data_ptr()
        with tuned(self.xpass_variant):
            _lib.call("em3d_matvec_dots", self._kind, ctypes_ref(self._grid_c), self._dt, self._spectrum.data_ptr(),
                      self._chi_layout, self._chi.data_ptr(), x.data_ptr(), out.data_ptr(), ws.data_ptr(), ws.numel(),
                      skip_ptr, partials.data_ptr(), w, _lib.stream_handle(stream))
        return out

    # x-pass implementation chosen for this operator by ``em3d_b200.tune.autotune``
    # (None: the library's process-wide setting)
    xpass_variant = None

    def _grid_key(self):
        g = self._grid_c
        return (g.nx, g.ny, g.nz, g.lx, g.ly, g.lz)

    def _apply_checked(self, x, out, adjoint: bool = False):
        """``apply_into`` followed by :meth:`check_status`: the public
        ``matvec`` / ``rmatvec`` return only results whose transfers all
        completed.  (``apply_into`` itself does not synchronise; the solvers
        read the status words together with their own flags.)"""
        self.apply_into(x, out, adjoint=adjoint)
        self.check_status()
        return out


class Operator(_Applier):
    """``A = I - B chi`` for one EM problem (reference ``src/em3d/operator.py:320-428``)."""

    _kind = _lib.EM3D_EM
    _native_names = ("em3d_em_matvec", "em3d_em_rmatvec")

    def __init__(self, problem: Problem, *, prepared_kernel: PreparedEMKernel | None = None):
        self.problem = problem
        grid = problem.grid
        if prepared_kernel is None:
            prepared_kernel = PreparedEMKernel.build(grid, k=problem.k0)
        else:
            prepared_kernel.validate(grid, k=problem.k0)
        self._prepared_kernel = prepared_kernel
        self._be = grid.backend
        self._N = tuple(grid.N)
        layout, chi = compact_contrast(problem.eps_tensor)
        self._setup_native(grid, prepared_kernel.spectrum, chi, layout)

    @property
    def chi_layout(self) -> str:
        """How the passes read the contrast: ``"isotropic"`` (chi = s I, one
        value per cell), ``"symmetric"`` (six) or ``"full"`` (nine)."""
        return {1: "isotropic", 6: "symmetric", 9: "full"}[self._chi_layout]

    @property
    def backend(self):
        return self._be

    @property
    def shape(self):
        d = 3 * prod(self._N)
        return d, d

    @property
    def prepared_kernel(self) -> PreparedEMKernel:
        return self._prepared_kernel

    def _field_shape(self):
        return (3,) + self._N

    def matvec(self, field):
        x = self._as_field(field)
        import torch

        out = torch.empty_like(x)
        return self._apply_checked(x, out)

    def with_precision(self, precision) -> "Operator":
        """The same operator (grid, k0, contrast) at another precision: the
        FP32 twin used for inner solves of a defect-correction loop.  Its
        spectrum is this operator's, converted (``em3d_spectrum_convert``:
        complex128 -> complex64 gives the bytes of a complex64 build) rather
        than sampled and transformed again."""
        from .backend import Backend
        from .problem import Grid, Problem

        if precision == self._be.precision:
            return self
        be = Backend.b200(precision, device_index=self._be.device_index)
        g = self.problem.grid
        grid = Grid(N=g.N, L=g.L, center=g.center, backend=be)
        tc = precision.torch_complex
        prob = Problem(grid=grid, eps_tensor=self.problem.eps_tensor.to(tc), wave=self.problem.wave.to(tc),
                       k0=self.problem.k0, volume=self.problem.volume)
        src = self._prepared_kernel
        spec = convert_spectrum(src.spectrum, grid, _lib.EM3D_EM, self._be.precision, precision)
        pk = PreparedEMKernel(grid_shape=src.grid_shape, grid_lengths=src.grid_lengths, wave_number=src.wave_number,
                              device=str(be.device), precision=str(precision.value), spectrum=spec,
                              adjoint_storage=src.adjoint_storage, build_strategy=src.build_strategy, _backend=be)
        return Operator(prob, prepared_kernel=pk)

    def rmatvec(self, field):
        if not self._prepared_kernel.supports_adjoint:
            raise RuntimeError("adjoint action is unavailable: build PreparedEMKernel with include_adjoint=True")
        x = self._as_field(field)
        import torch

        out = torch.empty_like(x)
        return self._apply_checked(x, out, adjoint=True)

    def _flat(self, vector):
        """A flat vector (host or device) as a device tensor of the operator's dtype."""
        import torch

        if not isinstance(vector, torch.Tensor):
            vector = torch.as_tensor(np.asarray(vector))
        return vector.to(device=self._be.torch_device, dtype=self._tc)

    def matvec_flat(self, vector):
        """``A`` on a cell-major, component-minor flat vector (reference
        ``src/em3d/operator.py:400-402``); returns a device vector."""
        from .layout import flatten_field, unflatten_field

        return flatten_field(self.matvec(unflatten_field(self._flat(vector), self._N)))

    def rmatvec_flat(self, vector):
        """``A*`` on a flat vector (reference ``src/em3d/operator.py:404-406``)."""
        from .layout import flatten_field, unflatten_field

        return flatten_field(self.rmatvec(unflatten_field(self._flat(vector), self._N)))

    def iteration_matvec_flat(self, vector, *, mu: complex):
        """``x - A x / mu`` (reference ``src/em3d/operator.py:408-409``)."""
        if abs(mu) == 0.0:
            raise ValueError("mu must be non-zero")
        v = self._flat(vector)
        return v - self.matvec_flat(v) / complex(mu)

    def to_dense_operator(self):
        raise RuntimeError("dense matrix construction requires a NumPy backend")

    to_dense_kernel = to_dense_operator
    to_dense = to_dense_operator

"""Device-resident BiCGStab, SIM and TwoStep with the reference's interface.

Mirror of ``src/em3d/solvers/{base,bicgstab,sim,twostep}.py``: the same
``SolverConfig`` / ``SolverResult`` fields, statuses, action counting and
residual histories.  The iteration runs on the GPU: fused update kernels with
FP64 inner products keep every scalar on the device and decide the stopping
rules there (``em3d_b200/csrc/krylov.cu``); the host launches a chunk of
iterations (replayed from a CUDA graph) and reads the status word once per
chunk instead of synchronising on every reduction as the reference does.

Additions over the reference (all optional, defaults keep its behaviour):
``solve(operator, rhs, x0=None)`` accepts an initial guess, and
``DefectCorrection`` runs FP32 inner solves inside an FP64 residual loop.
"""
from __future__ import annotations

import ctypes
from ctypes import c_double, c_int32, c_uint32
from dataclasses import dataclass, field
from typing import Any, List, Optional, Protocol

import numpy as np

from . import _lib

STATUS_NAMES = {
    0: "running", 1: "converged", 2: "max_iter", 3: "max_operator_actions", 4: "nonfinite",
    5: "divergence_guard", 6: "breakdown_rho", 7: "breakdown_alpha", 8: "breakdown_omega",
    9: "breakdown_t", 10: "breakdown_gradient",
}


@dataclass
class SolverConfig:
    """Same fields and defaults as the reference (``src/em3d/solvers/base.py:7-25``)."""

    max_iter: int = 200
    rtol: float = 1e-6
    atol: float = 0.0
    divergence_guard: float | None = None
    max_operator_actions: int | None = None
    log: bool = False
    mu: Optional[complex] = None
    radius: Optional[float] = None

    def require_gamma(self) -> None:
        if self.mu is None or self.radius is None:
            raise ValueError("SolverConfig: mu and radius must be set (call gamma0.find_params)")
        if abs(self.mu) == 0.0:
            raise ValueError("SolverConfig: mu must be non-zero")


@dataclass
class SolverResult:
    """Same fields as the reference (``src/em3d/solvers/base.py:28-44``)."""

    u: Any
    iterations: int
    residual_history: List[float]
    converged: bool
    matvec_count: int = 0
    rmatvec_count: int = 0
    residual_action_counts: List[int] = field(default_factory=list)
    status: str = "unknown"
    true_final_residual: float | None = None

    @property
    def operator_action_count(self) -> int:
        return int(self.matvec_count + self.rmatvec_count)


class BaseSolver(Protocol):
    def solve(self, operator, rhs) -> SolverResult: ...


class KrylovState(ctypes.Structure):
    """Host mirror of ``em3d_krylov_state`` (``include/em3d_b200.h``)."""

    _fields_ = [
        ("rhs_norm", c_double), ("tol", c_double), ("guard", c_double),
        ("gamma_re", c_double), ("gamma_im", c_double),
        ("rho_re", c_double), ("rho_im", c_double), ("rho_prev_re", c_double), ("rho_prev_im", c_double),
        ("alpha_re", c_double), ("alpha_im", c_double), ("omega_re", c_double), ("omega_im", c_double),
        ("t", c_double), ("h", c_double), ("last_rel", c_double), ("dots", c_double * 4),
        ("status", c_int32), ("iter", c_int32), ("matvecs", c_int32), ("rmatvecs", c_int32),
        ("max_iter", c_int32), ("max_actions", c_int32), ("hist_len", c_int32), ("hist_cap", c_int32),
        ("pending", c_int32), ("first", c_int32), ("ticket", c_uint32), ("batch_running", c_int32),
        ("batch_done", c_int32), ("n_used", c_int32),
    ]


def _check_abi():
    lib = _lib.load()
    got = lib.em3d_krylov_state_size()
    if got != ctypes.sizeof(KrylovState):
        raise ImportError(f"em3d_krylov_state size mismatch: library {got}, binding {ctypes.sizeof(KrylovState)}")


class DeviceState:
    """The solver states of a batch of right-hand sides on the device: one
    block per right-hand side (struct + history + reduction partials)."""

    DONE_OFFSET = KrylovState.batch_done.offset
    # states up to this size (one or a few right-hand sides) move by
    # em3d_copy_small; a wide batch's megabytes of states upload faster by a
    # copy engine than by a kernel reading host memory
    SMALL_LIMIT = 256 * 1024

    def __init__(self, device, hist_cap: int, batch: int = 1):
        import torch

        _check_abi()
        lib = _lib.load()
        self.cap = int(max(hist_cap, 2))
        self.batch = int(batch)
        self.stride = int(lib.em3d_krylov_state_bytes(self.cap))
        self.buf = torch.zeros(self.stride * self.batch, dtype=torch.uint8, device=device)
        self.hist_off = lib.em3d_krylov_history_offset(self.cap)
        self.counts_off = lib.em3d_krylov_counts_offset(self.cap)
        self.hosts = [KrylovState() for _ in range(self.batch)]
        for h in self.hosts:
            h.hist_cap = self.cap
        self._done_view = self.buf[self.DONE_OFFSET:self.DONE_OFFSET + 4].view(torch.int32)
        # pinned mirrors of the buffer: read-backs and uploads go through them
        # by em3d_copy_small (a kernel on the solving stream), so they never wait
        # behind a large copy-engine transfer issued on another stream
        nbytes = self.stride * self.batch
        self._small = nbytes <= min(self.SMALL_LIMIT, int(lib.em3d_copy_small_max_bytes()))
        self._hbuf = self._hstage = None
        self._staged = None  # event after the last upload from the staging buffer
        if self._small:
            self._hbuf = torch.empty(nbytes, dtype=torch.uint8).pin_memory()
            self._hstage = torch.empty(nbytes, dtype=torch.uint8).pin_memory()
            self._hview = self._hbuf.numpy()
            self._sview = self._hstage.numpy()
            # pinned memory that this device cannot address (an allocation made
            # for another device's context) is refused: the copies then stay
            # with torch (copy engines)
            status = lib.em3d_copy_small(self._hbuf.data_ptr(), self.buf.data_ptr(), 4,
                                         torch.cuda.current_stream(self.buf.device).cuda_stream)
            if status != 0:
                self._small = False
                self._hbuf = self._hstage = None
            else:
                _lib.count_launches("em3d_copy_small")

    def _read(self, off: int, nbytes: int) -> np.ndarray:
        """Bytes [off, off + nbytes) of the device buffer once the current
        stream has reached this point (a view into the pinned mirror, valid
        until the next read)."""
        import torch

        if not self._small:
            return self.buf.cpu().numpy()
        stream = torch.cuda.current_stream(self.buf.device)
        _lib.call("em3d_copy_small", self._hbuf.data_ptr() + off, self.buf.data_ptr() + off, nbytes,
                  stream.cuda_stream)
        stream.synchronize()
        return self._hview

    @property
    def host(self) -> KrylovState:
        return self.hosts[0]

    @property
    def ptr(self) -> int:
        return self.buf.data_ptr()

    @property
    def done_ptr(self) -> int:
        """Device address of the batch-wide done flag (the operators' skip flag)."""
        return self.buf.data_ptr() + self.DONE_OFFSET

    def upload(self, hists=None, counts=None):
        """Copy the host headers (and initial histories) of all right-hand sides.
        The batch running count and done flag are derived from the statuses."""
        import torch

        running = sum(1 for h in self.hosts if h.status == 0)
        raw = bytearray()
        for b, h in enumerate(self.hosts):
            h.hist_cap = self.cap
            h.hist_len = len(hists[b]) if hists else 0
            h.ticket = 0
            h.batch_running = running if b == 0 else 0
            h.batch_done = (1 if running == 0 else 0) if b == 0 else 0
            blk = bytearray(self.stride)
            hb = bytes(h)
            blk[: len(hb)] = hb
            if hists and len(hists[b]):
                hv = np.asarray(hists[b], dtype=np.float64).tobytes()
                cv = np.asarray(counts[b], dtype=np.int32).tobytes()
                blk[self.hist_off:self.hist_off + len(hv)] = hv
                blk[self.counts_off:self.counts_off + len(cv)] = cv
            raw += blk
        if not self._small:
            self.buf.copy_(torch.frombuffer(raw, dtype=torch.uint8))
            return
        if self._staged is not None:
            self._staged.synchronize()  # the previous upload has left the staging buffer
        self._sview[:len(raw)] = np.frombuffer(bytes(raw), dtype=np.uint8)
        stream = torch.cuda.current_stream(self.buf.device)
        _lib.call("em3d_copy_small", self.buf.data_ptr(), self._hstage.data_ptr(), len(raw), stream.cuda_stream)
        self._staged = torch.cuda.Event()
        self._staged.record(stream)

    def done(self) -> bool:
        if not self._small:
            return int(self._done_view.item()) != 0
        host = self._read(self.DONE_OFFSET, 4)
        return int(host[self.DONE_OFFSET:self.DONE_OFFSET + 4].view(np.int32)[0]) != 0

    def download(self):
        """[(state, history, counts)] for every right-hand side."""
        host = self._read(0, self.stride * self.batch)
        out = []
        sz = ctypes.sizeof(KrylovState)
        for b in range(self.batch):
            base = b * self.stride
            st = KrylovState.from_buffer_copy(host[base:base + sz].tobytes())
            n = int(st.hist_len)
            hist = host[base + self.hist_off:base + self.hist_off + 8 * n].view(np.float64).tolist()
            counts = host[base + self.counts_off:base + self.counts_off + 4 * n].view(np.int32).tolist()
            out.append((st, hist, counts))
        return out

    def dots(self):
        """[(dot0, dot1)] per right-hand side from the last em3d_vec_dots."""
        host = self._read(0, self.stride * self.batch)
        sz = ctypes.sizeof(KrylovState)
        res = []
        for b in range(self.batch):
            st = KrylovState.from_buffer_copy(host[b * self.stride:b * self.stride + sz].tobytes())
            res.append((complex(st.dots[0], st.dots[1]), complex(st.dots[2], st.dots[3])))
        return res


def _check_status(operator) -> None:
    """Raise if one of ``operator``'s applications lost a transfer (operators
    of this package; other operators have no status words)."""
    if hasattr(operator, "check_status"):
        operator.check_status()


def _dcopy(dst, src):
    """``dst = src``.  Between contiguous CUDA complex tensors of one dtype and
    size this is the library's vector kernel on the current stream: a
    device-to-device memcpy would run on a copy engine, queued behind any
    large host transfer that another stream has issued there.  Otherwise
    torch's copy."""
    import torch

    if (dst.is_cuda and src.is_cuda and dst.device == src.device and dst.dtype == src.dtype
            and dst.dtype in (torch.complex64, torch.complex128) and dst.numel() == src.numel()
            and dst.is_contiguous() and src.is_contiguous()):
        if dst.numel():
            dt = _native_dtype(dst)
            _lib.call("em3d_vec_convert", dst.numel(), dt, src.data_ptr(), dt, dst.data_ptr(), 0,
                      _lib.stream_handle())
        return dst
    return dst.copy_(src)


def _dclone(x):
    """A copy of ``x`` (see :func:`_dcopy`)."""
    import torch

    return _dcopy(torch.empty_like(x, memory_format=torch.contiguous_format), x)


def _native_dtype(t) -> int:
    import torch

    if t.dtype == torch.complex64:
        return _lib.EM3D_C64
    if t.dtype == torch.complex128:
        return _lib.EM3D_C128
    raise TypeError(f"solver vectors must be complex64 or complex128, got {t.dtype}")


class _Engine:
    """Vector plumbing shared by the solvers.  ``rhs`` holds ``batch``
    right-hand sides stacked along a leading axis (batch 1: no extra axis)."""

    def __init__(self, operator, rhs, hist_cap, batch: int = 1):
        import torch

        self.op = operator
        self.be = operator.backend
        if not isinstance(rhs, torch.Tensor):
            rhs = torch.as_tensor(np.asarray(rhs))
        tc = self.be.precision.torch_complex if hasattr(self.be, "precision") else rhs.dtype
        self.rhs = torch.empty(rhs.shape, dtype=tc, device=self.be.torch_device)
        _dcopy(self.rhs, rhs)
        self.batch = int(batch)
        self.n = int(self.rhs.numel()) // self.batch
        self.dt = _native_dtype(self.rhs)
        self.state = DeviceState(self.rhs.device, hist_cap, self.batch)
        lens = getattr(operator, "entry_lengths", None)
        if lens is not None and self.batch > 1:
            # rows padded beyond their problem's field (UnevenGroup): the step
            # kernels work on each row's own length
            for h, m in zip(self.state.hosts, lens):
                h.n_used = int(m)
        self.native_op = hasattr(operator, "apply_into")
        if self.batch > 1 and not self.native_op:
            raise TypeError("batched solves need an operator with apply_into (em3d_b200.Operator / AcousticOperator)")
        self.lib = _lib.load()
        self.graph = None
        self.per_replay = 0
        self.vectors = {}

    def load_rhs(self, rhs):
        """Reuse this engine (its buffers and captured graph) for a new right-hand side."""
        _dcopy(self.rhs, rhs.reshape(self.rhs.shape))

    def vec(self):
        import torch

        return torch.zeros_like(self.rhs)

    def stream(self):
        return _lib.stream_handle()

    def apply(self, x, out, adjoint=False, skip=True):
        """``out = A x`` (or ``A* x``).  Inside the iteration the batch-wide done
        flag is the skip flag; set-up calls pass ``skip=False`` because the
        state may still hold the previous solve's flags."""
        if self.native_op:
            if skip and self.batch > 1 and getattr(self.op, "accepts_entry_skip", False):
                # a group of problems: stopped entries skip their share of the work
                self.op.apply_into(x, out, adjoint=adjoint, skip_ptr=self.state.done_ptr,
                                   entry_done=(self.state.ptr + KrylovState.status.offset, self.state.stride))
            else:
                self.op.apply_into(x, out, adjoint=adjoint, skip_ptr=self.state.done_ptr if skip else None)
        else:
            import torch

            y = self.op.rmatvec(x) if adjoint else self.op.matvec(x)
            out.copy_(torch.as_tensor(y, device=out.device).reshape(out.shape))

    def norms(self, x) -> np.ndarray:
        _lib.call("em3d_vec_dots", self.dt, self.n, self.batch, x.data_ptr(), x.data_ptr(), None, None,
                  self.state.ptr, self.state.stride, self.stream())
        return np.array([np.sqrt(max(d0.real, 0.0)) for d0, _ in self.state.dots()])

    def norm(self, x) -> float:
        return float(self.norms(x)[0])

    def step(self, name, *ptrs):
        fn = getattr(self.lib, name)
        status = fn(self.dt, ctypes.c_size_t(self.n), self.batch, ctypes.c_void_p(self.state.ptr),
                    ctypes.c_size_t(self.state.stride), *[ctypes.c_void_p(p) for p in ptrs],
                    ctypes.c_void_p(self.stream()))
        _lib.check(status, name)
        _lib.count_launches(name)

    def _dot_parts(self, fuse: bool):
        """(CTAs, partials buffer) of the fused inner products, or (0, None)
        when they are not available (several right-hand sides, an operator
        without them, or a z axis without a register FFT)."""
        parts = self.op.dot_parts() if (fuse and self.batch == 1 and hasattr(self.op, "dot_parts")) else 0
        if parts <= 0:
            return 0, None
        buf = self.vectors.get("_dot_parts")
        if buf is None:
            import torch

            buf = torch.zeros(3 * parts, dtype=torch.float64, device=self.rhs.device)
            self.vectors["_dot_parts"] = buf
        return parts, buf

    def alpha_step(self, p, v, r_hat, fuse: bool = True):
        """``v = A p`` and BiCGStab's alpha step.  With one right-hand side and
        an operator that supports it, vdot(r_hat, v) comes from the operator's
        last pass (per-CTA partial sums added by one CTA), so v is not read
        again; otherwise the apply and the alpha kernel run separately."""
        parts, buf = self._dot_parts(fuse)
        if parts <= 0:
            self.apply(p, v)
            self.step("em3d_bicgstab_alpha", r_hat.data_ptr(), v.data_ptr())
            return
        self.op.apply_dots_into(p, v, buf, dot_with=r_hat, skip_ptr=self.state.done_ptr)
        _lib.call("em3d_bicgstab_alpha_parts", parts, self.state.ptr, buf.data_ptr(), self.stream())

    def omega_step(self, s, t, fuse: bool = True):
        """``t = A s`` and BiCGStab's omega step.  With one right-hand side and
        an operator that supports it, the inner products |t|^2 and vdot(t, s)
        come from the operator's last pass (per-CTA partial sums added by one
        CTA), so t and s are not read again; otherwise the apply and the
        omega kernel run separately."""
        parts, buf = self._dot_parts(fuse)
        if parts <= 0:
            self.apply(s, t)
            self.step("em3d_bicgstab_omega", t.data_ptr(), s.data_ptr())
            return
        self.op.apply_dots_into(s, t, buf, skip_ptr=self.state.done_ptr)
        _lib.call("em3d_bicgstab_omega_parts", parts, self.state.ptr, buf.data_ptr(), self.stream())

    def run(self, iteration, chunk: int, use_graph: bool):
        """Launch ``iteration`` until every right-hand side has stopped (the
        states as last uploaded by :meth:`DeviceState.upload`).  With a native
        operator the iterations are replayed ``chunk`` at a time from a CUDA
        graph."""
        import torch

        # every caller uploads the states right before: whether any right-hand
        # side runs is known on the host, without a read-back
        if not any(int(h.status) == 0 for h in self.state.hosts):
            return
        if self.graph is None and use_graph and self.native_op:
            iteration()  # the first iteration runs eagerly (and loads the kernels)
            if self.poll():
                return
            with _lib.capturing() as captured:
                try:
                    graph = torch.cuda.CUDAGraph()
                    side = torch.cuda.Stream(device=self.rhs.device)
                    side.wait_stream(torch.cuda.current_stream())
                    with torch.cuda.graph(graph, stream=side, capture_error_mode="thread_local"):
                        for _ in range(chunk):
                            iteration()
                    torch.cuda.current_stream().wait_stream(side)
                    self.graph = graph
                except RuntimeError:
                    self.graph = None
            self.per_replay = captured[0]
        while not self.poll():
            if self.graph is not None:
                self.graph.replay()
                _lib.add_launches(self.per_replay)
            else:
                for _ in range(chunk if self.native_op else 1):
                    iteration()

    def poll(self) -> bool:
        """Whether every right-hand side has stopped: one host read of the done
        flag.  The operator's status word (bounded waits inside its passes that
        gave up) is copied to pinned memory ahead of that read and checked after
        it, so a lost transfer ends the solve with ``NativeError`` at no extra
        synchronisation."""
        import torch

        src = self.op.status_word(self.batch) if hasattr(self.op, "status_word") else None
        if src is not None:
            if getattr(self, "_status_host", None) is None:
                self._status_host = torch.zeros(1, dtype=torch.int32).pin_memory()
            # by a kernel on this stream (em3d_copy_small), not a copy engine
            _lib.call("em3d_copy_small", self._status_host.data_ptr(), src.data_ptr(), 4, self.stream())
        done = self.state.done()
        if src is not None and int(self._status_host[0]) != 0:
            self.op.check_status()
        return done


def _status_name(code: int) -> str:
    return STATUS_NAMES.get(int(code), f"status_{code}")


def _log(tag, history, counts, label="iter"):
    for i, (r, c) in enumerate(zip(history, counts)):
        print(f"[{tag}] {label}={i}, actions={c}, rel_res={r:.3e}")


def _result(u, st, hist, counts) -> SolverResult:
    status = _status_name(st.status)
    return SolverResult(u=u, iterations=int(st.iter), residual_history=[float(h) for h in hist],
                        converged=status == "converged", matvec_count=int(st.matvecs),
                        rmatvec_count=int(st.rmatvecs), residual_action_counts=[int(c) for c in counts],
                        status=status, true_final_residual=float(hist[-1]) if hist else float("inf"))


def _trivial_result(u) -> SolverResult:
    return SolverResult(u=u, iterations=0, residual_history=[0.0], converged=True, matvec_count=0,
                        residual_action_counts=[0], status="converged", true_final_residual=0.0)


def _guard(v):
    return -1.0 if v is None else float(v)


def _budget(v):
    return -1 if v is None else int(v)


def _load_u(buf, x0):
    """Initial iterate in a reused buffer: zero, or a copy of ``x0``."""
    import torch

    if x0 is None:
        buf.zero_()
    else:
        x = x0 if isinstance(x0, torch.Tensor) else torch.as_tensor(np.asarray(x0))
        _dcopy(buf, x.to(device=buf.device, dtype=buf.dtype).reshape(buf.shape))
    return buf


def _entry(operator, u, b: int, batch: int):
    """Right-hand side ``b``'s part of the stacked ``u``: the operator's view
    of it where the operator stacks fields of different shapes
    (``UnevenGroup.entry_field``), else ``u[b]``."""
    if batch == 1:
        return u
    view = getattr(operator, "entry_field", None)
    return view(u, b) if view is not None else u[b]


def _batch_of(operator, rhs) -> int:
    """Number of right-hand sides stacked in front of the operator's field shape."""
    fs = operator._field_shape() if hasattr(operator, "_field_shape") else None
    if fs is None:
        return 1
    lead = tuple(rhs.shape[: len(rhs.shape) - len(fs)])
    if tuple(rhs.shape[len(lead):]) != tuple(fs):
        raise ValueError(f"rhs.shape {tuple(rhs.shape)} != expected (..., {', '.join(map(str, fs))})")
    return int(np.prod(lead)) if lead else 1


class _KrylovSolver:
    """``solve(operator, rhs)`` for one right-hand side (the reference's API) and
    ``solve_batch(operator, rhs)`` for a stack of them sharing the operator.

    Repeated solves with the same operator and shape reuse the device buffers
    and the captured CUDA graph of the iteration (the solver configuration is
    re-read at every solve)."""

    # Engines (device buffers + captured graph) kept per solver object; the
    # oldest is dropped beyond this many, which releases its operator too.
    max_cached_engines = 2

    def _engine(self, operator, rhs, hist_cap, batch):
        from collections import OrderedDict

        if not hasattr(self, "_engines"):
            self._engines = OrderedDict()
        key = (id(operator), tuple(rhs.shape), str(rhs.dtype), batch, hist_cap)
        hit = self._engines.get(key)
        if hit is not None and hit.op is operator:
            self._engines.move_to_end(key)
            hit.load_rhs(rhs)
            return hit
        eng = _Engine(operator, rhs, hist_cap=hist_cap, batch=batch)
        if hasattr(operator, "apply_into"):
            self._engines[key] = eng
            while len(self._engines) > self.max_cached_engines:
                self._engines.popitem(last=False)
        return eng

    def _vec(self, eng, name):
        v = eng.vectors.get(name)
        if v is None:
            v = eng.vec()
            eng.vectors[name] = v
        return v

    def solve(self, operator, rhs, x0=None) -> SolverResult:
        import torch

        t = rhs if isinstance(rhs, torch.Tensor) else torch.as_tensor(np.asarray(rhs))
        return self._solve(operator, t, x0, batch=1)[0]

    def solve_batch(self, operator, rhs, x0=None) -> list:
        import torch

        t = rhs if isinstance(rhs, torch.Tensor) else torch.as_tensor(np.asarray(rhs))
        b = _batch_of(operator, t)
        t = t.reshape((b,) + tuple(operator._field_shape()))
        return self._solve(operator, t, x0, batch=b)

    def _results(self, eng, u, trivial):
        out = []
        u = _dclone(u)  # the engine's buffer is reused by the next solve
        for b, (st, hist, counts) in enumerate(eng.state.download()):
            ub = _entry(eng.op, u, b, eng.batch)
            if trivial[b]:
                out.append(_trivial_result(ub))
            else:
                out.append(_result(ub, st, hist, counts))
        return out


class BiCGStab(_KrylovSolver):
    """BiCGStab (reference ``src/em3d/solvers/bicgstab.py``), device resident."""

    graph_chunk = 4
    # one right-hand side: alpha's and omega's inner products formed in the operator's last pass
    fuse_dots = True

    def __init__(self, config: SolverConfig):
        self.cfg = config

    def _solve(self, operator, rhs, x0, batch):
        cfg = self.cfg
        eng = self._engine(operator, rhs, int(cfg.max_iter) + 2, batch)
        rhs = eng.rhs
        rhs_norms = eng.norms(rhs)
        u = _load_u(self._vec(eng, "u"), x0)
        r = self._vec(eng, "r")
        eng.apply(u, r, skip=False)
        _lib.call("em3d_vec_axpby", eng.dt, eng.n * batch, r.data_ptr(), 1.0, 0.0, rhs.data_ptr(), -1.0, 0.0,
                  r.data_ptr(), eng.stream())
        rr = eng.norms(r)
        trivial = [bool(nrm == 0.0) for nrm in rhs_norms]
        hists, counts = [], []
        for b, st in enumerate(eng.state.hosts):
            nrm = rhs_norms[b] if rhs_norms[b] != 0.0 else 1.0
            rel0 = rr[b] / nrm
            st.rhs_norm, st.tol, st.guard = nrm, max(float(cfg.rtol), float(cfg.atol) / nrm), _guard(cfg.divergence_guard)
            st.matvecs, st.rmatvecs, st.iter = 1, 0, 0
            st.max_iter, st.max_actions = int(cfg.max_iter), _budget(cfg.max_operator_actions)
            st.last_rel = rel0
            st.rho_re, st.rho_im = rr[b] * rr[b], 0.0
            st.rho_prev_re, st.rho_prev_im = 1.0, 0.0
            st.alpha_re, st.alpha_im = 1.0, 0.0
            st.omega_re, st.omega_im = 1.0, 0.0
            st.pending = 0
            if trivial[b]:
                st.status = 1
            elif not np.isfinite(rel0):
                st.status = 4
            elif rel0 < st.tol:
                st.status = 1
            elif cfg.max_operator_actions is not None and 1 >= int(cfg.max_operator_actions):
                st.status = 3
            elif int(cfg.max_iter) <= 0:
                st.status = 2
            else:
                st.status = 0
            hists.append([rel0])
            counts.append([1])
        eng.state.upload(hists, counts)
        r_hat = self._vec(eng, "r_hat")
        _dcopy(r_hat, r)
        p, v, s, t = (self._vec(eng, k) for k in ("p", "v", "s", "t"))

        def iteration():
            eng.step("em3d_bicgstab_p", r.data_ptr(), p.data_ptr(), v.data_ptr())
            eng.alpha_step(p, v, r_hat, self.fuse_dots)
            eng.step("em3d_bicgstab_s", r.data_ptr(), v.data_ptr(), s.data_ptr())
            eng.omega_step(s, t, self.fuse_dots)
            # (the update also completes an early exit taken at s: u + alpha p)
            eng.step("em3d_bicgstab_update", u.data_ptr(), p.data_ptr(), s.data_ptr(), t.data_ptr(), r.data_ptr(),
                     r_hat.data_ptr())

        eng.run(iteration, self.graph_chunk, use_graph=True)
        res = self._results(eng, u, trivial)
        if cfg.log:
            for rb in res:
                _log("BiCGStab", rb.residual_history, rb.residual_action_counts)
        return res


class SIM(_KrylovSolver):
    """Simple iteration ``u <- u - gamma (A u - f)`` (reference ``src/em3d/solvers/sim.py``)."""

    graph_chunk = 8

    def __init__(self, config: SolverConfig):
        config.require_gamma()
        self.cfg = config

    def _solve(self, operator, rhs, x0, batch):
        cfg = self.cfg
        eng = self._engine(operator, rhs, int(cfg.max_iter) + 2, batch)
        rhs = eng.rhs
        rhs_norms = eng.norms(rhs)
        gamma = 1.0 / complex(cfg.mu)
        trivial = [bool(nrm == 0.0) for nrm in rhs_norms]
        for b, st in enumerate(eng.state.hosts):
            nrm = rhs_norms[b] if rhs_norms[b] != 0.0 else 1.0
            st.rhs_norm = nrm
            st.tol = max(float(cfg.rtol), float(cfg.atol) / nrm)
            st.guard = _guard(cfg.divergence_guard)
            st.gamma_re, st.gamma_im = gamma.real, gamma.imag
            st.max_iter, st.max_actions = int(cfg.max_iter), _budget(cfg.max_operator_actions)
            st.iter = st.matvecs = st.rmatvecs = 0
            st.status = 1 if trivial[b] else 0
        eng.state.upload()
        u = _load_u(self._vec(eng, "u"), x0)
        res = self._vec(eng, "res")

        def iteration():
            eng.apply(u, res)
            eng.step("em3d_sim_residual", res.data_ptr(), rhs.data_ptr())
            eng.step("em3d_sim_update", u.data_ptr(), res.data_ptr())

        eng.run(iteration, self.graph_chunk, use_graph=True)
        out = self._results(eng, u, trivial)
        if cfg.log:
            for rb in out:
                _log("SIM", rb.residual_history, rb.residual_action_counts, "updates")
        return out


class TwoStep(_KrylovSolver):
    """Two-step minimal-residual gradient method (reference ``src/em3d/solvers/twostep.py``)."""

    graph_chunk = 4

    def __init__(self, config: SolverConfig):
        self.cfg = config

    def _solve(self, operator, rhs, x0, batch):
        cfg = self.cfg
        eng = self._engine(operator, rhs, int(cfg.max_iter) + 2, batch)
        rhs = eng.rhs
        rhs_norms = eng.norms(rhs)
        trivial = [bool(nrm == 0.0) for nrm in rhs_norms]
        for b, st in enumerate(eng.state.hosts):
            nrm = rhs_norms[b] if rhs_norms[b] != 0.0 else 1.0
            st.rhs_norm = nrm
            st.tol = max(float(cfg.rtol), float(cfg.atol) / nrm)
            st.guard = _guard(cfg.divergence_guard)
            st.max_iter, st.max_actions = int(cfg.max_iter), _budget(cfg.max_operator_actions)
            st.iter = st.matvecs = st.rmatvecs = 0
            st.first = 1
            st.status = 1 if trivial[b] else 0
        eng.state.upload()
        u = _load_u(self._vec(eng, "u"), x0)
        up, r, rp, g, hg = (self._vec(eng, k) for k in ("up", "r", "rp", "g", "hg"))

        def iteration():
            eng.apply(u, r)
            eng.step("em3d_twostep_residual", r.data_ptr(), rhs.data_ptr())
            eng.apply(r, g, adjoint=True)
            eng.apply(g, hg)
            eng.step("em3d_twostep_coeffs", r.data_ptr(), rp.data_ptr(), g.data_ptr(), hg.data_ptr())
            eng.step("em3d_twostep_update", u.data_ptr(), up.data_ptr(), r.data_ptr(), rp.data_ptr(), g.data_ptr())

        eng.run(iteration, self.graph_chunk, use_graph=True)
        out = self._results(eng, u, trivial)
        if cfg.log:
            for rb in out:
                _log("TwoStep", rb.residual_history, rb.residual_action_counts, "updates")
        return out


def true_relative_residual(operator, solution, rhs) -> float:
    """``||A u - f|| / ||f||`` with FP64 norms (reference
    ``src/em3d/experiments/stationary_validation.py:172-180``)."""
    eng = _Engine(operator, rhs, hist_cap=2)
    import torch

    u = solution if isinstance(solution, torch.Tensor) else torch.as_tensor(np.asarray(solution))
    u = u.to(device=eng.rhs.device, dtype=eng.rhs.dtype).reshape(eng.rhs.shape).contiguous()
    rhs_norm = eng.norm(eng.rhs)
    res = eng.vec()
    if eng.native_op:
        operator.apply_into(u, res)
    else:
        res.copy_(torch.as_tensor(operator.matvec(u)).reshape(res.shape))
    _lib.call("em3d_vec_axpby", eng.dt, eng.n, res.data_ptr(), 1.0, 0.0, res.data_ptr(), -1.0, 0.0,
              eng.rhs.data_ptr(), eng.stream())
    rn = eng.norm(res)
    _check_status(operator)
    return rn if rhs_norm == 0.0 else rn / rhs_norm


@dataclass
class DefectCorrectionResult(SolverResult):
    """``SolverResult`` of :class:`DefectCorrection`; the counts above add both
    precisions, the fields below split them."""

    outer_iterations: int = 0
    inner_iterations: List[int] = field(default_factory=list)
    fp64_matvecs: int = 0
    fp32_matvecs: int = 0
    fp32_rmatvecs: int = 0
    guess_rejected: bool = False


class DefectCorrection:
    """FP64 defect correction around low-precision inner Krylov solves.

    Each outer step forms the true residual ``r = f - A u`` with the FP64
    operator and FP64 norms, solves ``A d = r`` with the FP32 twin of the
    operator to a loose tolerance, and updates ``u += d`` in FP64.  The
    outer relative residual is the stopping test, so the returned accuracy
    is that of the FP64 operator.  ``residual_history`` holds the outer true
    residuals.

    ``inner_rtol`` is the FP32 solve's tolerance for the first correction;
    later corrections only need to bring the remaining residual down to
    ``rtol`` (with a safety factor), never looser than ``inner_rtol_max``.
    ``solve_batch`` corrects a stack of right-hand sides together (batched
    operator applications, batched inner solves); each stops on its own.

    An initial guess ``x0`` (a learned warm start, say) is judged by its true
    residual: when ``||f - A x0|| >= ||f||`` (or is not finite) the solve
    falls back to the zero guess (``guess_rejected`` in the result), so a bad
    guess never costs more than one FP64 matvec.
    """

    def __init__(self, config: SolverConfig, *, inner: str = "bicgstab", inner_rtol: float = 1e-4,
                 inner_rtol_max: float = 1e-2, inner_max_iter: int | None = None, max_outer: int = 20,
                 safety: float = 0.3, guess_fallback: bool = True):
        if inner not in ("bicgstab", "twostep"):
            raise ValueError(f"inner must be 'bicgstab' or 'twostep', got {inner!r}")
        self.cfg = config
        self.inner = inner
        self.inner_rtol = float(inner_rtol)
        self.inner_rtol_max = float(inner_rtol_max)
        self.inner_max_iter = inner_max_iter
        self.max_outer = int(max_outer)
        self.safety = float(safety)
        self.guess_fallback = bool(guess_fallback)

    def solve(self, operator, rhs, x0=None, *, operator_low=None) -> DefectCorrectionResult:
        import torch

        t = rhs if isinstance(rhs, torch.Tensor) else torch.as_tensor(np.asarray(rhs))
        return self._solve(operator, t, x0, 1, operator_low)[0]

    def solve_batch(self, operator, rhs, x0=None, *, operator_low=None) -> list:
        import torch

        t = rhs if isinstance(rhs, torch.Tensor) else torch.as_tensor(np.asarray(rhs))
        b = _batch_of(operator, t)
        t = t.reshape((b,) + tuple(operator._field_shape()))
        return self._solve(operator, t, x0, b, operator_low)

    max_cached = 2

    def _buffers(self, operator, rhs, batch, operator_low):
        """Engine, buffers, FP32 operator and inner solver, reused across solves
        with the same operator and shape (a small LRU; evicting an entry
        releases its operators)."""
        from collections import OrderedDict

        import torch

        from .backend import Precision

        if not hasattr(self, "_cache"):
            self._cache = OrderedDict()
        key = (id(operator), tuple(rhs.shape), batch)
        hit = self._cache.get(key)
        if hit is not None and hit["op"] is operator and (operator_low is None or hit["op_lo"] is operator_low):
            self._cache.move_to_end(key)
            hit["eng"].load_rhs(rhs)
            return hit
        eng = _Engine(operator, rhs, hist_cap=4, batch=batch)
        op_lo = operator_low if operator_low is not None else operator.with_precision(Precision.SINGLE)
        inner_cls = BiCGStab if self.inner == "bicgstab" else TwoStep
        hit = {"op": operator, "op_lo": op_lo, "eng": eng, "u": eng.vec(), "r": eng.vec(),
               "r_lo": torch.empty(eng.rhs.shape, dtype=torch.complex64, device=eng.rhs.device),
               "inner": inner_cls(SolverConfig())}
        self._cache[key] = hit
        while len(self._cache) > self.max_cached:
            self._cache.popitem(last=False)
        return hit

    def _solve(self, operator, rhs, x0, batch, operator_low):
        cfg = self.cfg
        buf = self._buffers(operator, rhs, batch, operator_low)
        eng, op_lo, inner = buf["eng"], buf["op_lo"], buf["inner"]
        f = eng.rhs
        fn = eng.norms(f)
        fs = np.where(fn == 0.0, 1.0, fn)
        tol = np.maximum(float(cfg.rtol), float(cfg.atol) / fs)
        u = _load_u(buf["u"], x0)
        r = buf["r"]
        r_lo = buf["r_lo"]
        hist = [[] for _ in range(batch)]
        counts = [[] for _ in range(batch)]
        status = [("converged" if fn[b] == 0.0 else None) for b in range(batch)]
        mv64 = 0
        mv32 = np.zeros(batch, dtype=int)
        rmv32 = np.zeros(batch, dtype=int)
        inner_its = [[] for _ in range(batch)]
        budget_inner = int(self.inner_max_iter or cfg.max_iter)
        rejected = [False] * batch
        for outer in range(self.max_outer + 1):
            if outer == 0 and x0 is None:
                # zero guess: the residual is f itself (A 0 = 0), no FP64 application
                _dcopy(r, f)
                rel = np.where(fn == 0.0, 0.0, 1.0)
            else:
                operator.apply_into(u, r)
                mv64 += 1
                _lib.call("em3d_vec_axpby", eng.dt, eng.n * batch, r.data_ptr(), 1.0, 0.0, f.data_ptr(), -1.0, 0.0,
                          r.data_ptr(), eng.stream())
                rel = eng.norms(r) / fs
                _check_status(operator)
            if outer == 0 and x0 is not None and self.guess_fallback:
                for b in range(batch):
                    if status[b] is None and not rel[b] < 1.0:
                        (u if batch == 1 else u[b]).zero_()
                        _dcopy(r if batch == 1 else r[b], f if batch == 1 else f[b])
                        rel[b] = 1.0
                        rejected[b] = True
            for b in range(batch):
                if status[b] is not None:
                    continue
                hist[b].append(float(rel[b]))
                counts[b].append(int(mv64 + mv32[b] + rmv32[b]))
                if cfg.log:
                    print(f"[DefectCorrection] rhs={b}, outer={outer}, actions={counts[b][-1]}, rel_res={rel[b]:.3e}")
                if not np.isfinite(rel[b]):
                    status[b] = "nonfinite"
                elif rel[b] < tol[b]:
                    status[b] = "converged"
                elif cfg.divergence_guard is not None and rel[b] > float(cfg.divergence_guard):
                    status[b] = "divergence_guard"
                elif outer == self.max_outer:
                    status[b] = "max_iter"
            running = [b for b in range(batch) if status[b] is None]
            if not running:
                break
            target = min(min(self.inner_rtol_max, max(self.inner_rtol, self.safety * tol[b] / rel[b]))
                         for b in running)
            _lib.call("em3d_vec_convert", eng.n * batch, eng.dt, r.data_ptr(), _lib.EM3D_C64, r_lo.data_ptr(), 0,
                      eng.stream())
            if len(running) < batch:
                for b in range(batch):
                    if status[b] is not None:
                        r_lo[b].zero_()
            inner.cfg = SolverConfig(max_iter=budget_inner, rtol=target)
            res = inner.solve(op_lo, r_lo) if batch == 1 else inner.solve_batch(op_lo, r_lo)
            for b in running:
                mv32[b] += res[b].matvec_count if batch > 1 else res.matvec_count
                rmv32[b] += res[b].rmatvec_count if batch > 1 else res.rmatvec_count
                inner_its[b].append(res[b].iterations if batch > 1 else res.iterations)
            d = (res.u if batch == 1 else res[0].u._base if res[0].u._base is not None else res[0].u).contiguous()
            if d.numel() != r_lo.numel():
                d = torch.stack([rb.u for rb in res]).contiguous()
            _lib.call("em3d_vec_convert", eng.n * batch, _lib.EM3D_C64, d.data_ptr(), eng.dt, u.data_ptr(), 1,
                      eng.stream())
        out = []
        u = _dclone(u)  # the cached buffer is reused by the next solve
        for b in range(batch):
            ub = _entry(operator, u, b, batch)
            h = hist[b] if hist[b] else [0.0]
            out.append(DefectCorrectionResult(
                u=ub, iterations=int(sum(inner_its[b])), residual_history=h, converged=status[b] == "converged",
                matvec_count=int(mv64 + mv32[b]), rmatvec_count=int(rmv32[b]),
                residual_action_counts=counts[b] if counts[b] else [0], status=status[b] or "max_iter",
                true_final_residual=float(h[-1]), outer_iterations=len(inner_its[b]),
                inner_iterations=inner_its[b], fp64_matvecs=int(mv64), fp32_matvecs=int(mv32[b]),
                fp32_rmatvecs=int(rmv32[b]), guess_rejected=rejected[b]))
        return out


class MixedBiCGStab:
    """BiCGStab in FP32 with reliable updates in FP64.

    The iteration (vectors, operator applications, vector updates) runs on the
    FP32 twin of the operator and accumulates a correction ``x32``.  Whenever
    the FP32 recursive residual has dropped by ``delta`` since the last update
    (or has reached the target), the correction is added to the FP64 solution,
    the true residual ``f - A u`` is formed with the FP64 operator and FP64
    norms, and it replaces the FP32 residual.  The search direction, the shadow
    residual and the BiCGStab scalars carry over (``rho`` is recomputed against
    the new residual), so, unlike restarted defect correction, the FP32 run
    needs about as many iterations as FP64 BiCGStab; a cycle that ends inside
    an iteration (the half-step exit) or on a breakdown restarts the
    recurrence from the true residual (cycles run with BiCGStab's half-step
    convergence exit turned off, so they end on full iterations unless the
    half step breaks down).  The stopping test is the FP64 true
    residual, as in :class:`DefectCorrection` (whose result type this returns:
    ``outer_iterations`` counts updates, ``inner_iterations`` the FP32
    iterations of each cycle).  Method: Sleijpen & van der Vorst, "Reliable
    updated residuals in hybrid Bi-CG methods", Computing 56 (1996).

    ``x0`` is judged like in :class:`DefectCorrection`: a guess whose true
    residual is not below ``||f||`` is replaced by the zero guess.
    ``solve_batch`` runs many right-hand sides (or a group of problems) at once.
    """

    graph_chunk = 4
    max_cached = 2
    # one right-hand side: alpha's and omega's inner products formed in the operator's last pass
    fuse_dots = True

    def __init__(self, config: SolverConfig, *, delta: float = 1e-3, safety: float = 0.5,
                 guess_fallback: bool = True, max_cycles: int = 200):
        if not 0.0 < delta < 1.0:
            raise ValueError(f"delta must be in (0, 1), got {delta!r}")
        self.cfg = config
        self.delta = float(delta)
        self.safety = float(safety)
        self.guess_fallback = bool(guess_fallback)
        self.max_cycles = int(max_cycles)

    def _buffers(self, operator, rhs, batch, operator_low):
        from collections import OrderedDict

        import torch

        from .backend import Precision

        if not hasattr(self, "_cache"):
            self._cache = OrderedDict()
        key = (id(operator), tuple(rhs.shape), batch)
        hit = self._cache.get(key)
        if hit is not None and hit["op"] is operator and (operator_low is None or hit["op_lo"] is operator_low):
            self._cache.move_to_end(key)
            hit["eng"].load_rhs(rhs)
            return hit
        eng = _Engine(operator, rhs, hist_cap=4, batch=batch)
        op_lo = operator_low if operator_low is not None else operator.with_precision(Precision.SINGLE)
        zero32 = torch.zeros(eng.rhs.shape, dtype=torch.complex64, device=eng.rhs.device)
        e32 = _Engine(op_lo, zero32, hist_cap=int(self.cfg.max_iter) + 4, batch=batch)
        vec32 = {k: e32.vec() for k in ("u", "r", "r_hat", "p", "v", "s", "t")}
        hit = {"op": operator, "op_lo": op_lo, "eng": eng, "u": eng.vec(), "r": eng.vec(), "e32": e32,
               "v32": vec32}
        self._cache[key] = hit
        while len(self._cache) > self.max_cached:
            self._cache.popitem(last=False)
        return hit

    def solve(self, operator, rhs, x0=None, *, operator_low=None) -> DefectCorrectionResult:
        import torch

        t = rhs if isinstance(rhs, torch.Tensor) else torch.as_tensor(np.asarray(rhs))
        if _batch_of(operator, t) != 1:
            raise NotImplementedError("MixedBiCGStab.solve takes one right-hand side; use solve_batch")
        return self._solve(operator, t, x0, 1, operator_low)[0]

    def solve_batch(self, operator, rhs, x0=None, *, operator_low=None) -> list:
        """``rhs`` stacked along a leading axis (or a group of problems and its
        stacked right-hand sides).  Each right-hand side runs its own cycles
        and stops on its own true residual, exactly as its single solve: a
        cycle of the batch runs until every entry has met its cycle target,
        entries that met theirs wait (their iteration work is skipped), then
        one FP64 application forms every true residual."""
        import torch

        t = rhs if isinstance(rhs, torch.Tensor) else torch.as_tensor(np.asarray(rhs))
        b = _batch_of(operator, t)
        t = t.reshape((b,) + tuple(operator._field_shape()))
        return self._solve(operator, t, x0, b, operator_low)

    def _solve(self, operator, rhs, x0, batch, operator_low) -> list:
        cfg = self.cfg
        buf = self._buffers(operator, rhs, batch, operator_low)
        eng, e32, V = buf["eng"], buf["e32"], buf["v32"]
        f = eng.rhs
        x = _load_u(buf["u"], x0)
        r = buf["r"]
        stream = eng.stream()

        def row(t, b):
            return t if batch == 1 else t[b]

        fn = eng.norms(f)
        fs = np.where(fn == 0.0, 1.0, fn)
        tol = np.maximum(float(cfg.rtol), float(cfg.atol) / fs)
        status = [None] * batch
        for b in range(batch):
            if fn[b] == 0.0:
                row(x, b).zero_()
                status[b] = "zero"
        skip_entries = batch > 1 and getattr(operator, "accepts_entry_skip", False)
        mv64 = np.zeros(batch, dtype=np.int64)

        def true_residual(active):
            if skip_entries:
                # entries that have stopped skip the FP64 application
                for b, h in enumerate(eng.state.hosts):
                    h.status = 0 if b in active else 1
                eng.state.upload()
                operator.apply_into(x, r, entry_done=(eng.state.ptr + KrylovState.status.offset,
                                                      eng.state.stride))
            else:
                operator.apply_into(x, r)
            mv64[list(active)] += 1
            _lib.call("em3d_vec_axpby", eng.dt, eng.n * batch, r.data_ptr(), 1.0, 0.0, f.data_ptr(), -1.0, 0.0,
                      r.data_ptr(), stream)
            # (the FP64 operator's status words are read once, at the end)
            return eng.norms(r) / fs

        hist = [[] for _ in range(batch)]
        counts = [[] for _ in range(batch)]
        rejected = [False] * batch
        estimated = [False] * batch  # history holds only the FP32 estimate
        n32_guess = None  # FP32 norms of r32 as the guess left it (the first cycle reuses them)
        u32, r32, rh, p, v, s, tt = (V[k] for k in ("u", "r", "r_hat", "p", "v", "s", "t"))
        mv32 = np.zeros(batch, dtype=np.int64)
        r32_ready = False  # the first cycle starts from r32 as it stands
        active = [b for b in range(batch) if status[b] is None]
        if active:
            if x0 is None:
                # zero guess: the residual is f itself (A 0 = 0), no FP64 application
                _dcopy(r, f)
                rel = np.ones(batch)
            else:
                # a guess only starts the iteration: its residual is formed with
                # the FP32 operator (the first update takes the FP64 one); a
                # guess that may already meet the tolerance is judged in FP64
                n_all = eng.n * batch
                _lib.call("em3d_vec_convert", n_all, eng.dt, x.data_ptr(), _lib.EM3D_C64, u32.data_ptr(), 0, stream)
                buf["op_lo"].apply_into(u32, v)
                _lib.call("em3d_vec_convert", n_all, eng.dt, f.data_ptr(), _lib.EM3D_C64, r32.data_ptr(), 0, stream)
                _lib.call("em3d_vec_axpby", _lib.EM3D_C64, n_all, r32.data_ptr(), 1.0, 0.0, r32.data_ptr(), -1.0, 0.0,
                          v.data_ptr(), stream)
                mv32[active] += 1
                n32 = e32.norms(r32)
                rel = n32 / fs
                if any(rel[b] < 10.0 * tol[b] or not np.isfinite(rel[b]) for b in active):
                    rel = true_residual(active)
                else:
                    r32_ready = True
                    n32_guess = n32
            for b in active:
                if x0 is not None and self.guess_fallback and not rel[b] < 1.0:
                    n32_guess = None  # r32 changes below
                    row(x, b).zero_()
                    _dcopy(row(r, b), row(f, b))
                    if r32_ready:
                        _lib.call("em3d_vec_convert", eng.n, eng.dt, row(f, b).data_ptr(), _lib.EM3D_C64,
                                  row(r32, b).data_ptr(), 0, stream)
                    rel[b] = 1.0
                    rejected[b] = True
                # residual_history[0] of an accepted guess is this FP32-operator
                # estimate; the reported final residual is always an FP64 one
                estimated[b] = r32_ready and not rejected[b]
                hist[b].append(float(rel[b]))
                counts[b].append(int(mv64[b] + mv32[b]))
                if not np.isfinite(rel[b]):
                    status[b] = "nonfinite"
                elif rel[b] < tol[b]:
                    status[b] = "converged"

        def iteration():
            e32.step("em3d_bicgstab_p", r32.data_ptr(), p.data_ptr(), v.data_ptr())
            e32.alpha_step(p, v, rh, self.fuse_dots)
            e32.step("em3d_bicgstab_s", r32.data_ptr(), v.data_ptr(), s.data_ptr())
            e32.omega_step(s, tt, self.fuse_dots)
            e32.step("em3d_bicgstab_update", u32.data_ptr(), p.data_ptr(), s.data_ptr(), tt.data_ptr(), r32.data_ptr(),
                     rh.data_ptr())

        hosts = e32.state.hosts
        restart = [True] * batch
        total_its = np.zeros(batch, dtype=np.int64)
        cycles = [[] for _ in range(batch)]
        stalled = np.zeros(batch, dtype=np.int64)
        budget = int(cfg.max_iter)
        it0 = np.zeros(batch, dtype=np.int64)
        mv_before = np.zeros(batch, dtype=np.int64)
        while True:
            for b in range(batch):
                if status[b] is None and (total_its[b] >= budget or len(cycles[b]) >= self.max_cycles):
                    status[b] = "max_iter"
            running = [b for b in range(batch) if status[b] is None]
            if not running:
                break
            if not r32_ready:
                _lib.call("em3d_vec_convert", eng.n * batch, eng.dt, r.data_ptr(), _lib.EM3D_C64, r32.data_ptr(), 0,
                          stream)
            n0 = n32_guess if (r32_ready and n32_guess is not None) else e32.norms(r32)
            r32_ready = False
            n32_guess = None
            u32.zero_()
            dots = None
            if any(not restart[b] for b in running):
                _lib.call("em3d_vec_dots", _lib.EM3D_C64, e32.n, batch, rh.data_ptr(), r32.data_ptr(), None, None,
                          e32.state.ptr, e32.state.stride, stream)
                dots = e32.state.dots()
            for b, st in enumerate(hosts):
                if status[b] is not None:
                    # stopped: every kernel of the cycle skips this entry
                    st.status = 1
                    st.pending = 0
                    continue
                if restart[b]:
                    _dcopy(row(rh, b), row(r32, b))
                    st.iter = 0
                    st.rho_re, st.rho_im = n0[b] * n0[b], 0.0
                    st.rho_prev_re, st.rho_prev_im = 1.0, 0.0
                    st.alpha_re, st.alpha_im = 1.0, 0.0
                    st.omega_re, st.omega_im = 1.0, 0.0
                else:
                    rho_new = dots[b][0]
                    st.rho_prev_re, st.rho_prev_im = st.rho_re, st.rho_im
                    st.rho_re, st.rho_im = rho_new.real, rho_new.imag
                it0[b] = int(st.iter)
                st.rhs_norm = n0[b]
                st.tol = max(self.delta, self.safety * tol[b] * fs[b] / n0[b])
                st.guard = -1.0
                st.status = 0
                st.pending = 0
                st.first = 1  # cycles end on full iterations only
                st.max_iter = int(it0[b] + (budget - total_its[b]))
                st.max_actions = -1
                st.last_rel = 1.0
                mv_before[b] = int(st.matvecs)
            e32.state.upload([[1.0]] * batch, [[int(m)] for m in mv_before])
            e32.run(iteration, self.graph_chunk, use_graph=True)
            got_all = e32.state.download()
            its_of = {}
            for b in running:
                got = got_all[b][0]
                st = hosts[b]
                for name in ("rho_re", "rho_im", "rho_prev_re", "rho_prev_im", "alpha_re", "alpha_im", "omega_re",
                             "omega_im", "iter", "matvecs", "status", "pending"):
                    setattr(st, name, getattr(got, name))
                its = int(got.iter) - int(it0[b])
                its_of[b] = its
                total_its[b] += its
                mv32[b] += int(got.matvecs) - int(mv_before[b])
                cycles[b].append(its)
            _lib.call("em3d_vec_convert", eng.n * batch, _lib.EM3D_C64, u32.data_ptr(), eng.dt, x.data_ptr(), 1,
                      stream)
            rel = true_residual(running)
            for b in running:
                st = hosts[b]
                hist[b].append(float(rel[b]))
                counts[b].append(int(mv64[b] + mv32[b]))
                inner = _status_name(st.status)
                if cfg.log:
                    print(f"[MixedBiCGStab] rhs={b}, update={len(cycles[b])}, fp32_iterations={its_of[b]} "
                          f"({inner}), rel_res={rel[b]:.3e}")
                if not np.isfinite(rel[b]):
                    status[b] = "nonfinite"
                elif rel[b] < tol[b]:
                    status[b] = "converged"
                elif cfg.divergence_guard is not None and rel[b] > float(cfg.divergence_guard):
                    status[b] = "divergence_guard"
                stalled[b] = stalled[b] + 1 if its_of[b] == 0 else 0
                if status[b] is None and stalled[b] >= 2:
                    status[b] = inner if inner not in ("converged", "running") else "max_iter"
                restart[b] = int(st.pending) != 0 or inner not in ("converged", "max_iter")
            for b in running:
                estimated[b] = False
        # a solve that ended before any cycle (no budget) still reports the FP64
        # true residual of its guess as the final residual
        final = {b: float(hist[b][-1]) for b in range(batch) if hist[b]}
        late = [b for b in range(batch) if estimated[b]]
        if late:
            rel_t = true_residual(late)
            for b in late:
                final[b] = float(rel_t[b])
        _check_status(operator)  # a lost transfer in any FP64 application of this solve
        u = _dclone(x)  # the cached buffer is reused by the next solve
        out = []
        for b in range(batch):
            ub = _entry(operator, u, b, batch)
            if status[b] == "zero":
                out.append(DefectCorrectionResult(u=ub, iterations=0, residual_history=[0.0], converged=True,
                                                  matvec_count=0, residual_action_counts=[0], status="converged",
                                                  true_final_residual=0.0))
                continue
            out.append(DefectCorrectionResult(
                u=ub, iterations=int(total_its[b]), residual_history=hist[b], converged=status[b] == "converged",
                matvec_count=int(mv64[b] + mv32[b]), rmatvec_count=0, residual_action_counts=counts[b],
                status=status[b], true_final_residual=final[b], outer_iterations=len(cycles[b]),
                inner_iterations=cycles[b], fp64_matvecs=int(mv64[b]), fp32_matvecs=int(mv32[b]),
                guess_rejected=rejected[b]))
        return out

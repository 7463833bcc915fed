"""The B200 backend: the plugin point of the reference (``em3d.Backend``).

Mirrors ``Backend`` / ``Precision`` of the reference
(``src/em3d/backend.py:10-119``, ``src/em3d/dtypes.py:9-19``): a frozen
dataclass ``Backend(xp, device, precision)`` whose ``xp`` is an array
namespace.  Here arrays are torch CUDA tensors; device memory, streams and the
caching allocator come from PyTorch, and the operator and solver arithmetic
runs in this package's own sm_100a kernels.
"""
from __future__ import annotations

from dataclasses import dataclass
from enum import Enum
from typing import Any, Literal

import numpy as np


class Precision(Enum):
    """Same members and dtype pairs as the reference ``em3d.dtypes.Precision``."""

    SINGLE = "single"
    DOUBLE = "double"

    @property
    def real_dtype(self) -> type:
        return np.float32 if self is Precision.SINGLE else np.float64

    @property
    def complex_dtype(self) -> type:
        return np.complex64 if self is Precision.SINGLE else np.complex128

    @property
    def torch_complex(self):
        import torch

        return torch.complex64 if self is Precision.SINGLE else torch.complex128

    @property
    def torch_real(self):
        import torch

        return torch.float32 if self is Precision.SINGLE else torch.float64

    @property
    def native_dtype(self) -> int:
        from ._lib import EM3D_C64, EM3D_C128

        return EM3D_C64 if self is Precision.SINGLE else EM3D_C128


_DEVICE_ARRAY = None


def device_array_type():
    """``torch.Tensor`` subclass carrying NumPy's ``copy()`` method.

    The reference solvers copy vectors with ``x.copy()``
    (``src/em3d/solvers/bicgstab.py:76, 91``), which plain torch tensors lack.
    Arrays made by :class:`TorchNamespace` are of this type, and torch
    propagates it through arithmetic (and ``Operator.matvec`` keeps the type
    of its argument), so every vector the reference solvers derive from them
    has ``copy()`` as well.  Created on first use so that importing this
    module does not import torch.

    The type also passes NumPy complex scalars to torch as Python ``complex``:
    the reference scales vectors by ``be.complex_dtype(alpha)``
    (``bicgstab.py:95-114``), and torch drops the imaginary part of a
    ``numpy.complex64`` scalar operand (only ``numpy.complex128``, a subclass
    of ``complex``, is read correctly).  ``complex(np.complex64(a))`` holds the
    same FP32-rounded value, and a Python scalar does not promote a complex64
    tensor, so the product is the reference's complex64 product."""
    global _DEVICE_ARRAY
    if _DEVICE_ARRAY is None:
        import torch

        def _scalar(a):
            return complex(a) if isinstance(a, np.complexfloating) else a

        class DeviceArray(torch.Tensor):
            def copy(self):
                return self.clone()

            @classmethod
            def __torch_function__(cls, func, types, args=(), kwargs=None):
                args = tuple(_scalar(a) for a in args)
                return super().__torch_function__(func, types, args, kwargs or {})

        _DEVICE_ARRAY = DeviceArray
    return _DEVICE_ARRAY


def as_device_array(t):
    """View a torch tensor as :func:`device_array_type` (no copy)."""
    return t.as_subclass(device_array_type())


def _torch_dtype(dtype):
    import torch

    if dtype is None or isinstance(dtype, torch.dtype):
        return dtype
    return {
        np.dtype(np.complex64): torch.complex64, np.dtype(np.complex128): torch.complex128,
        np.dtype(np.float32): torch.float32, np.dtype(np.float64): torch.float64,
        np.dtype(np.int64): torch.int64, np.dtype(np.int32): torch.int32, np.dtype(bool): torch.bool,
    }[np.dtype(dtype)]


class TorchNamespace:
    """The subset of the NumPy namespace that the reference layers above the
    backend call (``xp.zeros_like``, ``xp.linalg.norm``, ``xp.vdot`` ...),
    expressed with torch on one CUDA device.  Plumbing only: the operator and
    the solvers of this package do not route their arithmetic through it."""

    def __init__(self, device):
        import torch

        self._torch = torch
        self.device = device
        self.pi = float(np.pi)
        self.linalg = self
        self.fft = self

    # construction
    def zeros(self, shape, dtype=None):
        return as_device_array(self._torch.zeros(shape, dtype=_torch_dtype(dtype), device=self.device))

    def empty(self, shape, dtype=None):
        return as_device_array(self._torch.empty(shape, dtype=_torch_dtype(dtype), device=self.device))

    def zeros_like(self, x):
        return as_device_array(self._torch.zeros_like(x))

    def ones_like(self, x):
        return as_device_array(self._torch.ones_like(x))

    def asarray(self, obj, dtype=None):
        t = self._torch
        if isinstance(obj, t.Tensor):
            out = obj.to(device=self.device)
            out = out if dtype is None else out.to(_torch_dtype(dtype))
        else:
            arr = np.asarray(obj) if dtype is None else np.asarray(obj, dtype=dtype)
            out = t.as_tensor(arr, device=self.device)
        return as_device_array(out)

    array = asarray

    def arange(self, *args, dtype=None):
        return self._torch.arange(*args, dtype=_torch_dtype(dtype), device=self.device)

    def linspace(self, start, stop, num, dtype=None):
        return self.asarray(np.linspace(start, stop, num, dtype=dtype))

    def meshgrid(self, *xs, indexing="ij"):
        return self._torch.meshgrid(*xs, indexing=indexing)

    def concatenate(self, xs, axis=0):
        return self._torch.cat(list(xs), dim=axis)

    # elementwise / reductions
    def conj(self, x):
        return self._torch.conj(x).resolve_conj()

    def exp(self, x):
        return self._torch.exp(x)

    def sqrt(self, x):
        return self._torch.sqrt(x)

    def abs(self, x):
        return self._torch.abs(x)

    def where(self, c, a, b):
        t = self._torch
        a = a if isinstance(a, t.Tensor) else t.as_tensor(a, device=self.device)
        b = b if isinstance(b, t.Tensor) else t.as_tensor(b, device=self.device)
        return t.where(c, a, b)

    def vdot(self, a, b):
        return self._torch.vdot(a.reshape(-1), b.reshape(-1))

    def norm(self, x, axis=None):
        if axis is None:
            return self._torch.linalg.vector_norm(x.reshape(-1))
        return self._torch.linalg.vector_norm(x, dim=axis)

    def einsum(self, spec, *ops, **_):
        return self._torch.einsum(spec, *ops)

    def roll(self, x, shift, axis):
        return self._torch.roll(x, shifts=shift, dims=axis)

    def flip(self, x, axis):
        return self._torch.flip(x, dims=axis if isinstance(axis, (tuple, list)) else (axis,))

    # FFT (cuFFT through torch: a comparison column, not the operator path)
    def fftn(self, x, axes=None):
        return self._torch.fft.fftn(x, dim=axes)

    def ifftn(self, x, axes=None):
        return self._torch.fft.ifftn(x, dim=axes)


@dataclass(frozen=True)
class Backend:
    """``Backend(xp, device, precision)`` for one B200.

    ``device`` is ``"cuda"`` (the reference's literal); ``device_index``
    selects the GPU.
    """

    xp: Any
    device: Literal["cuda"]
    precision: Precision
    device_index: int = 0

    @property
    def real_dtype(self) -> type:
        return self.precision.real_dtype

    @property
    def complex_dtype(self) -> type:
        return self.precision.complex_dtype

    @property
    def torch_device(self):
        import torch

        return torch.device("cuda", self.device_index)

    @classmethod
    def b200(cls, precision: Precision = Precision.DOUBLE, device_index: int = 0) -> "Backend":
        import torch

        if not torch.cuda.is_available():
            raise RuntimeError("Backend.b200 needs a CUDA device; none is available")
        from . import _lib

        _lib.load()
        dev = torch.device("cuda", device_index)
        return cls(xp=TorchNamespace(dev), device="cuda", precision=precision, device_index=device_index)

    # the reference names the CuPy constructor ``cupy`` and the chooser ``auto``
    cuda = b200
    auto = b200

    def array(self, obj, dtype=None):
        return self.xp.asarray(obj, dtype=dtype)

    def zeros(self, shape, kind: Literal["real", "complex"]):
        if kind not in ("real", "complex"):
            raise ValueError(f"kind must be 'real' or 'complex', got {kind!r}")
        dt = self.real_dtype if kind == "real" else self.complex_dtype
        return self.xp.zeros(shape, dtype=dt)

    def empty(self, shape, kind: Literal["real", "complex"]):
        if kind not in ("real", "complex"):
            raise ValueError(f"kind must be 'real' or 'complex', got {kind!r}")
        dt = self.real_dtype if kind == "real" else self.complex_dtype
        return self.xp.empty(shape, dtype=dt)

    def to_host(self, arr) -> np.ndarray:
        import torch

        if isinstance(arr, torch.Tensor):
            return arr.detach().resolve_conj().cpu().numpy()
        return np.asarray(arr)

    def fftn(self, x, axes=None):
        return self.xp.fftn(x, axes=axes)

    def ifftn(self, x, axes=None):
        return self.xp.ifftn(x, axes=axes)

    def asarray_of_kind(self, obj, kind: Literal["real", "complex"]):
        dt = self.real_dtype if kind == "real" else self.complex_dtype
        return self.xp.asarray(obj, dtype=dt)

    def synchronize(self) -> None:
        import torch

        torch.cuda.synchronize(self.torch_device)

    def memory_info(self) -> dict:
        import torch

        free_b, total_b = torch.cuda.mem_get_info(self.torch_device)
        return {
            "device_id": int(self.device_index),
            "device_name": torch.cuda.get_device_name(self.torch_device),
            "free_bytes": int(free_b),
            "total_bytes": int(total_b),
            "pool_used_bytes": int(torch.cuda.memory_allocated(self.torch_device)),
            "pool_total_bytes": int(torch.cuda.memory_reserved(self.torch_device)),
            "pinned_pool_free_blocks": 0,
        }

    def clear_memory_pool(self) -> None:
        import torch

        self.synchronize()
        torch.cuda.empty_cache()

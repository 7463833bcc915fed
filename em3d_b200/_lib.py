"""ctypes binding of the C ABI declared in ``include/em3d_b200.h``.

The library is loaded from the package's ``_native`` folder.  There is no
fallback: if the shared library is missing or a call fails, an exception is
raised.
"""
from __future__ import annotations

import contextlib
import ctypes
import os
import threading
from ctypes import POINTER, c_double, c_int, c_int32, c_size_t, c_void_p

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_native", "libem3d_b200.so")

EM3D_OK = 0
EM3D_ERR_INVALID = 1
EM3D_ERR_CUDA = 2
EM3D_ERR_UNSUPPORTED = 3
EM3D_C64 = 0
EM3D_C128 = 1
EM3D_ACOUSTIC = 1
EM3D_EM = 3
EM3D_CHI_ISOTROPIC = 1
EM3D_CHI_SYMMETRIC = 6
EM3D_CHI_FULL = 9
EM3D_TUNE_XPASS_VARIANT = 0
EM3D_TUNE_FFT_GENERIC = 1
EM3D_TUNE_FNO_SIMT = 2
EM3D_TUNE_FNO_CONTRACT = 3


class EmGrid(ctypes.Structure):
    _fields_ = [("nx", c_int32), ("ny", c_int32), ("nz", c_int32),
                ("lx", c_double), ("ly", c_double), ("lz", c_double)]


EM3D_MAX_SEGMENTS = 8


class Segment(ctypes.Structure):
    """Mirror of ``em3d_segment``: problems of one grid size in an application
    over uneven sizes (all strides in bytes)."""

    _fields_ = [("grid", EmGrid), ("count", c_int32), ("chi_layout", c_int32),
                ("spectra", c_void_p), ("spectrum_stride", c_size_t), ("chi", c_void_p), ("chi_stride", c_size_t),
                ("u", c_void_p), ("out", c_void_p), ("field_stride", c_size_t),
                ("entry_done", c_void_p), ("entry_done_stride", c_size_t)]


class NativeError(RuntimeError):
    """A native entry point returned a non-zero status."""


# name -> (restype, argtypes); every entry point of include/em3d_b200.h
_GRID = POINTER(EmGrid)
SIGNATURES = {
    "em3d_abi_version": (c_int, []),
    "em3d_last_error": (ctypes.c_char_p, []),
    "em3d_spectrum_bytes": (c_size_t, [_GRID, c_int, c_int]),
    "em3d_build_workspace_bytes": (c_size_t, [_GRID]),
    "em3d_apply_workspace_bytes": (c_size_t, [_GRID, c_int, c_int, c_int]),
    "em3d_em_spectrum_build": (c_int, [_GRID, c_double, c_int, c_void_p, c_void_p, c_size_t, c_void_p]),
    "em3d_acoustic_spectrum_build": (c_int, [_GRID, c_double, c_int, c_void_p, c_void_p, c_size_t, c_void_p]),
    "em3d_spectrum_convert": (c_int, [_GRID, c_int, c_int, c_void_p, c_int, c_void_p, c_void_p]),
    "em3d_em_kernel_hat_full": (c_int, [_GRID, c_double, c_int, c_int, c_void_p, c_void_p, c_size_t, c_void_p]),
    "em3d_acoustic_kernel_hat_full": (c_int, [_GRID, c_double, c_int, c_int, c_void_p, c_void_p, c_size_t, c_void_p]),
    "em3d_em_matvec": (c_int, [_GRID, c_int, c_int, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_size_t,
                               c_void_p, c_void_p]),
    "em3d_em_rmatvec": (c_int, [_GRID, c_int, c_int, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_size_t,
                                c_void_p, c_void_p]),
    "em3d_em_matvec_chi": (c_int, [_GRID, c_int, c_int, c_void_p, c_int, c_void_p, c_void_p, c_void_p, c_void_p,
                                   c_size_t, c_void_p, c_void_p]),
    "em3d_em_rmatvec_chi": (c_int, [_GRID, c_int, c_int, c_void_p, c_int, c_void_p, c_void_p, c_void_p, c_void_p,
                                    c_size_t, c_void_p, c_void_p]),
    "em3d_acoustic_matvec": (c_int, [_GRID, c_int, c_int, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
                                     c_size_t, c_void_p, c_void_p]),
    "em3d_acoustic_rmatvec": (c_int, [_GRID, c_int, c_int, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
                                      c_size_t, c_void_p, c_void_p]),
    "em3d_em_matvec_grouped": (c_int, [_GRID, c_int, c_int, c_void_p, c_size_t, c_void_p, c_void_p, c_void_p, c_void_p, c_size_t, c_void_p,
        c_void_p, c_size_t, c_void_p]),
    "em3d_em_rmatvec_grouped": (c_int, [_GRID, c_int, c_int, c_void_p, c_size_t, c_void_p, c_void_p, c_void_p, c_void_p, c_size_t, c_void_p,
        c_void_p, c_size_t, c_void_p]),
    "em3d_acoustic_matvec_grouped": (c_int, [_GRID, c_int, c_int, c_void_p, c_size_t, c_void_p, c_void_p, c_void_p, c_void_p, c_size_t, c_void_p,
        c_void_p, c_size_t, c_void_p]),
    "em3d_acoustic_rmatvec_grouped": (c_int, [_GRID, c_int, c_int, c_void_p, c_size_t, c_void_p, c_void_p, c_void_p, c_void_p, c_size_t, c_void_p,
        c_void_p, c_size_t, c_void_p]),
    "em3d_segment_size": (c_size_t, []),
    "em3d_uneven_supported": (c_int, [_GRID, c_int, c_int]),
    "em3d_uneven_workspace_bytes": (c_size_t, [c_int, c_int, c_int, POINTER(Segment)]),
    "em3d_em_matvec_uneven": (c_int, [c_int, c_int, POINTER(Segment), c_void_p, c_size_t, c_void_p, c_void_p]),
    "em3d_em_rmatvec_uneven": (c_int, [c_int, c_int, POINTER(Segment), c_void_p, c_size_t, c_void_p, c_void_p]),
    "em3d_acoustic_matvec_uneven": (c_int, [c_int, c_int, POINTER(Segment), c_void_p, c_size_t, c_void_p, c_void_p]),
    "em3d_acoustic_rmatvec_uneven": (c_int, [c_int, c_int, POINTER(Segment), c_void_p, c_size_t, c_void_p,
                                             c_void_p]),
    "em3d_em_matvec_static_scratch": (c_int, [_GRID, c_int, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
                                              c_void_p]),
    "em3d_static_scratch_bytes": (c_size_t, []),
    "em3d_farfield_workspace_bytes": (c_size_t, [_GRID, c_int]),
    "em3d_fno_failures": (c_int, [c_int]),
    "em3d_matvec_dot_parts": (c_int, [c_int, _GRID, c_int]),
    "em3d_matvec_dots": (c_int, [c_int, _GRID, c_int, c_void_p, c_int, c_void_p, c_void_p, c_void_p, c_void_p,
                                 c_size_t, c_void_p, c_void_p, c_void_p, c_void_p]),
    "em3d_bicgstab_omega_parts": (c_int, [c_int, c_void_p, c_void_p, c_void_p]),
    "em3d_bicgstab_alpha_parts": (c_int, [c_int, c_void_p, c_void_p, c_void_p]),
    "em3d_copy_small_max_bytes": (c_size_t, []),
    "em3d_copy_small": (c_int, [c_void_p, c_void_p, c_size_t, c_void_p]),
    "em3d_fno_spectral": (c_int, [c_int, c_int, c_int, c_int, c_int, c_void_p, c_void_p, c_void_p, c_void_p,
                                  c_void_p]),
    "em3d_em_farfield": (c_int, [_GRID, c_int, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_double, c_double,
                                 c_int, c_void_p, c_void_p, c_void_p, c_size_t, c_void_p]),
    "em3d_acoustic_farfield": (c_int, [_GRID, c_int, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_double,
                                       c_double, c_int, c_void_p, c_void_p, c_void_p, c_size_t, c_void_p]),
    "em3d_sample_ellipsoids": (c_int, [c_int, c_int, c_int, c_int, c_int, c_void_p, c_void_p, c_void_p, c_int,
                                       c_void_p, c_double, c_void_p, c_void_p, c_void_p]),
    "em3d_plane_wave": (c_int, [c_int, c_int, c_int, c_int, c_void_p, c_void_p, c_void_p, c_double, c_void_p,
                                c_void_p, c_double, c_int, c_void_p, c_void_p]),
    "em3d_set_tuning": (c_int, [c_int, c_int]),
    "em3d_get_tuning": (c_int, [c_int]),
    "em3d_fno_lift": (c_int, [c_int, c_int, c_size_t, c_int, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
                              c_void_p]),
    "em3d_fno_lift_bwd": (c_int, [c_int, c_size_t, c_int, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
                                  c_void_p]),
    "em3d_fno_contract": (c_int, [c_int, c_int, c_size_t, c_int, c_int, c_int, c_void_p, c_void_p, c_void_p,
                                  c_void_p]),
    "em3d_fno_row_forward": (c_int, [c_int, c_int, c_int, c_int, c_int, c_int, c_int, c_int, c_void_p, c_void_p,
                                     c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_void_p, c_void_p, c_void_p,
                                     c_void_p, c_void_p, c_void_p, c_void_p]),
    "em3d_fno_modemix": (c_int, [c_int, c_int, c_int, c_int, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    "em3d_fno_modemix_bwd": (c_int, [c_int, c_int, c_int, c_int, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
                                     c_void_p, c_void_p, c_void_p]),
    "em3d_fno_layer_out": (c_int, [c_int, c_int, c_int, c_int, c_int, c_int, c_int, c_void_p, c_void_p, c_void_p,
                                   c_void_p, c_int, c_void_p, c_void_p, c_void_p]),
    "em3d_fno_layer_out_bwd": (c_int, [c_int, c_int, c_int, c_int, c_int, c_int, c_int, c_void_p, c_void_p,
                                       c_void_p, c_int, c_void_p, c_void_p, c_void_p, c_void_p]),
    "em3d_fno_pointwise_wgrad": (c_int, [c_int, c_int, c_size_t, c_int, c_void_p, c_void_p, c_void_p, c_void_p,
                                         c_void_p]),
    "em3d_fno_project": (c_int, [c_int, c_int, c_size_t, c_int, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
                                 c_void_p]),
    "em3d_fno_project_bwd": (c_int, [c_int, c_int, c_size_t, c_int, c_void_p, c_void_p, c_void_p, c_void_p,
                                     c_void_p, c_void_p, c_void_p]),
    "em3d_fno_loss": (c_int, [c_int, c_size_t, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    "em3d_fno_adam": (c_int, [c_int, c_size_t, c_void_p, c_void_p, c_void_p, c_void_p, ctypes.c_float,
                              ctypes.c_float, ctypes.c_float, ctypes.c_float, c_int, c_void_p, c_void_p]),
    "em3d_fno_downsample2": (c_int, [c_int, c_int, c_int, c_int, c_int, c_void_p, c_void_p, c_void_p]),
    "em3d_fno_upsample2": (c_int, [c_int, c_int, c_int, c_int, c_int, c_void_p, c_void_p, c_void_p]),
    "em3d_fno_cast": (c_int, [c_int, c_size_t, c_void_p, c_void_p, c_void_p]),
    "em3d_fno_uncast": (c_int, [c_int, c_size_t, c_void_p, c_void_p, c_void_p]),
    "em3d_krylov_state_size": (c_size_t, []),
    "em3d_krylov_state_bytes": (c_size_t, [c_int]),
    "em3d_krylov_history_offset": (c_size_t, [c_int]),
    "em3d_krylov_counts_offset": (c_size_t, [c_int]),
    "em3d_vec_dots": (c_int, [c_int, c_size_t, c_int, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_size_t,
                              c_void_p]),
    "em3d_vec_axpby": (c_int, [c_int, c_size_t, c_void_p, c_double, c_double, c_void_p, c_double, c_double,
                               c_void_p, c_void_p]),
    "em3d_vec_convert": (c_int, [c_size_t, c_int, c_void_p, c_int, c_void_p, c_int, c_void_p]),
    "em3d_bicgstab_p": (c_int, [c_int, c_size_t, c_int, c_void_p, c_size_t, c_void_p, c_void_p, c_void_p, c_void_p]),
    "em3d_bicgstab_alpha": (c_int, [c_int, c_size_t, c_int, c_void_p, c_size_t, c_void_p, c_void_p, c_void_p]),
    "em3d_bicgstab_s": (c_int, [c_int, c_size_t, c_int, c_void_p, c_size_t, c_void_p, c_void_p, c_void_p, c_void_p]),
    "em3d_bicgstab_omega": (c_int, [c_int, c_size_t, c_int, c_void_p, c_size_t, c_void_p, c_void_p, c_void_p]),
    "em3d_bicgstab_update": (c_int, [c_int, c_size_t, c_int, c_void_p, c_size_t, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    "em3d_bicgstab_finalize": (c_int, [c_int, c_size_t, c_int, c_void_p, c_size_t, c_void_p, c_void_p, c_void_p]),
    "em3d_sim_residual": (c_int, [c_int, c_size_t, c_int, c_void_p, c_size_t, c_void_p, c_void_p, c_void_p]),
    "em3d_sim_update": (c_int, [c_int, c_size_t, c_int, c_void_p, c_size_t, c_void_p, c_void_p, c_void_p]),
    "em3d_twostep_residual": (c_int, [c_int, c_size_t, c_int, c_void_p, c_size_t, c_void_p, c_void_p, c_void_p]),
    "em3d_twostep_coeffs": (c_int, [c_int, c_size_t, c_int, c_void_p, c_size_t, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    "em3d_twostep_update": (c_int, [c_int, c_size_t, c_int, c_void_p, c_size_t, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
}

_lib = None


def load():
    """Load the native library once (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"em3d_b200 native library not found at {LIB_PATH}; build it with "
            "`python -c 'import __graft_entry__ as g; g.build()'` (nvcc, sm_100a)")
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def last_error() -> str:
    return load().em3d_last_error().decode("utf-8", "replace")


def check(status: int, what: str) -> None:
    if status == EM3D_OK:
        return
    msg = last_error()
    if status == EM3D_ERR_INVALID or status == EM3D_ERR_UNSUPPORTED:
        raise ValueError(f"{what}: {msg}")
    raise NativeError(f"{what}: CUDA error: {msg}")


# kernels each entry point launches (the operator passes count five)
LAUNCHES = {
    "em3d_em_matvec": 5, "em3d_em_rmatvec": 5, "em3d_acoustic_matvec": 5, "em3d_acoustic_rmatvec": 5,
    "em3d_em_matvec_chi": 5, "em3d_em_rmatvec_chi": 5, "em3d_em_matvec_grouped": 5, "em3d_em_rmatvec_grouped": 5,
    "em3d_acoustic_matvec_grouped": 5, "em3d_acoustic_rmatvec_grouped": 5,
    "em3d_em_matvec_uneven": 5, "em3d_em_rmatvec_uneven": 5, "em3d_acoustic_matvec_uneven": 5,
    "em3d_acoustic_rmatvec_uneven": 5, "em3d_matvec_dots": 5,
}
# Kernels launched by this process (graph replays add their captured counts).
# Host threads update it under a lock; a thread that is capturing a graph
# counts into its own capture counter instead (captured, not launched).
launch_count = 0
_count_lock = threading.Lock()
_tls = threading.local()


def add_launches(n: int) -> None:
    global launch_count
    with _count_lock:
        launch_count += int(n)


@contextlib.contextmanager
def capturing():
    """Count this thread's launches into a list ``[n]`` instead of
    ``launch_count`` while a CUDA graph is being captured."""
    prev = getattr(_tls, "capture", None)
    _tls.capture = [0]
    try:
        yield _tls.capture
    finally:
        _tls.capture = prev


def count_launches(name: str) -> None:
    if name.startswith("em3d_") and not name.endswith(("_bytes", "_offset", "_size", "_error", "_version",
                                                       "_tuning")):
        n = LAUNCHES.get(name, 1)
        cap = getattr(_tls, "capture", None)
        if cap is not None:
            cap[0] += n
        else:
            add_launches(n)


def call(name: str, *args) -> int:
    """Call ``name`` and raise on a non-zero status."""
    fn = getattr(load(), name)
    status = fn(*args)
    check(status, name)
    count_launches(name)
    return status


def make_grid(N, L) -> EmGrid:
    return EmGrid(int(N[0]), int(N[1]), int(N[2]), float(L[0]), float(L[1]), float(L[2]))


def ptr(t) -> int:
    """Raw device address of a torch tensor (or None -> NULL)."""
    return None if t is None else t.data_ptr()


def stream_handle(stream=None) -> int:
    import torch

    s = stream if stream is not None else torch.cuda.current_stream()
    return s.cuda_stream

"""CPU checks of the C ABI: the library loads and exports every declared entry
point, and the host mirrors of its structs match the compiled layout."""
from __future__ import annotations

import ctypes
import os
import re

import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "em3d_b200.h")


def _declared():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(em3d_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_entry_points():
    names = _declared()
    assert "em3d_em_matvec" in names and "em3d_bicgstab_update" in names
    assert len(names) >= 30


def test_library_exports_every_declared_symbol():
    from em3d_b200 import _lib

    lib = _lib.load()
    missing = [n for n in _declared() if not hasattr(lib, n)]
    assert not missing, missing
    # the ctypes binding covers the whole header too
    assert set(_declared()) <= set(_lib.SIGNATURES), set(_declared()) - set(_lib.SIGNATURES)


def test_size_queries_without_gpu():
    from em3d_b200 import _lib

    lib = _lib.load()
    g = _lib.make_grid((128, 128, 128), (1.0, 1.0, 1.0))
    ref = ctypes.byref(g)
    oct_ = 129 ** 3
    assert lib.em3d_spectrum_bytes(ref, _lib.EM3D_EM, _lib.EM3D_C64) >= 6 * oct_ * 8
    assert lib.em3d_spectrum_bytes(ref, _lib.EM3D_EM, _lib.EM3D_C64) < 6 * oct_ * 8 + 64 * 1024
    assert lib.em3d_spectrum_bytes(ref, _lib.EM3D_ACOUSTIC, _lib.EM3D_C128) >= oct_ * 16
    ws = lib.em3d_apply_workspace_bytes(ref, _lib.EM3D_EM, _lib.EM3D_C64, 1)
    assert ws >= 3 * 128 * 128 * 256 * 8 * 3
    assert lib.em3d_apply_workspace_bytes(ref, _lib.EM3D_EM, _lib.EM3D_C64, 4) >= 4 * ws - 1024
    assert lib.em3d_build_workspace_bytes(ref) >= 256 ** 3 * 16
    bad = _lib.make_grid((0, 4, 4), (1.0, 1.0, 1.0))
    assert lib.em3d_spectrum_bytes(ctypes.byref(bad), _lib.EM3D_EM, _lib.EM3D_C64) == 0
    assert "positive" in _lib.last_error()
    big = _lib.make_grid((1024, 4, 4), (1.0, 1.0, 1.0))
    assert lib.em3d_apply_workspace_bytes(ctypes.byref(big), _lib.EM3D_EM, _lib.EM3D_C64, 1) == 0
    assert "unsupported grid size" in _lib.last_error()


def test_invalid_arguments_are_reported_not_launched():
    """Argument errors return a status before any launch (safe without a GPU)."""
    from em3d_b200 import _lib

    g = _lib.make_grid((4, 4, 4), (1.0, 1.0, 1.0))
    with pytest.raises(ValueError, match="NULL"):
        _lib.call("em3d_em_matvec", ctypes.byref(g), _lib.EM3D_C64, 1, None, None, None, None, None, 0, None, None)
    with pytest.raises(ValueError, match="dtype"):
        _lib.call("em3d_em_matvec", ctypes.byref(g), 7, 1, 1, 1, 1, 2, 1, 1 << 30, None, None)
    with pytest.raises(ValueError, match="state is NULL"):
        _lib.call("em3d_bicgstab_p", _lib.EM3D_C64, 10, 1, None, 0, 1, 1, 1, None)
    with pytest.raises(ValueError, match="batch"):
        _lib.call("em3d_bicgstab_p", _lib.EM3D_C64, 10, 0, 1, 0, 1, 1, 1, None)
    # the one-CTA finishes of the fused inner products
    with pytest.raises(ValueError, match="state is NULL"):
        _lib.call("em3d_bicgstab_alpha_parts", 4, None, 16, None)
    with pytest.raises(ValueError, match="no partial sums"):
        _lib.call("em3d_bicgstab_omega_parts", 0, 16, 16, None)
    with pytest.raises(ValueError, match="no partial sums"):
        _lib.call("em3d_bicgstab_alpha_parts", 4, 16, None, None)
    # small transfers by kernel: null, oversized and misaligned requests
    lib = _lib.load()
    assert lib.em3d_copy_small_max_bytes() >= 1 << 20
    with pytest.raises(ValueError, match="null pointer"):
        _lib.call("em3d_copy_small", None, 16, 16, None)
    with pytest.raises(ValueError, match="max_bytes"):
        _lib.call("em3d_copy_small", 16, 32, lib.em3d_copy_small_max_bytes() + 4, None)
    with pytest.raises(ValueError, match="4-byte aligned"):
        _lib.call("em3d_copy_small", 18, 32, 16, None)
    assert lib.em3d_copy_small(16, 32, 0, None) == 0  # nothing to copy


def test_krylov_state_layout_matches_library():
    from em3d_b200 import _lib
    from em3d_b200.solvers import KrylovState

    lib = _lib.load()
    assert lib.em3d_krylov_state_size() == ctypes.sizeof(KrylovState)
    assert lib.em3d_krylov_history_offset(10) >= ctypes.sizeof(KrylovState)
    assert lib.em3d_krylov_counts_offset(10) >= lib.em3d_krylov_history_offset(10) + 80
    assert lib.em3d_krylov_state_bytes(10) > lib.em3d_krylov_counts_offset(10)


def test_solver_config_mirrors_reference_defaults():
    from em3d_b200.solvers import SolverConfig, SolverResult

    cfg = SolverConfig()
    assert (cfg.max_iter, cfg.rtol, cfg.atol, cfg.log) == (200, 1e-6, 0.0, False)
    with pytest.raises(ValueError, match="mu and radius"):
        SolverConfig().require_gamma()
    with pytest.raises(ValueError, match="non-zero"):
        SolverConfig(mu=0j, radius=1.0).require_gamma()
    r = SolverResult(u=None, iterations=1, residual_history=[1.0], converged=False, matvec_count=2, rmatvec_count=3)
    assert r.operator_action_count == 5


def test_tuning_keys_validate_without_gpu():
    from em3d_b200 import _lib

    lib = _lib.load()
    assert lib.em3d_get_tuning(_lib.EM3D_TUNE_XPASS_VARIANT) == -1   # automatic by default
    assert lib.em3d_set_tuning(_lib.EM3D_TUNE_XPASS_VARIANT, 11) == _lib.EM3D_ERR_INVALID
    assert "variant" in _lib.last_error()
    for v in (5, 6, 3, 4, 7, 8, 9, 10, 0, -1):
        assert lib.em3d_set_tuning(_lib.EM3D_TUNE_XPASS_VARIANT, v) == 0
        assert lib.em3d_get_tuning(_lib.EM3D_TUNE_XPASS_VARIANT) == v


def test_tuned_context_restores_the_process_setting():
    from em3d_b200 import _lib
    from em3d_b200.operator import tuned

    lib = _lib.load()
    before = (lib.em3d_get_tuning(_lib.EM3D_TUNE_XPASS_VARIANT), lib.em3d_get_tuning(_lib.EM3D_TUNE_FFT_GENERIC))
    with tuned(7):
        assert lib.em3d_get_tuning(_lib.EM3D_TUNE_XPASS_VARIANT) == 7
    with tuned("generic"):
        assert lib.em3d_get_tuning(_lib.EM3D_TUNE_FFT_GENERIC) == 1
    with tuned(None):
        assert lib.em3d_get_tuning(_lib.EM3D_TUNE_XPASS_VARIANT) == before[0]
    assert (lib.em3d_get_tuning(_lib.EM3D_TUNE_XPASS_VARIANT),
            lib.em3d_get_tuning(_lib.EM3D_TUNE_FFT_GENERIC)) == before

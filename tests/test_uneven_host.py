"""CPU checks of the uneven-size application's host side: the segment layout
matches the library, the supported grids and workspace sizes, and argument
errors that are reported before any launch."""
from __future__ import annotations

import ctypes

import pytest


def _lib():
    from em3d_b200 import _lib

    return _lib, _lib.load()


def _ok(N, kind, dtype):
    L, lib = _lib()
    g = L.make_grid(N, (1.0, 1.0, 1.0))
    return bool(lib.em3d_uneven_supported(ctypes.byref(g), kind, dtype))


def test_segment_layout_matches_library():
    L, lib = _lib()
    assert lib.em3d_segment_size() == ctypes.sizeof(L.Segment)


def test_supported_grids():
    L, _ = _lib()
    EM, AC, C64, C128 = L.EM3D_EM, L.EM3D_ACOUSTIC, L.EM3D_C64, L.EM3D_C128
    for N in [(32, 32, 32), (48, 48, 48), (64, 64, 64), (80, 80, 80), (96, 96, 96), (128, 128, 128), (32, 16, 48)]:
        assert _ok(N, EM, C64), N
        assert _ok(N, AC, C64), N
    # a 32-point x pencil in complex64 is two threads wide: no 128-thread CTA shape
    assert not _ok((16, 16, 16), EM, C64)
    assert _ok((16, 16, 16), EM, C128)
    assert _ok((80, 80, 80), EM, C128)
    assert _ok((64, 80, 80), EM, C128)
    # lengths without a register plan, or beyond 256
    assert not _ok((40, 40, 40), EM, C64)
    assert not _ok((256, 32, 32), EM, C64)
    assert not _ok((32, 32, 12), EM, C64)


def _segment(L, N, count, layout=9):
    s = L.Segment()
    s.grid = L.make_grid(N, (1.0, 1.0, 1.0))
    s.count = count
    s.chi_layout = layout
    g = ctypes.byref(s.grid)
    s.spectrum_stride = L.load().em3d_spectrum_bytes(g, L.EM3D_EM, L.EM3D_C64)
    cells = N[0] * N[1] * N[2]
    s.chi_stride = layout * cells * 8
    s.field_stride = 3 * cells * 8
    return s


def test_workspace_bytes():
    L, lib = _lib()
    segs = (L.Segment * 2)(_segment(L, (32, 32, 32), 2), _segment(L, (48, 32, 64), 1))

    def al(v):
        return (v + 255) // 256 * 256

    want = 0
    for (nx, ny, nz), c in (((32, 32, 32), 2), ((48, 32, 64), 1)):
        want += al(c * 3 * nx * ny * 2 * nz * 8) + al(c * 3 * nx * 2 * ny * 2 * nz * 8)
    want += 256
    assert lib.em3d_uneven_workspace_bytes(L.EM3D_EM, L.EM3D_C64, 2, segs) == want
    assert lib.em3d_uneven_workspace_bytes(L.EM3D_EM, L.EM3D_C64, 0, segs) == 0
    assert lib.em3d_uneven_workspace_bytes(L.EM3D_EM, L.EM3D_C64, 9, segs) == 0
    bad = (L.Segment * 1)(_segment(L, (40, 40, 40), 1))
    assert lib.em3d_uneven_workspace_bytes(L.EM3D_EM, L.EM3D_C64, 1, bad) == 0


def test_invalid_arguments_are_reported_not_launched():
    L, lib = _lib()
    segs = (L.Segment * 2)(_segment(L, (32, 32, 32), 2, layout=1), _segment(L, (48, 48, 48), 1, layout=6))
    for s in segs:
        s.spectra, s.chi, s.u, s.out = 16, 16, 32, 48  # never dereferenced: every check fails first
    big = 1 << 40
    with pytest.raises(ValueError, match="nseg"):
        L.call("em3d_em_matvec_uneven", L.EM3D_C64, 0, segs, 64, big, None, None)
    with pytest.raises(ValueError, match="same chi_layout"):
        L.call("em3d_em_matvec_uneven", L.EM3D_C64, 2, segs, 64, big, None, None)
    with pytest.raises(ValueError, match="too small"):
        L.call("em3d_em_matvec_uneven", L.EM3D_C64, 2, segs, 64, 1024, None, None)
    segs[1].chi_layout = 5
    with pytest.raises(ValueError, match="chi_layout must be"):
        L.call("em3d_em_matvec_uneven", L.EM3D_C64, 2, segs, 64, big, None, None)
    segs[1].chi_layout = 1
    segs[1].u = segs[1].out
    with pytest.raises(ValueError, match="alias"):
        L.call("em3d_em_matvec_uneven", L.EM3D_C64, 2, segs, 64, big, None, None)
    segs[1].u = 32
    segs[0].field_stride = 8
    with pytest.raises(ValueError, match="field_stride"):
        L.call("em3d_em_matvec_uneven", L.EM3D_C64, 2, segs, 64, big, None, None)
    one = (L.Segment * 1)(_segment(L, (40, 40, 40), 1))
    one[0].spectra, one[0].chi, one[0].u, one[0].out = 16, 16, 32, 48
    with pytest.raises(ValueError, match="not supported"):
        L.call("em3d_acoustic_matvec_uneven", L.EM3D_C64, 1, one, 64, big, None, None)
    with pytest.raises(ValueError, match="dtype"):
        L.call("em3d_em_rmatvec_uneven", 5, 2, segs, 64, big, None, None)


def test_fused_dot_parts_counts():
    """CTAs of the last pass that em3d_matvec_dots writes partial sums for:
    ceil(Nx Ny / rows per CTA) on register-FFT z lengths, 0 elsewhere."""
    L, lib = _lib()

    def parts(N, kind, dtype):
        g = L.make_grid(N, (1.0, 1.0, 1.0))
        return lib.em3d_matvec_dot_parts(kind, ctypes.byref(g), dtype)

    # complex64 EM, 2 Nz = 256: 16 threads per row, 5 rows of 3 components per CTA
    assert parts((128, 128, 128), L.EM3D_EM, L.EM3D_C64) == -(-128 * 128 // 5)
    # acoustic: 16 rows per CTA
    assert parts((128, 128, 128), L.EM3D_ACOUSTIC, L.EM3D_C64) == 128 * 128 // 16
    assert parts((16, 16, 40), L.EM3D_EM, L.EM3D_C64) == 0          # 80 points: generic passes
    assert parts((16, 16, 16), 2, L.EM3D_C64) == 0
    g = L.make_grid((16, 16, 16), (1.0, 1.0, 1.0))
    with pytest.raises(ValueError, match="partials"):
        L.call("em3d_matvec_dots", L.EM3D_EM, ctypes.byref(g), L.EM3D_C64, 16, 9, 16, 32, 48, 64, 1 << 30, None,
               None, None, None)

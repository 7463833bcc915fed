"""NumPy restatement of the device input builders (``em3d_b200/csrc/materials.cu``).

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).

* ``scene_hits``: index of the last ellipsoid containing each cell centre.
  The per-shape test follows the reference's ``center_mask``
  (``src/em3d/geometry.py:67-93``): float64 cell centres, ``sum (d_i/a_i)^2 <=
  1 + tol``, here with the offset first rotated into the body frame,
  ``p_i = (R[0][i] d0 + R[1][i] d1) + R[2][i] d2`` (every operation rounded in
  that order, as the kernel does).  With R = I it is the reference test.
* ``sample_contrast``: ``chi = eps - I`` with the reference's rounding
  (``src/em3d/geometry.py:203-252``): ``eps = bg + (feature - bg)`` in
  complex128, cast to the output type, then ``- I`` in that type.
* ``sample_eta``: the acoustic material value, as ``eta_sphere`` /
  ``eta_ellipsoid`` (``src/em3d/acoustics/materials.py:44-83``) painted in order.
* ``plane_wave``: ``amplitude exp(i sign (k orient.r + phi0))``
  (``src/em3d/wave.py:9-37``).

Parity: pinned against the reference-built contrast, eta and wave arrays in
``tests/golden/em_*.npz`` / ``ac_*.npz``.
"""
from __future__ import annotations

import numpy as np

SHAPE_DOUBLES = 33


def pack(center, radii, rotation=None, eps=1.0) -> np.ndarray:
    """One shape as the kernel's 33 float64 values."""
    R = np.eye(3) if rotation is None else np.asarray(rotation, dtype=np.float64)
    e = np.asarray(eps, dtype=np.complex128)
    if e.ndim == 0:
        e = complex(e) * np.eye(3, dtype=np.complex128)
    ev = np.stack([e.real.reshape(-1), e.imag.reshape(-1)], axis=1).reshape(-1)
    return np.concatenate([np.asarray(center, np.float64), np.asarray(radii, np.float64), R.reshape(-1), ev])


def scene_hits(axes, shapes: np.ndarray, tol: float) -> np.ndarray:
    x, y, z = (np.asarray(a, dtype=np.float64) for a in axes)
    X, Y, Z = np.meshgrid(x, y, z, indexing="ij")
    lim = 1.0 + tol
    hit = np.full(X.shape, -1, dtype=np.int64)
    for s, sh in enumerate(np.asarray(shapes, dtype=np.float64).reshape(-1, SHAPE_DOUBLES)):
        c, a, R = sh[0:3], sh[3:6], sh[6:15].reshape(3, 3)
        d0, d1, d2 = X - c[0], Y - c[1], Z - c[2]
        acc = np.zeros(X.shape)
        for i in range(3):
            p = (R[0, i] * d0 + R[1, i] * d1) + R[2, i] * d2
            q = p / a[i]
            acc = acc + q * q
        hit[acc <= lim] = s
    return hit


def em_tol(L) -> float:
    """The reference EM builder's tolerance: 64 eps_f64 max(1, |L|)."""
    return 64.0 * np.finfo(np.float64).eps * max(1.0, *(abs(float(v)) for v in L))


def sample_contrast(axes, shapes, tol, background=1.0, dtype=np.complex128) -> np.ndarray:
    hit = scene_hits(axes, shapes, tol)
    bg = np.asarray(background, dtype=np.complex128)
    if bg.ndim == 0:
        bg = complex(bg) * np.eye(3, dtype=np.complex128)
    sh = np.asarray(shapes, dtype=np.float64).reshape(-1, SHAPE_DOUBLES)
    feats = [(s[15::2] + 1j * s[16::2]).reshape(3, 3) for s in sh]
    out = np.empty((3, 3) + hit.shape, dtype=dtype)
    eye = np.eye(3)
    for a in range(3):
        for b in range(3):
            eps = np.full(hit.shape, bg[a, b], dtype=np.complex128)
            for s, f in enumerate(feats):
                eps[hit == s] = bg[a, b] + (f[a, b] - bg[a, b])
            out[a, b] = eps.astype(dtype) - np.asarray(eye[a, b], dtype=dtype)
    return out


def sample_eta(axes, shapes, tol=0.0, background=1.0, dtype=np.complex128) -> np.ndarray:
    hit = scene_hits(axes, shapes, tol)
    sh = np.asarray(shapes, dtype=np.float64).reshape(-1, SHAPE_DOUBLES)
    out = np.full(hit.shape, dtype(background), dtype=dtype)
    for s, row in enumerate(sh):
        out[hit == s] = dtype(complex(row[15], row[16]))
    return out


def plane_wave(axes, k, orient, amplitude, phi0=0.0, sign=1, dtype=np.complex128) -> np.ndarray:
    x, y, z = (np.asarray(a, dtype=np.float64) for a in axes)
    X, Y, Z = np.meshgrid(x, y, z, indexing="ij")
    phase = sign * (k * ((orient[0] * X + orient[1] * Y) + orient[2] * Z) + phi0)
    carrier = np.exp(1j * phase)
    return np.stack([(complex(a) * carrier).astype(dtype) for a in amplitude])

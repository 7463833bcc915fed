"""NumPy restatement of the far-field sums (TEST INFRASTRUCTURE ONLY, see
``oracle/__init__.py``).

EM (reference ``src/em3d/farfield/_core.py:8-71``):
    F[m][c] = dV sum_q (chi u)_c(q) exp(-i k0 e_m . r_q)
acoustic (reference ``src/em3d/acoustics/farfield.py:29-60``), e_m normalised:
    F[m] = k0^2 dV / (4 pi) sum_q chi(q) u(q) exp(-i k0 e_m . r_q)
Parity: pinned against ``tests/golden/farfield.npz`` (the reference run on the
committed golden inputs).
"""
from __future__ import annotations

import numpy as np


def _coords(axes):
    X, Y, Z = np.meshgrid(*(np.asarray(a, dtype=np.float64) for a in axes), indexing="ij")
    return np.stack([X.ravel(), Y.ravel(), Z.ravel()])


def em_scatter_integral(chi, u, axes, k0, dv, dirs):
    J = np.einsum("ij...,j...->i...", chi.astype(np.complex128), u.astype(np.complex128)).reshape(3, -1)
    phase = np.exp(-1j * k0 * (np.asarray(dirs, np.float64) @ _coords(axes)))
    return dv * (J @ phase.T).T


def acoustic_amplitude(chi, u, axes, k0, dv, dirs):
    d = np.asarray(dirs, np.float64)
    d = d / np.linalg.norm(d, axis=1)[:, None]
    src = (chi.astype(np.complex128) * u.astype(np.complex128)).ravel()
    phase = np.exp(-1j * k0 * (d @ _coords(axes)))
    return (k0 ** 2) * dv / (4.0 * np.pi) * (phase @ src)

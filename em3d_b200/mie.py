"""Mie series for a homogeneous sphere: the exact plane-wave scattering
solution the EM results are compared against (host NumPy/SciPy; not part of
the solve).

Restated from the published theory (Bohren & Huffman, "Absorption and
Scattering of Light by Small Particles", 1983, ch. 4): Riccati-Bessel
functions psi_n(z) = z j_n(z), xi_n(z) = z h1_n(z); external coefficients
a_n, b_n; angular functions pi_n, tau_n by their upward recurrence; amplitude
functions S1, S2.  The truncation n_max = round(x + 4 x^(1/3) + 2) and the
in-plane RCS conventions follow the reference's ``em3d.mie``
(``src/em3d/mie.py:18-241``) so that curves agree point by point:
xy plane (theta = 90 deg): (|S2|^2 cos^2 phi + |S1|^2 sin^2 phi) / k0^2;
xz plane (theta = 90 deg - phi, E-plane): |S2|^2 / k0^2; yz plane: |S1|^2 / k0^2.
"""
from __future__ import annotations

import warnings

import numpy as np


def _check(a: float, eps_r: complex, k0: float) -> None:
    if a <= 0:
        raise ValueError(f"a must be > 0, got {a}")
    if k0 <= 0:
        raise ValueError(f"k0 must be > 0, got {k0}")
    if np.real(eps_r) <= 0 and np.imag(eps_r) == 0:
        raise ValueError(f"Re(eps_r) must be > 0 for lossless medium, got {eps_r}")


def n_terms(x: float) -> int:
    return max(1, round(float(x) + 4.0 * float(x) ** (1.0 / 3.0) + 2.0))


def _psi_xi(ns: np.ndarray, z: complex):
    """psi_n, psi_n', xi_n, xi_n' at z for the orders ``ns``."""
    from scipy.special import spherical_jn, spherical_yn

    j = spherical_jn(ns, z)
    dj = spherical_jn(ns, z, derivative=True)
    y = spherical_yn(ns, z)
    dy = spherical_yn(ns, z, derivative=True)
    h, dh = j + 1j * y, dj + 1j * dy
    return z * j, j + z * dj, z * h, h + z * dh


def mie_coefficients(a: float, eps_r: complex, k0: float) -> dict:
    """External (a_n, b_n) and internal (c_n, d_n) coefficients, n = 1..n_max."""
    _check(a, eps_r, k0)
    x = k0 * a
    nmax = n_terms(x)
    if abs(complex(eps_r) - 1.0) <= 1e-14:
        z, o = np.zeros(nmax, np.complex128), np.ones(nmax, np.complex128)
        return {"a": z.copy(), "b": z.copy(), "c": o.copy(), "d": o.copy(), "n_max": nmax}
    if x > 10:
        warnings.warn(f"mie_coefficients: size parameter x={x:.2f} > 10; the Riccati-Bessel series may lose "
                      "accuracy", UserWarning, stacklevel=2)
    m = np.sqrt(complex(eps_r))
    ns = np.arange(1, nmax + 1)
    pm, dpm, _, _ = _psi_xi(ns, m * x)
    px, dpx, xx, dxx = _psi_xi(ns, complex(x))
    den_a = m * pm * dxx - xx * dpm
    den_b = pm * dxx - m * xx * dpm
    return {"a": (m * pm * dpx - px * dpm) / den_a, "b": (pm * dpx - m * px * dpm) / den_b,
            "c": 1j * m / den_b, "d": 1j * m / den_a, "n_max": nmax}


def mie_cross_sections(a: float, eps_r: complex, k0: float) -> dict:
    co = mie_coefficients(a, eps_r, k0)
    w = 2.0 * np.arange(1, co["n_max"] + 1) + 1.0
    scat = float((2 * np.pi / k0 ** 2) * np.sum(w * (np.abs(co["a"]) ** 2 + np.abs(co["b"]) ** 2)))
    ext = float((2 * np.pi / k0 ** 2) * np.sum(w * np.real(co["a"] + co["b"])))
    return {"scat": scat, "ext": ext, "abs": ext - scat}


def angular_functions(n_max: int, mu: np.ndarray):
    """pi_n(mu), tau_n(mu) for n = 1..n_max, shape (n_max, len(mu))."""
    mu = np.asarray(mu, dtype=np.float64)
    pi = np.zeros((n_max, mu.size))
    tau = np.zeros((n_max, mu.size))
    p_nm2, p_nm1 = np.zeros(mu.size), np.ones(mu.size)   # pi_0, pi_1
    for n in range(1, n_max + 1):
        p_n = p_nm1 if n == 1 else ((2 * n - 1) * mu * p_nm1 - n * p_nm2) / (n - 1)
        p_prev = p_nm2 if n == 1 else p_nm1
        pi[n - 1] = p_n
        tau[n - 1] = n * mu * p_n - (n + 1) * p_prev
        p_nm2, p_nm1 = p_prev, p_n
    return pi, tau


def mie_rcs_plane(a: float, eps_r: complex, k0: float, n_phi: int = 180, plane: str = "xy") -> tuple:
    """(phi, sigma) of the sphere's RCS in a coordinate plane, incidence +z with
    x polarisation (the reference's convention)."""
    _check(a, eps_r, k0)
    if plane not in ("xy", "xz", "yz"):
        raise ValueError(f"plane must be 'xy', 'xz', or 'yz', got {plane!r}")
    if n_phi < 1:
        raise ValueError(f"n_phi must be >= 1, got {n_phi}")
    co = mie_coefficients(a, eps_r, k0)
    nmax = co["n_max"]
    ns = np.arange(1, nmax + 1, dtype=np.float64)
    w = (2 * ns + 1) / (ns * (ns + 1))
    phi = np.linspace(0.0, 2.0 * np.pi, n_phi, endpoint=False)
    mu = np.zeros(n_phi) if plane == "xy" else np.cos(np.pi / 2.0 - phi)
    pi, tau = angular_functions(nmax, mu)
    S1 = (w * co["a"]) @ pi + (w * co["b"]) @ tau
    S2 = (w * co["a"]) @ tau + (w * co["b"]) @ pi
    if plane == "xy":
        sigma = (np.abs(S2) ** 2 * np.cos(phi) ** 2 + np.abs(S1) ** 2 * np.sin(phi) ** 2) / k0 ** 2
    elif plane == "xz":
        sigma = np.abs(S2) ** 2 / k0 ** 2
    else:
        sigma = np.abs(S1) ** 2 / k0 ** 2
    return phi, np.real(sigma).astype(np.float64)


def compare_rcs_plane(u, problem, *, a: float, eps_r: complex, n_phi: int = 180, plane: str = "xy",
                      method: str = "direct", batch_size: int = 64, normalize: str = "max") -> dict:
    """The numerical RCS of ``u`` (GPU far field) against the Mie curve: shape
    error of the peak-normalised curves, peak ratio and max deviation relative
    to the Mie peak (keys as the reference's ``compare_rcs_plane``)."""
    if normalize != "max":
        raise ValueError(f"normalize must be 'max', got {normalize!r}")
    if n_phi < 1:
        raise ValueError(f"n_phi must be >= 1, got {n_phi}")
    from . import farfield

    phi, s_num = farfield.rcs_plane(u, problem, n_phi=n_phi, plane=plane, method=method, batch_size=batch_size)
    phi_m, s_mie = mie_rcs_plane(a, eps_r, problem.k0, n_phi=n_phi, plane=plane)
    if not np.allclose(phi, phi_m, rtol=0.0, atol=1e-15):
        raise RuntimeError("numerical and Mie RCS angle grids differ")
    s_num = np.asarray(s_num, dtype=np.float64)
    p_num = float(s_num.max()) if s_num.size else 0.0
    p_mie = float(s_mie.max()) if s_mie.size else 0.0
    n_num = s_num / p_num if p_num > 0 else np.zeros_like(s_num)
    n_mie = s_mie / p_mie if p_mie > 0 else np.zeros_like(s_mie)
    den = float(np.linalg.norm(n_mie))
    if den > 0:
        shape = float(np.linalg.norm(n_num - n_mie) / den)
    else:
        shape = 0.0 if np.linalg.norm(n_num) == 0 else float("inf")
    if p_mie > 0:
        ratio, absrel = p_num / p_mie, float(np.max(np.abs(s_num - s_mie)) / p_mie)
    else:
        ratio, absrel = float("nan"), (0.0 if p_num == 0 else float("inf"))
    return {"phi": phi, "sigma_num": s_num, "sigma_mie": s_mie, "sigma_num_norm": n_num, "sigma_mie_norm": n_mie,
            "shape_err": shape, "scale_ratio": float(ratio), "abs_rel_err": absrel}

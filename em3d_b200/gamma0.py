"""Step size of the SIM solver from the spectrum of a coarse operator
(reference ``src/em3d/gamma0.py:104-221`` and ``src/em3d/acoustics/gamma0.py:1-63``).

``estimate_from_problem(problem, coarse_N=(4, 4, 4))`` resamples the
problem's contrast onto a coarse grid by nearest cell centres, forms the
coarse operator's dense matrix, takes its eigenvalues and localises them:
the circle (centre ``mu``, ``radius``) that contains their convex hull,
excludes the origin and has the smallest ``q = radius / |mu|``.  SIM then
runs with ``gamma = 1 / mu``.

The dense matrix is obtained by applying this library's FP64 operator on the
device to every unit field of the coarse grid in one batched application
(192 columns for the EM operator on 4^3): the FFT convolution equals the
reference's direct cell-to-cell matrix, and the eigenvalues do not depend on
the order of the unknowns.  The eigenvalues and the localisation are host
NumPy work on a 192 x 192 matrix, as in the reference.
"""
from __future__ import annotations

from dataclasses import dataclass
from itertools import combinations

import numpy as np

# the reference's hull settings (spectral/complex_geometry.py:9-12)
ROUND_DECIMALS = 13
CROSS_TOL = 1e-13
CONTAIN_TOL = 1e-12


@dataclass(frozen=True)
class Gamma0Analysis:
    mu: complex
    radius: float
    rho: float
    spectrum: np.ndarray
    hull: np.ndarray
    coarse_N: tuple | None = None
    matrix_shape: tuple | None = None

    @property
    def margin(self) -> float:
        return float(abs(self.mu) - self.radius)

    def as_solver_config_kwargs(self) -> dict:
        return {"mu": self.mu, "radius": self.radius}


def _cross(o, a, b) -> float:
    return float((a[0] - o[0]) * (b[1] - o[1]) - (a[1] - o[1]) * (b[0] - o[0]))


def convex_hull(points) -> np.ndarray:
    """Monotone-chain hull of complex points, counter-clockwise from the
    lowest-leftmost point: coordinates rounded to 13 decimals and
    deduplicated, turns with cross product <= 1e-13 dropped."""
    z = np.asarray(points, dtype=np.complex128).reshape(-1)
    xy = np.round(np.column_stack((z.real, z.imag)), decimals=ROUND_DECIMALS)
    xy = np.unique(xy, axis=0)
    if len(xy) < 2:
        raise ValueError("at least two distinct points are required")
    pts = [tuple(v) for v in xy[np.lexsort((xy[:, 1], xy[:, 0]))]]
    if len(pts) == 2:
        a = np.asarray(pts)
        return a[:, 0] + 1j * a[:, 1]

    def chain(seq):
        out = []
        for q in seq:
            while len(out) >= 2 and _cross(out[-2], out[-1], q) <= CROSS_TOL:
                out.pop()
            out.append(q)
        return out

    lo, hi = chain(pts), chain(pts[::-1])
    hull = lo[:-1] + hi[:-1]
    if len(hull) < 2:
        hull = [pts[0], pts[-1]]
    a = np.asarray(hull)
    return a[:, 0] + 1j * a[:, 1]


def _segment_distance(z: complex, a: complex, b: complex) -> float:
    d = b - a
    den = abs(d) ** 2
    if den == 0.0:
        return abs(z - a)
    f = min(1.0, max(0.0, ((z - a) * np.conj(d)).real / den))
    return abs(z - (a + f * d))


def origin_in_hull(hull: np.ndarray, tol: float = CONTAIN_TOL) -> bool:
    """Whether 0 lies in the convex polygon (edges, vertices and a tolerance
    of ``tol`` on the edge cross products included)."""
    h = np.asarray(hull, dtype=np.complex128).reshape(-1)
    if len(h) == 1:
        return abs(h[0]) <= tol
    if len(h) == 2:
        return _segment_distance(0j, h[0], h[1]) <= tol
    area = 0.5 * float(np.sum(h.real * np.roll(h.imag, -1) - h.imag * np.roll(h.real, -1)))
    sign = 1.0 if area >= 0.0 else -1.0
    for a, b in zip(h, np.roll(h, -1)):
        e, r = b - a, -a
        if sign * (e.real * r.imag - e.imag * r.real) < -tol:
            return False
    return True


def circle_two_points(z1: complex, z2: complex) -> tuple:
    """The localisation circle through z1 and z2 whose centre lies where the
    two points subtend equal angles at the origin: centre
    ``(z1 + z2)/2 + i Im(z1 conj z2) (z2 - z1) / (2 (|z1 conj z2| + Re(z1 conj z2)))``."""
    z1, z2 = complex(z1), complex(z2)
    pr = z1 * np.conj(z2)
    den = 2.0 * (abs(pr) + pr.real)
    if abs(den) < 1e-30:
        raise ValueError("two-point localization circle is undefined")
    mu = 0.5 * (z1 + z2) + 1j * pr.imag * (z2 - z1) / den
    pq = np.conj(z1) * z2
    den2 = 2.0 * (abs(pq) + pq.real)
    if abs(den2) < 1e-30:
        raise ValueError("two-point localization radius is undefined")
    r2 = abs(z1 - z2) ** 2 * abs(pq) / den2
    return complex(mu), float(np.sqrt(max(float(np.real(r2)), 0.0)))


def circle_three_points(z1: complex, z2: complex, z3: complex) -> tuple:
    """Circumcircle of three points."""
    ax, ay, bx, by, cx, cy = z1.real, z1.imag, z2.real, z2.imag, z3.real, z3.imag
    den = 2.0 * (ax * (by - cy) + bx * (cy - ay) + cx * (ay - by))
    if abs(den) < 1e-30:
        raise ValueError("three points are collinear")
    a2, b2, c2 = ax * ax + ay * ay, bx * bx + by * by, cx * cx + cy * cy
    ux = (a2 * (by - cy) + b2 * (cy - ay) + c2 * (ay - by)) / den
    uy = (a2 * (cx - bx) + b2 * (ax - cx) + c2 * (bx - ax)) / den
    mu = complex(ux, uy)
    return mu, float(abs(mu - complex(z1)))


def best_circle(hull: np.ndarray, tol: float = CONTAIN_TOL) -> tuple:
    """(mu, radius, q) over the two-point and three-point circles of the hull
    vertices that contain every vertex and exclude the origin, smallest q."""
    v = np.asarray(hull, dtype=np.complex128).reshape(-1)
    best = None

    def consider(mu, radius):
        nonlocal best
        if not np.all(np.abs(v - mu) <= radius + tol):
            return
        m = abs(mu)
        if m <= radius + tol or m <= tol:
            return
        q = radius / m
        if best is None or q < best[2]:
            best = (mu, radius, q)

    for a, b in combinations(v, 2):
        try:
            consider(*circle_two_points(a, b))
        except ValueError:
            pass
    for a, b, c in combinations(v, 3):
        try:
            consider(*circle_three_points(a, b, c))
        except ValueError:
            pass
    if best is None:
        raise ValueError("could not find a gamma0 circle that excludes the origin")
    return best


def analyze_spectrum(spectrum, *, coarse_N=None, matrix_shape=None) -> Gamma0Analysis:
    """Localise eigenvalues; raises ``ValueError`` with the reference's
    messages when the origin is in their hull or no circle exists."""
    values = np.asarray(spectrum, dtype=np.complex128).reshape(-1)
    try:
        hull = convex_hull(values)
    except ValueError:
        raise ValueError("spectrum samples are degenerate") from None
    if origin_in_hull(hull):
        raise ValueError("could not find a gamma0 circle: the origin belongs to the convex spectral hull")
    mu, radius, q = best_circle(hull)
    return Gamma0Analysis(mu=complex(mu), radius=float(radius), rho=float(q), spectrum=values, hull=hull,
                          coarse_N=coarse_N, matrix_shape=matrix_shape)


def find_params(spectrum) -> dict:
    return analyze_spectrum(spectrum).as_solver_config_kwargs()


def _shape(coarse_N) -> tuple:
    shape = (coarse_N,) * 3 if isinstance(coarse_N, int) else tuple(int(n) for n in coarse_N)
    if len(shape) != 3 or any(n <= 0 for n in shape):
        raise ValueError(f"coarse_N must be a positive int or 3-tuple, got {coarse_N!r}")
    return shape


def _nearest(source, target) -> np.ndarray:
    """Index of the nearest source cell centre for every target centre (ties
    to the left)."""
    s = np.asarray(source, dtype=np.float64)
    t = np.asarray(target, dtype=np.float64)
    i = np.clip(np.searchsorted(s, t), 0, len(s) - 1)
    left = np.clip(i - 1, 0, len(s) - 1)
    return np.where(np.abs(t - s[left]) <= np.abs(t - s[i]), left, i)


def _coarse_grid(problem, shape):
    from .backend import Backend, Precision
    from .problem import Grid

    g = problem.grid
    be = Backend.b200(Precision.DOUBLE, device_index=g.backend.device_index)
    return Grid(N=shape, L=g.L, center=g.center, backend=be)


def _resample(field, fine_grid, coarse_grid) -> np.ndarray:
    """Nearest-cell resampling of the trailing three axes (host complex128)."""
    a = np.asarray(fine_grid.backend.to_host(field), dtype=np.complex128)
    fx, fy, fz = (np.asarray(v, dtype=np.float64) for v in fine_grid.host_axes)
    cx, cy, cz = (np.asarray(v, dtype=np.float64) for v in coarse_grid.host_axes)
    ix, iy, iz = _nearest(fx, cx), _nearest(fy, cy), _nearest(fz, cz)
    return a[..., ix, :, :][..., :, iy, :][..., :, :, iz]


def _dense(op, field_shape) -> np.ndarray:
    """Columns A e_j for every unit field e_j, in one batched application."""
    import torch

    n = int(np.prod(field_shape))
    eye = torch.eye(n, dtype=torch.complex128, device=op.backend.torch_device).reshape((n,) + tuple(field_shape))
    cols = op.matvec(eye).reshape(n, n)
    return cols.transpose(0, 1).cpu().numpy()


def coarse_operator_matrix(problem, coarse_N=(4, 4, 4)) -> np.ndarray:
    """Dense matrix of the problem's operator on the coarse grid (EM:
    ``I - B chi``, 3 n x 3 n; acoustic: ``H``, n x n)."""
    from .acoustics import AcousticOperator, AcousticProblem
    from .operator import Operator
    from .problem import Problem

    shape = _shape(coarse_N)
    grid = _coarse_grid(problem, shape)
    if isinstance(problem, AcousticProblem):
        eta = _resample(problem.eta, problem.grid, grid)
        wave = np.ones(shape, dtype=np.complex128)
        coarse = AcousticProblem(grid=grid, eta=eta, wave=wave, k0=problem.k0, volume=problem.volume)
        return _dense(AcousticOperator(coarse), shape)
    chi = _resample(problem.eps_tensor, problem.grid, grid)
    wave = np.ones((3,) + shape, dtype=np.complex128)
    coarse = Problem(grid=grid, eps_tensor=chi, wave=wave, k0=problem.k0, volume=problem.volume)
    return _dense(Operator(coarse), (3,) + shape)


def estimate_from_problem(problem, coarse_N=(4, 4, 4)) -> Gamma0Analysis:
    """``mu`` and ``radius`` for SIM from the coarse operator's eigenvalues
    (EM ``Problem`` or ``AcousticProblem``)."""
    shape = _shape(coarse_N)
    matrix = coarse_operator_matrix(problem, shape)
    return analyze_spectrum(np.linalg.eigvals(matrix), coarse_N=shape, matrix_shape=matrix.shape)

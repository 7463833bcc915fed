"""Seeded synthetic inputs of the benchmark configurations (host NumPy).

Each builder returns plain arrays (contrast, incident wave, grid data) so that
the same inputs can feed the B200 operator, the CPU oracle and the reference.

* ``sphere_em``: dielectric sphere, README configuration (16^3, k0 = 4,
  eps_r = 2, radius 0.25, +z, x-polarised).
* ``aniso_ellipsoid_em``: absorbing anisotropic ellipsoid, radii
  (0.30, 0.20, 0.25), eps = R diag(2.5+0.1i, 3.0+0.2i, 2.0+0.05i) R^T with R
  a seeded uniform rotation, k0 = 12, +z, x-polarised (128^3 by default).
* ``acoustic_spheres``: 200 non-overlapping spheres, radius U[0.02, 0.06],
  eta U[1.2, 2.5] + i U[0, 0.1], k0 = 20 (256^3 by default).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import setup as _setup


@dataclass
class EMCase:
    name: str
    N: tuple
    L: tuple
    center: tuple
    k0: float
    chi: np.ndarray    # (3,3,Nx,Ny,Nz)
    wave: np.ndarray   # (3,Nx,Ny,Nz)


@dataclass
class AcousticCase:
    name: str
    N: tuple
    L: tuple
    center: tuple
    k0: float
    eta: np.ndarray    # (Nx,Ny,Nz)


def sphere_em(N: int = 16, precision: str = "double", k0: float = 4.0) -> EMCase:
    cdt = _setup.complex_dtype_of(precision)
    Ns, L, c = (N, N, N), (1.0, 1.0, 1.0), (0.0, 0.0, 0.0)
    axes = _setup.grid_axes_host(Ns, L, c, precision)
    chi = _setup.sample_contrast_tensor(axes, L, background_eps_r=1.0, feature_eps_r=2.0,
                                        geometry=_setup.Ellipsoid(c, (0.25, 0.25, 0.25)), dtype=cdt)
    wave = _setup.flat_wave_vec_host(axes, k=k0, orient=(0, 0, 1), amplitude=(1, 0, 0), dtype=cdt)
    return EMCase(f"em_sphere_{N}^3", Ns, L, c, k0, chi, wave)


def rotation_matrix(seed: int = 0) -> np.ndarray:
    """Uniform random SO(3) matrix (``scipy.spatial.transform.Rotation.random``)."""
    from scipy.spatial.transform import Rotation

    return Rotation.random(random_state=seed).as_matrix()


def aniso_permittivity(seed: int = 0) -> np.ndarray:
    R = rotation_matrix(seed)
    return R @ np.diag([2.5 + 0.1j, 3.0 + 0.2j, 2.0 + 0.05j]) @ R.T


def aniso_ellipsoid_em(N: int = 128, precision: str = "double", k0: float = 12.0, seed: int = 0,
                       orient=(0.0, 0.0, 1.0), amplitude=(1.0, 0.0, 0.0)) -> EMCase:
    cdt = _setup.complex_dtype_of(precision)
    Ns, L, c = (N, N, N), (1.0, 1.0, 1.0), (0.0, 0.0, 0.0)
    axes = _setup.grid_axes_host(Ns, L, c, precision)
    chi = _setup.sample_contrast_tensor(axes, L, background_eps_r=1.0, feature_eps_r=aniso_permittivity(seed),
                                        geometry=_setup.Ellipsoid(c, (0.30, 0.20, 0.25)), dtype=cdt)
    wave = _setup.flat_wave_vec_host(axes, k=k0, orient=orient, amplitude=amplitude, dtype=cdt)
    return EMCase(f"em_aniso_ellipsoid_{N}^3", Ns, L, c, k0, chi, wave)


def acoustic_sphere_list(count: int = 200, seed: int = 0) -> list:
    """Rejection-sampled non-overlapping spheres with centres in
    [-0.5+r, 0.5-r]^3: [(centre, radius, eta)], radius U[0.02, 0.06],
    eta U[1.2, 2.5] + i U[0, 0.1]."""
    rng = np.random.default_rng(seed)
    spheres = []
    tries = 0
    while len(spheres) < count:
        tries += 1
        if tries > 200000:
            raise RuntimeError("could not place the spheres")
        r = rng.uniform(0.02, 0.06)
        ctr = rng.uniform(-0.5 + r, 0.5 - r, size=3)
        if all(np.linalg.norm(ctr - c2) > r + r2 for c2, r2, _ in spheres):
            val = rng.uniform(1.2, 2.5) + 1j * rng.uniform(0.0, 0.1)
            spheres.append((ctr, r, val))
    return spheres


def acoustic_spheres(N: int = 256, precision: str = "double", k0: float = 20.0, count: int = 200,
                     seed: int = 0) -> AcousticCase:
    """eta of ``acoustic_sphere_list`` painted in order with the reference's
    sphere test ``sum ((x_i - c_i) / r)^2 <= 1`` (``acoustics/materials.py:62-83``),
    evaluated inside each sphere's bounding box."""
    cdt = _setup.complex_dtype_of(precision)
    Ns, L, c = (N, N, N), (1.0, 1.0, 1.0), (0.0, 0.0, 0.0)
    axes = _setup.grid_axes_host(Ns, L, c, precision)
    eta = np.ones(Ns, dtype=cdt)
    ax = [np.asarray(a, dtype=np.float64) for a in axes]
    for ctr, r, val in acoustic_sphere_list(count, seed):
        sl = []
        for d in range(3):
            lo = int(np.searchsorted(ax[d], ctr[d] - r, side="left"))
            hi = int(np.searchsorted(ax[d], ctr[d] + r, side="right"))
            sl.append(slice(max(lo - 1, 0), min(hi + 1, N)))
        X, Y, Z = np.meshgrid(ax[0][sl[0]], ax[1][sl[1]], ax[2][sl[2]], indexing="ij")
        m = (((X - ctr[0]) / r) ** 2 + ((Y - ctr[1]) / r) ** 2) + ((Z - ctr[2]) / r) ** 2 <= 1.0
        box = eta[sl[0], sl[1], sl[2]]
        box[m] = cdt(val)
    return AcousticCase(f"acoustic_{count}_spheres_{N}^3", Ns, L, c, k0, eta)


def acoustic_spheres_device(grid, count: int = 200, seed: int = 0):
    """The same eta sampled on the device (``em3d_sample_ellipsoids``)."""
    from .scenes import EllipsoidShape, sample_scene_eta

    shapes = [EllipsoidShape(tuple(ctr), (r, r, r), None, val) for ctr, r, val in acoustic_sphere_list(count, seed)]
    return sample_scene_eta(grid, shapes, eta_outside=1.0, tol=0.0)


def fibonacci_directions(n: int) -> np.ndarray:
    """n unit vectors on a golden-angle (Fibonacci) spiral over the sphere."""
    i = np.arange(n, dtype=np.float64)
    z = 1.0 - 2.0 * (i + 0.5) / n
    r = np.sqrt(np.maximum(0.0, 1.0 - z * z))
    phi = i * np.pi * (3.0 - np.sqrt(5.0))
    return np.stack([r * np.cos(phi), r * np.sin(phi), z], axis=-1)


def orthogonal_polarisations(direction) -> tuple:
    """Two unit polarisations orthogonal to ``direction`` and to each other,
    built from a fixed helper axis (z, or x when the direction is near z)."""
    d = np.asarray(direction, dtype=np.float64)
    d = d / np.linalg.norm(d)
    helper = np.array([0.0, 0.0, 1.0]) if abs(d[2]) < 0.9 else np.array([1.0, 0.0, 0.0])
    p1 = np.cross(helper, d)
    p1 /= np.linalg.norm(p1)
    p2 = np.cross(d, p1)
    return p1, p2


def plane_wave_batch(axes, k: float, n_directions: int, dtype=np.complex128) -> np.ndarray:
    """(2 n_directions, 3, Nx, Ny, Nz): every Fibonacci direction with both
    orthogonal polarisations, through ``flat_wave_vec``'s arithmetic."""
    out = []
    for d in fibonacci_directions(n_directions):
        for p in orthogonal_polarisations(d):
            out.append(_setup.flat_wave_vec_host(axes, k=k, orient=tuple(d), amplitude=tuple(p), dtype=dtype))
    return np.stack(out)


def multi_rhs_ellipsoid(N: int = 96, k0: float = 10.0, n_directions: int = 64, precision: str = "double"):
    """The anisotropic ellipsoid at N^3 with 2 n_directions incident waves."""
    case = aniso_ellipsoid_em(N, precision, k0=k0)
    axes = _setup.grid_axes_host(case.N, case.L, case.center, precision)
    waves = plane_wave_batch(axes, k0, n_directions, dtype=_setup.complex_dtype_of(precision))
    return case, waves


def uneven_sphere_params(count: int = 48, seed: int = 0, sizes=(32, 48, 64, 80)) -> list:
    """A set of ``count`` independent single-sphere EM problems of uneven grid
    sizes (L = 1, centred sphere): N drawn uniformly from ``sizes``, radius
    U[0.15, 0.35], eps_r U[1.5, 4] + i U[0, 0.2], k0 U[2, 8], incident along
    +z, x-polarised.  Returns dicts (N, center, radius, eps, k0, orient,
    amplitude)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        N = int(rng.choice(np.asarray(sizes)))
        radius = float(rng.uniform(0.15, 0.35))
        eps = complex(rng.uniform(1.5, 4.0), rng.uniform(0.0, 0.2))
        k0 = float(rng.uniform(2.0, 8.0))
        out.append(dict(N=N, center=(0.0, 0.0, 0.0), radius=radius, eps=eps, k0=k0, orient=(0.0, 0.0, 1.0),
                        amplitude=(1.0, 0.0, 0.0)))
    return out


def uneven_sphere_problems(precision: str = "single", count: int = 48, seed: int = 0, sizes=(32, 48, 64, 80),
                           device_index: int = 0) -> list:
    """``uneven_sphere_params`` built on the device (contrast by the scene
    sampler at the reference's tolerance, plane wave by the wave kernel)."""
    from . import scenes
    from .backend import Backend, Precision
    from .problem import Grid, Problem

    be = Backend.b200(Precision.SINGLE if precision == "single" else Precision.DOUBLE, device_index=device_index)
    problems = []
    for p in uneven_sphere_params(count, seed, sizes):
        grid = Grid(N=(p["N"],) * 3, L=(1.0, 1.0, 1.0), center=(0.0, 0.0, 0.0), backend=be)
        chi = scenes.sample_scene(grid, [scenes.EllipsoidShape(p["center"], (p["radius"],) * 3, None, p["eps"])])
        wave = scenes.plane_wave(grid, k=p["k0"], orient=p["orient"], amplitude=p["amplitude"])
        problems.append(Problem(grid=grid, eps_tensor=chi, wave=wave, k0=p["k0"], volume=1.0))
    return problems

"""Scene builders: the NumPy restatement pinned to reference-built inputs (CPU),
and the device kernels bit-exact against it (GPU)."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import golden

PRECS = (("double", np.complex128), ("single", np.complex64))

# (fixture, centre, radii, feature eps) of the reference-built EM contrasts
EM_CASES = [
    ("em_sphere16.npz", (0.0, 0.0, 0.0), (0.25, 0.25, 0.25), "2.0"),
    ("em_aniso12.npz", (0.0, 0.0, 0.0), (0.30, 0.20, 0.25), "aniso"),
    ("em_odd567.npz", (0.05, 0.0, -0.1), (0.45, 0.3, 0.5), "aniso"),
]
# spheres painted in order by the reference's eta_sphere for ac_spheres16
AC_SPHERES16 = [((0.1, -0.2, 0.05), 0.12, 1.8 + 0.05j), ((-0.25, 0.2, -0.1), 0.09, 2.3 + 0.02j),
                ((0.2, 0.25, 0.3), 0.1, 1.4 + 0.08j)]
WAVE_CASES = [("em_sphere16.npz", (0, 0, 1), (1, 0, 0)), ("em_odd567.npz", (0.6, 0.0, 0.8), (0, 1, 0))]


def _eps(tag):
    return 2.0 if tag == "2.0" else golden("em_rotation_seed0.npz")["eps_aniso"]


def _axes(d, prec):
    from em3d_b200 import setup

    return setup.grid_axes_host(tuple(int(n) for n in d["N"]), tuple(float(v) for v in d["L"]), (0.0, 0.0, 0.0),
                                prec)


def _bits(a):
    return a.view(np.float64 if a.dtype == np.complex128 else np.float32)


def _random_scene(seed, count):
    from scipy.spatial.transform import Rotation

    from oracle import materials as om

    rng = np.random.default_rng(seed)
    rows = []
    for _ in range(count):
        radii = rng.uniform(0.05, 0.3, 3)
        c = rng.uniform(-0.3, 0.3, 3)
        R = Rotation.random(random_state=rng).as_matrix()
        e = rng.uniform(1.5, 4.0) + 1j * rng.uniform(0.0, 0.15)
        rows.append(om.pack(c, radii, R, e))
    return np.stack(rows)


# ----------------------------------------------------------------- CPU pins
@pytest.mark.parametrize("fixture,centre,radii,eps", EM_CASES)
@pytest.mark.parametrize("prec,dt", PRECS)
def test_oracle_contrast_equals_reference(fixture, centre, radii, eps, prec, dt):
    from oracle import materials as om

    d = golden(fixture)
    chi = om.sample_contrast(_axes(d, prec), om.pack(centre, radii, None, _eps(eps))[None], om.em_tol(d["L"]),
                             1.0, dt)
    assert np.array_equal(_bits(chi), _bits(d[f"chi_{prec}"]))


@pytest.mark.parametrize("prec,dt", PRECS)
def test_oracle_eta_equals_reference(prec, dt):
    from oracle import materials as om

    d = golden("ac_spheres16.npz")
    shapes = np.stack([om.pack(c, (r,) * 3, None, v) for c, r, v in AC_SPHERES16])
    eta = om.sample_eta(_axes(d, prec), shapes, 0.0, 1.0, dt)
    assert np.array_equal(eta, d[f"eta_{prec}"])


@pytest.mark.parametrize("fixture,orient,amp", WAVE_CASES)
def test_oracle_plane_wave_equals_reference(fixture, orient, amp):
    from oracle import materials as om

    d = golden(fixture)
    w = om.plane_wave(_axes(d, "double"), float(d["k"]), orient, amp)
    assert np.array_equal(w, d["wave_double"])
    # the reference evaluates the single-precision phase in float32
    w32 = om.plane_wave(_axes(d, "single"), float(d["k"]), orient, amp, dtype=np.complex64)
    assert np.abs(w32 - d["wave_single"]).max() < 2e-7


def test_rotation_moves_the_mask():
    """A rotated prolate ellipsoid covers different cells than the unrotated one,
    and a rotation by pi about an axis (a symmetry) covers the same cells."""
    from em3d_b200 import setup
    from oracle import materials as om

    axes = setup.grid_axes_host((24, 24, 24), (1.0, 1.0, 1.0), (0.0, 0.0, 0.0), "double")
    plain = om.scene_hits(axes, om.pack((0, 0, 0), (0.4, 0.1, 0.1))[None], 0.0)
    Rz = np.array([[0.0, -1.0, 0.0], [1.0, 0.0, 0.0], [0.0, 0.0, 1.0]])
    turned = om.scene_hits(axes, om.pack((0, 0, 0), (0.4, 0.1, 0.1), Rz)[None], 0.0)
    flip = np.diag([1.0, -1.0, -1.0])
    same = om.scene_hits(axes, om.pack((0, 0, 0), (0.4, 0.1, 0.1), flip)[None], 0.0)
    assert (plain >= 0).sum() == (turned >= 0).sum() > 0
    assert not np.array_equal(plain, turned)
    assert np.array_equal(plain, same)


def test_painting_order():
    from em3d_b200 import setup
    from oracle import materials as om

    axes = setup.grid_axes_host((8, 8, 8), (1.0, 1.0, 1.0), (0.0, 0.0, 0.0), "double")
    big = om.pack((0, 0, 0), (0.4, 0.4, 0.4), None, 2.0)
    small = om.pack((0, 0, 0), (0.2, 0.2, 0.2), None, 3.0)
    hits = om.scene_hits(axes, np.stack([big, small]), 0.0)
    assert set(np.unique(hits)) == {-1, 0, 1}
    hits_rev = om.scene_hits(axes, np.stack([small, big]), 0.0)
    assert set(np.unique(hits_rev)) == {-1, 1}


def test_sampler_rejects_bad_arguments():
    """Argument errors come back as statuses before any launch (no GPU needed)."""
    import ctypes

    from em3d_b200 import _lib

    lib = _lib.load()
    bg = (ctypes.c_double * 18)()
    rc = lib.em3d_sample_ellipsoids(7, _lib.EM3D_C64, 4, 4, 4, 1, 1, 1, 0, None, 0.0, bg, 1, None)
    assert rc == _lib.EM3D_ERR_INVALID and "kind" in _lib.last_error()
    rc = lib.em3d_sample_ellipsoids(_lib.EM3D_EM, _lib.EM3D_C64, 4, 4, 4, 1, 1, 1, 2, None, 0.0, bg, 1, None)
    assert rc == _lib.EM3D_ERR_INVALID and "shapes" in _lib.last_error()
    rc = lib.em3d_plane_wave(_lib.EM3D_C64, 4, 4, 4, 1, 1, 1, 1.0, bg, bg, 0.0, 3, 1, None)
    assert rc == _lib.EM3D_ERR_INVALID and "sign" in _lib.last_error()


# ------------------------------------------------------------- GPU kernels
@pytest.mark.gpu
@pytest.mark.parametrize("fixture,centre,radii,eps", EM_CASES)
@pytest.mark.parametrize("prec,dt", PRECS)
def test_device_contrast_equals_reference(fixture, centre, radii, eps, prec, dt):
    import em3d_b200 as e
    from em3d_b200 import scenes

    d = golden(fixture)
    be = e.Backend.b200(e.Precision.DOUBLE if prec == "double" else e.Precision.SINGLE)
    grid = e.Grid(N=tuple(int(n) for n in d["N"]), L=tuple(float(v) for v in d["L"]), center=(0.0, 0.0, 0.0),
                  backend=be)
    chi = scenes.sample_scene(grid, [scenes.EllipsoidShape(centre, radii, None, _eps(eps))]).cpu().numpy()
    assert np.array_equal(_bits(chi), _bits(d[f"chi_{prec}"]))


@pytest.mark.gpu
@pytest.mark.parametrize("prec,dt", PRECS)
@pytest.mark.parametrize("N", [(33, 20, 17), (64, 64, 64)])
def test_device_rotated_scene_equals_oracle(prec, dt, N):
    import em3d_b200 as e
    from em3d_b200 import scenes
    from oracle import materials as om

    be = e.Backend.b200(e.Precision.DOUBLE if prec == "double" else e.Precision.SINGLE)
    grid = e.Grid(N=N, L=(1.0, 1.1, 0.9), center=(0.0, 0.02, 0.0), backend=be)
    packed = _random_scene(7, 5)
    tol = scenes.reference_tol(grid)
    got = scenes.sample_scene(grid, packed, background_eps_r=1.2 + 0.01j).cpu().numpy()
    ref = om.sample_contrast(grid.host_axes, packed, tol, 1.2 + 0.01j, dt)
    assert np.array_equal(_bits(got), _bits(ref))
    eta = scenes.sample_scene_eta(grid, packed, eta_outside=1.0).cpu().numpy()
    assert np.array_equal(eta, om.sample_eta(grid.host_axes, packed, 0.0, 1.0, dt))


@pytest.mark.gpu
@pytest.mark.parametrize("prec,dt", PRECS)
def test_device_eta_equals_reference(prec, dt):
    import em3d_b200 as e
    from em3d_b200 import scenes

    d = golden("ac_spheres16.npz")
    be = e.Backend.b200(e.Precision.DOUBLE if prec == "double" else e.Precision.SINGLE)
    grid = e.Grid(N=(16, 16, 16), L=(1.0, 1.0, 1.0), center=(0.0, 0.0, 0.0), backend=be)
    shapes = [scenes.EllipsoidShape(c, (r,) * 3, None, v) for c, r, v in AC_SPHERES16]
    eta = scenes.sample_scene_eta(grid, shapes).cpu().numpy()
    assert np.array_equal(eta, d[f"eta_{prec}"])


@pytest.mark.gpu
@pytest.mark.parametrize("fixture,orient,amp", WAVE_CASES)
def test_device_plane_wave_matches_reference(fixture, orient, amp):
    import em3d_b200 as e
    from em3d_b200 import scenes

    d = golden(fixture)
    for prec, tol in (("double", 1e-14), ("single", 3e-7)):
        be = e.Backend.b200(e.Precision.DOUBLE if prec == "double" else e.Precision.SINGLE)
        grid = e.Grid(N=tuple(int(n) for n in d["N"]), L=tuple(float(v) for v in d["L"]), center=(0.0, 0.0, 0.0),
                      backend=be)
        w = scenes.plane_wave(grid, k=float(d["k"]), orient=orient, amplitude=amp).cpu().numpy()
        assert np.abs(w - d[f"wave_{prec}"]).max() < tol


def test_acoustic_sphere_workload_equals_oracle_scene():
    """The 200-sphere acoustic workload's host builder paints exactly what the
    scene restatement (reference sphere test, tol 0) gives."""
    from em3d_b200 import setup, workloads
    from oracle import materials as om

    for N, count in ((32, 40), (64, 200)):
        case = workloads.acoustic_spheres(N, count=count, seed=1)
        axes = setup.grid_axes_host(case.N, case.L, case.center, "double")
        shapes = np.stack([om.pack(c, (r,) * 3, None, v) for c, r, v in workloads.acoustic_sphere_list(count, 1)])
        assert np.array_equal(case.eta, om.sample_eta(axes, shapes, 0.0, 1.0, np.complex128))


@pytest.mark.gpu
def test_device_acoustic_sphere_workload_equals_host():
    import em3d_b200 as e
    from em3d_b200 import workloads

    for prec in ("double", "single"):
        case = workloads.acoustic_spheres(64, prec, count=200, seed=0)
        be = e.Backend.b200(e.Precision.DOUBLE if prec == "double" else e.Precision.SINGLE)
        grid = e.Grid(N=case.N, L=case.L, center=case.center, backend=be)
        eta = workloads.acoustic_spheres_device(grid, count=200, seed=0).cpu().numpy()
        assert np.array_equal(eta, case.eta)

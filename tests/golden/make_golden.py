"""Generate the golden fixtures in this folder by running the reference em3d.

Run from the repository root, in a container where the reference source is
available read-only:

    python tests/golden/make_golden.py <reference checkout>/src

It imports the UNMODIFIED reference package (qwerty29544/em3d v0.8.0) from the
given path, runs its own public functions on seeded inputs, and writes small
``.npz`` / ``.json`` files next to this script.  Nothing at test time reads
the reference; the tests read these files.
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def _save(name, **arrays):
    path = os.path.join(HERE, name)
    np.savez_compressed(path, **arrays)
    print(f"wrote {name}: {os.path.getsize(path) / 1024:.1f} KiB")


def _rng_field(rng, shape, dtype):
    return (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(dtype)


def main(ref_src: str) -> None:
    sys.path.insert(0, ref_src)
    import em3d
    from em3d import Backend, Grid, Precision, Problem
    from em3d.acoustics import AcousticOperator, eta_sphere, make_acoustic_problem
    from em3d.acoustics.kernel import kernel_on_doubled_grid, self_cell_coefficient
    from em3d.geometry import Ellipsoid, sample_contrast_tensor
    from em3d.operator import Operator, PreparedEMKernel
    from em3d.refraction import cylinder_refraction
    from em3d.solvers import SIM, BiCGStab, SolverConfig, TwoStep
    from em3d.wave import flat_wave_vec
    from em3d.experiments.stationary_validation import true_relative_residual
    from em3d import gamma0

    assert em3d.__version__ == "0.8.0", em3d.__version__
    be = {"double": Backend.numpy(Precision.DOUBLE), "single": Backend.numpy(Precision.SINGLE)}

    # ---- 1. kernel spectra on tiny and odd grids (explicit + adjoint) -------
    for N, L, k in (((4, 3, 3), (1.0, 1.0, 1.0), 1.7), ((4, 3, 2), (1.0, 1.0, 1.0), 2.1),
                    ((5, 6, 7), (1.0, 0.8, 1.3), 3.3)):
        out = {}
        for prec in ("double", "single"):
            grid = Grid(N=N, L=L, center=(0.0, 0.0, 0.0), backend=be[prec])
            pk = PreparedEMKernel.build(grid, k=k, include_adjoint=True, adjoint_storage="explicit")
            out[f"kernel_hat_{prec}"] = pk.kernel_hat
            out[f"kernel_hat_adjoint_{prec}"] = pk.kernel_hat_adjoint
        tag = "x".join(map(str, N))
        _save(f"em_kernel_hat_{tag}.npz", N=np.array(N), L=np.array(L), k=np.array(k), **out)

    # ---- 2. EM matvec / rmatvec, several problems and precisions ------------
    def em_case(name, N, L, k, chi_fn, seed, wave_kw):
        out = {"N": np.array(N), "L": np.array(L), "k": np.array(k)}
        for prec in ("double", "single"):
            grid = Grid(N=N, L=L, center=(0.0, 0.0, 0.0), backend=be[prec])
            chi = chi_fn(grid)
            wave = flat_wave_vec(grid, k=k, **wave_kw)
            problem = Problem(grid=grid, eps_tensor=chi, wave=wave, k0=k, volume=grid.dv * int(np.prod(N)))
            rng = np.random.default_rng(seed)
            u = _rng_field(rng, (3,) + tuple(N), be[prec].complex_dtype)
            op_e = Operator(problem)  # explicit adjoint
            pk_d = PreparedEMKernel.build(grid, k=k, include_adjoint=True, adjoint_storage="derived",
                                          build_strategy="streamed")
            op_d = Operator(problem, prepared_kernel=pk_d)
            out[f"chi_{prec}"] = chi
            out[f"wave_{prec}"] = wave
            out[f"u_{prec}"] = u
            out[f"matvec_u_{prec}"] = op_e.matvec(u)
            out[f"matvec_wave_{prec}"] = op_e.matvec(wave)
            out[f"rmatvec_u_{prec}"] = op_e.rmatvec(u)
            out[f"rmatvec_u_derived_{prec}"] = op_d.rmatvec(u)
        _save(f"em_{name}.npz", **out)

    em_case("sphere16", (16, 16, 16), (1.0, 1.0, 1.0), 4.0,
            lambda g: sample_contrast_tensor(g, background_eps_r=1.0, feature_eps_r=2.0,
                                             geometry=Ellipsoid((0.0, 0.0, 0.0), (0.25, 0.25, 0.25))),
            11, dict(orient=(0, 0, 1), amplitude=(1, 0, 0)))
    em_case("cyl_lossy4", (4, 4, 4), (1.0, 1.0, 1.0), 1.0,
            lambda g: cylinder_refraction(g, eps_real=2.0, eps_imag=0.5, radius=0.3, axis="z"),
            7, dict(orient=(0, 0, 1), amplitude=(1, 0, 0)))
    # anisotropic rotated ellipsoid (the 128^3 workload's material recipe at 12^3)
    from scipy.spatial.transform import Rotation

    R = Rotation.random(random_state=0).as_matrix()
    eps_diag = np.diag([2.5 + 0.1j, 3.0 + 0.2j, 2.0 + 0.05j])
    eps_aniso = R @ eps_diag @ R.T
    em_case("aniso12", (12, 12, 12), (1.0, 1.0, 1.0), 12.0,
            lambda g: sample_contrast_tensor(g, background_eps_r=1.0, feature_eps_r=eps_aniso,
                                             geometry=Ellipsoid((0.0, 0.0, 0.0), (0.30, 0.20, 0.25))),
            3, dict(orient=(0, 0, 1), amplitude=(1, 0, 0)))
    em_case("odd567", (5, 6, 7), (1.0, 0.8, 1.3), 3.3,
            lambda g: sample_contrast_tensor(g, background_eps_r=1.0, feature_eps_r=eps_aniso,
                                             geometry=Ellipsoid((0.05, 0.0, -0.1), (0.45, 0.3, 0.5))),
            5, dict(orient=(0.6, 0.0, 0.8), amplitude=(0, 1, 0)))
    _save("em_rotation_seed0.npz", R=R, eps_aniso=eps_aniso)

    # ---- 3. dense operator known answer (reference test setup, 4^3 lossy) ---
    grid = Grid(N=(4, 4, 4), L=(1.0, 1.0, 1.0), center=(0.0, 0.0, 0.0), backend=be["double"])
    chi = cylinder_refraction(grid, eps_real=2.0, eps_imag=0.5, radius=0.3, axis="z")
    wave = flat_wave_vec(grid, k=1.0, orient=(0, 0, 1), amplitude=(1, 0, 0))
    problem = Problem(grid=grid, eps_tensor=chi, wave=wave, k0=1.0, volume=grid.dv * 64)
    _save("em_dense_cyl_lossy4.npz", A=Operator(problem).to_dense_operator())

    # ---- 4. acoustic ---------------------------------------------------------
    def ac_case(name, N, L, k0, spheres, seed):
        out = {"N": np.array(N), "L": np.array(L), "k0": np.array(k0)}
        for prec in ("double", "single"):
            grid = Grid(N=N, L=L, center=(0.0, 0.0, 0.0), backend=be[prec])
            eta = np.ones(N, dtype=be[prec].complex_dtype)
            for (c, rad, val) in spheres:
                m = eta_sphere(grid, center=c, radius=rad, eta_inside=val, eta_outside=0.0)
                eta = np.where(m != 0, m, eta).astype(be[prec].complex_dtype)
            problem = make_acoustic_problem(grid, eta, k0=k0)
            op = AcousticOperator(problem)
            rng = np.random.default_rng(seed)
            u = _rng_field(rng, tuple(N), be[prec].complex_dtype)
            out[f"eta_{prec}"] = problem.eta
            out[f"wave_{prec}"] = problem.wave
            out[f"u_{prec}"] = u
            out[f"matvec_u_{prec}"] = op.matvec(u)
            out[f"rmatvec_u_{prec}"] = op.rmatvec(u)
            out[f"kernel_{prec}"] = kernel_on_doubled_grid(grid, k0=k0) if max(N) <= 6 else np.zeros(0)
            out[f"self_cell_{prec}"] = np.array(self_cell_coefficient(k0=k0, dv=grid.dv))
        _save(f"ac_{name}.npz", **out)

    ac_case("sphere332", (3, 3, 2), (1.0, 0.8, 0.6), 1.2, [((0.0, 0.0, 0.0), 0.45, 2.0 + 0.2j)], 123)
    ac_case("spheres16", (16, 16, 16), (1.0, 1.0, 1.0), 20.0,
            [((0.1, -0.2, 0.05), 0.12, 1.8 + 0.05j), ((-0.25, 0.2, -0.1), 0.09, 2.3 + 0.02j),
             ((0.2, 0.25, 0.3), 0.1, 1.4 + 0.08j)], 9)
    ac_case("odd765", (7, 6, 5), (1.2, 1.0, 0.9), 5.0, [((0.0, 0.1, 0.0), 0.35, 1.6 + 0.1j)], 21)

    # ---- 5. solvers -----------------------------------------------------------
    sol = {}
    # README-style sphere at 16^3 (k0=4), BiCGStab max_iter 200 rtol 1e-8
    for prec in ("double", "single"):
        grid = Grid(N=(16, 16, 16), L=(1.0, 1.0, 1.0), center=(0.0, 0.0, 0.0), backend=be[prec])
        chi = sample_contrast_tensor(grid, background_eps_r=1.0, feature_eps_r=2.0,
                                     geometry=Ellipsoid((0.0, 0.0, 0.0), (0.25, 0.25, 0.25)))
        wave = flat_wave_vec(grid, k=4.0, orient=(0, 0, 1), amplitude=(1, 0, 0))
        problem = Problem(grid=grid, eps_tensor=chi, wave=wave, k0=4.0, volume=grid.dv * 4096)
        op = Operator(problem)
        rtol = 1e-8 if prec == "double" else 1e-5
        g0 = gamma0.estimate_from_problem(problem, coarse_N=(4, 4, 4))
        sol[f"sphere16_gamma0_{prec}"] = {"mu": [g0.mu.real, g0.mu.imag], "radius": float(g0.radius)}
        for sname, solver in (("bicgstab", BiCGStab(SolverConfig(max_iter=200, rtol=rtol))),
                              ("twostep", TwoStep(SolverConfig(max_iter=200, rtol=rtol))),
                              ("sim", SIM(SolverConfig(max_iter=200, rtol=rtol, mu=g0.mu, radius=g0.radius)))):
            res = solver.solve(op, wave)
            key = f"sphere16_{sname}_{prec}"
            sol[key] = {
                "iterations": res.iterations, "residual_history": [float(v) for v in res.residual_history],
                "converged": bool(res.converged), "matvec_count": res.matvec_count,
                "rmatvec_count": res.rmatvec_count, "residual_action_counts": list(res.residual_action_counts),
                "status": res.status, "true_final_residual": float(res.true_final_residual),
                "true_relative_residual": float(true_relative_residual(op, res.u, wave)),
            }
            np.save(os.path.join(HERE, f"sol_{key}_u.npy"), np.asarray(res.u))
            print(key, res.status, res.iterations, res.residual_history[-1])
    # action budgets, toy problem of the reference solver tests
    grid = Grid(N=(4, 4, 4), L=(1.0, 1.0, 1.0), center=(0.0, 0.0, 0.0), backend=be["double"])
    chi = cylinder_refraction(grid, eps_real=1.1, eps_imag=0.0, radius=0.2, axis="z")
    wave = flat_wave_vec(grid, k=0.5, orient=(0, 0, 1), amplitude=(1, 0, 0))
    problem = Problem(grid=grid, eps_tensor=chi, wave=wave, k0=0.5, volume=grid.dv * 64)
    op = Operator(problem)
    for budget in (1, 2, 3, 4, 5):
        for sname, solver in (("bicgstab", BiCGStab(SolverConfig(max_iter=100, max_operator_actions=budget))),
                              ("twostep", TwoStep(SolverConfig(max_iter=100, max_operator_actions=budget))),
                              ("sim", SIM(SolverConfig(max_iter=100, max_operator_actions=budget, mu=2.0 + 0j,
                                                       radius=1.0)))):
            res = solver.solve(op, wave)
            sol[f"budget{budget}_{sname}"] = {
                "iterations": res.iterations, "residual_history": [float(v) for v in res.residual_history],
                "status": res.status, "matvec_count": res.matvec_count, "rmatvec_count": res.rmatvec_count,
                "residual_action_counts": list(res.residual_action_counts),
            }
    # acoustic solves on the 16^3 spheres case
    grid = Grid(N=(16, 16, 16), L=(1.0, 1.0, 1.0), center=(0.0, 0.0, 0.0), backend=be["double"])
    ac = np.load(os.path.join(HERE, "ac_spheres16.npz"))
    problem = make_acoustic_problem(grid, ac["eta_double"], k0=20.0)
    op = AcousticOperator(problem)
    for sname, solver in (("bicgstab", BiCGStab(SolverConfig(max_iter=300, rtol=1e-8))),
                          ("twostep", TwoStep(SolverConfig(max_iter=300, rtol=1e-8)))):
        res = solver.solve(op, problem.wave)
        key = f"ac16_{sname}_double"
        sol[key] = {
            "iterations": res.iterations, "residual_history": [float(v) for v in res.residual_history],
            "status": res.status, "matvec_count": res.matvec_count, "rmatvec_count": res.rmatvec_count,
            "residual_action_counts": list(res.residual_action_counts),
        }
        np.save(os.path.join(HERE, f"sol_{key}_u.npy"), np.asarray(res.u))
        print(key, res.status, res.iterations, res.residual_history[-1])
    # SIM parameter of the 128^3 anisotropic ellipsoid workload (k0=12)
    grid = Grid(N=(128, 128, 128), L=(1.0, 1.0, 1.0), center=(0.0, 0.0, 0.0), backend=be["single"])
    chi = sample_contrast_tensor(grid, background_eps_r=1.0, feature_eps_r=eps_aniso,
                                 geometry=Ellipsoid((0.0, 0.0, 0.0), (0.30, 0.20, 0.25)))
    wave = flat_wave_vec(grid, k=12.0, orient=(0, 0, 1), amplitude=(1, 0, 0))
    problem = Problem(grid=grid, eps_tensor=chi, wave=wave, k0=12.0, volume=1.0)
    try:
        g0 = gamma0.estimate_from_problem(problem, coarse_N=(4, 4, 4))
        sol["aniso128_gamma0"] = {"mu": [g0.mu.real, g0.mu.imag], "radius": float(g0.radius)}
    except ValueError as exc:  # the reference refuses: record its own message
        sol["aniso128_gamma0"] = {"error": str(exc)}
    print("aniso128 gamma0", sol["aniso128_gamma0"])
    with open(os.path.join(HERE, "solvers.json"), "w") as fh:
        json.dump(sol, fh, indent=1)
    print("wrote solvers.json")


def farfield_fixtures(ref_src: str) -> None:
    """Far fields, RCS curves, the acoustic pattern and Mie comparisons of the
    reference on the committed EM / acoustic golden inputs -> farfield.npz."""
    sys.path.insert(0, ref_src)
    import em3d
    from em3d import Backend, Grid, Precision, Problem, farfield, mie
    from em3d.acoustics import make_acoustic_problem
    from em3d.acoustics import farfield as acff

    be = {"double": Backend.numpy(Precision.DOUBLE), "single": Backend.numpy(Precision.SINGLE)}
    out = {}
    rng = np.random.default_rng(5)
    dirs = rng.standard_normal((16, 3))
    dirs /= np.linalg.norm(dirs, axis=1)[:, None]
    out["em_dirs"] = dirs
    for case, k in (("sphere16", 4.0), ("odd567", 3.3)):
        g = np.load(os.path.join(HERE, f"em_{case}.npz"))
        for prec in ("double", "single"):
            grid = Grid(N=tuple(int(n) for n in g["N"]), L=tuple(float(v) for v in g["L"]), center=(0.0, 0.0, 0.0),
                        backend=be[prec])
            prob = Problem(grid=grid, eps_tensor=g[f"chi_{prec}"], wave=g[f"wave_{prec}"], k0=k,
                           volume=grid.dv * int(np.prod(grid.N)))
            out[f"em_{case}_F_{prec}"] = farfield.scatter_integral(g[f"u_{prec}"], prob, dirs)
            phi, sig = farfield.rcs_plane(g[f"u_{prec}"], prob, n_phi=24, plane="xz")
            out[f"em_{case}_rcs_xz_{prec}"] = sig
            out[f"em_{case}_rcs_single_dir_{prec}"] = np.array(farfield.rcs(g[f"u_{prec}"], prob, dirs[3] * 2.0))
    # the README sphere: the reference's own BiCGStab solution against Mie
    g = np.load(os.path.join(HERE, "em_sphere16.npz"))
    grid = Grid(N=(16, 16, 16), L=(1.0, 1.0, 1.0), center=(0.0, 0.0, 0.0), backend=be["double"])
    prob = Problem(grid=grid, eps_tensor=g["chi_double"], wave=g["wave_double"], k0=4.0, volume=1.0)
    u = np.load(os.path.join(HERE, "sol_sphere16_bicgstab_double_u.npy"))
    cmp = mie.compare_rcs_plane(u, prob, a=0.25, eps_r=2.0, n_phi=120, plane="xz")
    for key in ("sigma_num", "sigma_mie", "shape_err", "scale_ratio", "abs_rel_err"):
        out[f"mie_readme_{key}"] = np.asarray(cmp[key])
    # the Mie series itself on a few parameter sets (lossless, lossy; all planes)
    for tag, (a, eps, k0) in {"a": (0.25, 2.0, 4.0), "b": (0.3, 2.5 + 0.3j, 6.0), "c": (0.1, 4.0, 2.0)}.items():
        co = mie.mie_coefficients(a, eps, k0)
        out[f"mie_{tag}_an"], out[f"mie_{tag}_bn"] = co["a"], co["b"]
        cs = mie.mie_cross_sections(a, eps, k0)
        out[f"mie_{tag}_cross"] = np.array([cs["scat"], cs["ext"], cs["abs"]])
        for plane in ("xy", "xz", "yz"):
            out[f"mie_{tag}_rcs_{plane}"] = mie.mie_rcs_plane(a, eps, k0, n_phi=36, plane=plane)[1]
    # acoustic far field on the spheres case
    ga = np.load(os.path.join(HERE, "ac_spheres16.npz"))
    adirs = rng.standard_normal((24, 3)) * 3.0   # not normalised: the reference normalises
    out["ac_dirs"] = adirs
    for prec in ("double", "single"):
        grid = Grid(N=(16, 16, 16), L=(1.0, 1.0, 1.0), center=(0.0, 0.0, 0.0), backend=be[prec])
        prob = make_acoustic_problem(grid, ga[f"eta_{prec}"], k0=float(ga["k0"]))
        out[f"ac_F_{prec}"] = acff.farfield_amplitude(ga[f"u_{prec}"], prob, adirs)
        out[f"ac_pattern_xz_{prec}"] = acff.pattern_plane(ga[f"u_{prec}"], prob, plane="xz", n_angles=36)[1]
    _save("farfield.npz", **out)
    print("mie readme shape_err", float(cmp["shape_err"]), "scale", float(cmp["scale_ratio"]))


if __name__ == "__main__":
    if len(sys.argv) > 2 and sys.argv[2] == "farfield":
        farfield_fixtures(sys.argv[1])
    else:
        main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference/src")
        farfield_fixtures(sys.argv[1] if len(sys.argv) > 1 else "/root/reference/src")

"""Learned warm start for EM solves: solver-generated training data, training
of the Fourier neural operator (``em3d_b200.fno``) on the GPU, and its
evaluation against the zero-guess solve.

Scene distribution (seeded, one scene per seed): 1-5 ellipsoids with radii
U[0.05, 0.3], a uniform random orientation and centre keeping the ellipsoid in
the unit box, isotropic eps_r U[1.5, 4.0] + i U[0, 0.15] (painted in order);
k0 U[4, 10]; a uniform random incident direction and a uniform random
polarisation orthogonal to it.  Grid: N^3 cells on the unit box centred at 0.

Training pairs ((chi, f) -> u) come from this library's own solver (FP32
BiCGStab to a relative residual of ``data_rtol`` on the FP32 operator); the
inputs are rebuilt on the device from each scene's parameters at every step,
so only the solutions are stored.

The network never decides accuracy: a solve started from its guess stops on
the true residual like any other, and the defect-correction solver falls back
to the zero guess when the guess's true residual is not below ``||f||``.

Command line (runs the whole protocol on one GPU and writes a JSON summary)::

    python -m em3d_b200.warmstart --train 4000 --epochs 8 --eval 256 --eval-n 64,128 --out summary.json
"""
from __future__ import annotations

import argparse
import json
import math
import time
from dataclasses import dataclass, field
from typing import List, Sequence

import numpy as np

from . import _lib
from .backend import Backend, Precision
from .fno import FNO
from .operator import Operator
from .problem import Grid, Problem
from .scenes import EllipsoidShape, plane_wave, sample_scene
from .solvers import BiCGStab, MixedBiCGStab, SolverConfig, true_relative_residual
from .workloads import orthogonal_polarisations

TRAIN_SEEDS = range(0, 4000)
EVAL_SEEDS = range(10000, 10256)


@dataclass(frozen=True)
class Scene:
    seed: int
    shapes: tuple
    k0: float
    direction: tuple
    polarisation: tuple


def random_scene(seed: int) -> Scene:
    from scipy.spatial.transform import Rotation

    rng = np.random.default_rng(int(seed))
    shapes = []
    for _ in range(int(rng.integers(1, 6))):
        radii = rng.uniform(0.05, 0.3, size=3)
        lim = 0.5 - float(radii.max())
        centre = rng.uniform(-lim, lim, size=3)
        R = Rotation.random(random_state=rng).as_matrix()
        eps = complex(rng.uniform(1.5, 4.0), rng.uniform(0.0, 0.15))
        shapes.append(EllipsoidShape(tuple(float(c) for c in centre), tuple(float(r) for r in radii), R, eps))
    k0 = float(rng.uniform(4.0, 10.0))
    d = rng.standard_normal(3)
    d /= np.linalg.norm(d)
    p1, p2 = orthogonal_polarisations(d)
    a = rng.uniform(0.0, 2.0 * math.pi)
    pol = math.cos(a) * p1 + math.sin(a) * p2
    return Scene(int(seed), tuple(shapes), k0, tuple(float(v) for v in d), tuple(float(v) for v in pol))


def unit_grid(N: int, precision: Precision = Precision.SINGLE, device_index: int = 0) -> Grid:
    be = Backend.b200(precision, device_index=device_index)
    return Grid(N=(N, N, N), L=(1.0, 1.0, 1.0), center=(0.0, 0.0, 0.0), backend=be)


def scene_problem(scene: Scene, grid: Grid) -> Problem:
    chi = sample_scene(grid, scene.shapes)
    wave = plane_wave(grid, k=scene.k0, orient=scene.direction, amplitude=scene.polarisation)
    return Problem(grid=grid, eps_tensor=chi, wave=wave, k0=scene.k0, volume=1.0)


def fill_inputs(scs: Sequence[Scene], grid: Grid, chi_out, wave_out) -> None:
    """Network inputs of a batch of scenes, sampled on the device into
    ``chi_out`` (B,3,3,N,N,N) and ``wave_out`` (B,3,N,N,N) (grid's dtype)."""
    for b, sc in enumerate(scs):
        sample_scene(grid, sc.shapes, out=chi_out[b])
        plane_wave(grid, k=sc.k0, orient=sc.direction, amplitude=sc.polarisation, out=wave_out[b])


# ----------------------------------------------------------------- data
@dataclass
class TrainingSet:
    N: int
    scenes: List[Scene]
    u: object                      # (S, 3, N, N, N) complex64, device
    iterations: np.ndarray
    converged: np.ndarray
    seconds: float = 0.0

    @property
    def usable(self) -> np.ndarray:
        return np.flatnonzero(self.converged)


def generate(seeds: Sequence[int], N: int = 64, *, data_rtol: float = 1e-4, max_iter: int = 2000,
             device_index: int = 0, log_every: int = 0) -> TrainingSet:
    """Solve every scene with FP32 BiCGStab and keep the solutions."""
    import torch

    grid = unit_grid(N, Precision.SINGLE, device_index)
    seeds = list(seeds)
    u = torch.empty((len(seeds), 3, N, N, N), dtype=torch.complex64, device=grid.backend.torch_device)
    its = np.zeros(len(seeds), dtype=np.int64)
    ok = np.zeros(len(seeds), dtype=bool)
    scs = []
    solver = BiCGStab(SolverConfig(max_iter=max_iter, rtol=data_rtol))
    t0 = time.perf_counter()
    for i, seed in enumerate(seeds):
        sc = random_scene(seed)
        scs.append(sc)
        prob = scene_problem(sc, grid)
        res = solver.solve(Operator(prob), prob.wave)
        u[i].copy_(res.u)
        its[i] = res.iterations
        ok[i] = bool(res.converged) and bool(np.isfinite(res.true_final_residual))
        if log_every and (i + 1) % log_every == 0:
            print(f"[warmstart] generated {i + 1}/{len(seeds)}  mean its {its[:i + 1].mean():.1f}  "
                  f"{time.perf_counter() - t0:.1f} s", flush=True)
    torch.cuda.synchronize()
    return TrainingSet(N=N, scenes=scs, u=u, iterations=its, converged=ok, seconds=time.perf_counter() - t0)


# ------------------------------------------------------------- training
def train(net: FNO, data: TrainingSet, *, epochs: int = 8, batch: int = 4, lr: float = 1e-3,
          lr_final: float = 1e-5, seed: int = 0, device_index: int = 0, log_every: int = 0) -> List[float]:
    """Adam with a cosine learning-rate decay; returns the mean loss per epoch."""
    import torch

    grid = unit_grid(data.N, Precision.SINGLE, device_index)
    N = data.N
    dev = grid.backend.torch_device
    chi = torch.empty((batch, 3, 3, N, N, N), dtype=torch.complex64, device=dev)
    wave = torch.empty((batch, 3, N, N, N), dtype=torch.complex64, device=dev)
    target = torch.empty((batch, 3, N, N, N), dtype=torch.complex64, device=dev)
    idx = data.usable
    steps_per_epoch = len(idx) // batch
    if steps_per_epoch == 0:
        raise ValueError("not enough converged training solves for one batch")
    total = epochs * steps_per_epoch
    rng = np.random.default_rng(seed)
    history = []
    step = 0
    t0 = time.perf_counter()
    for ep in range(epochs):
        perm = rng.permutation(idx)
        losses = []
        for j in range(steps_per_epoch):
            sel = perm[j * batch:(j + 1) * batch]
            fill_inputs([data.scenes[s] for s in sel], grid, chi, wave)
            torch.index_select(data.u, 0, torch.as_tensor(sel, device=dev), out=target)
            rate = lr_final + 0.5 * (lr - lr_final) * (1.0 + math.cos(math.pi * step / max(total - 1, 1)))
            losses.append(net.train_step(chi, wave, target, lr=rate))
            step += 1
            if log_every and step % log_every == 0:
                print(f"[warmstart] epoch {ep} step {step}/{total} loss {np.mean(losses[-log_every:]):.4f} "
                      f"lr {rate:.2e} {time.perf_counter() - t0:.1f} s", flush=True)
        history.append(float(np.mean(losses)))
    return history


def save(net: FNO, path: str) -> None:
    arrays = {k: v for k, v in net.params_numpy().items()}
    np.savez(path, _width=net.W, _modes=net.m, _layers=net.L, **arrays)


def load(path: str, act: str = "bf16") -> FNO:
    d = np.load(path)
    net = FNO(width=int(d["_width"]), modes=int(d["_modes"]), layers=int(d["_layers"]), act=act)
    net.set_params({k: d[k] for k in d.files if not k.startswith("_")})
    return net


# ----------------------------------------------------------- warm start
def guess(net: FNO, problem: Problem, wave=None, *, half_grid: bool = False):
    """The network's u for ``problem`` (incident field ``wave``, default the
    problem's own), in the problem's dtype (3, N, N, N).

    ``half_grid``: evaluate the network on the grid of half the resolution
    (2x2x2 cell means of the contrast and the incident field, on the device)
    and interpolate its output back to the problem's grid (trilinear between
    cell centres).  A network trained at 64^3 then runs at the resolution it
    was trained on for a 128^3 problem, at an eighth of the cells."""
    import torch

    w = problem.wave if wave is None else wave
    if not half_grid:
        chi = problem.eps_tensor.to(torch.complex64).unsqueeze(0)
        return net.forward(chi, w.to(torch.complex64).unsqueeze(0), train=False)[0].to(problem.wave.dtype)
    N = tuple(int(v) for v in problem.grid.N)
    if any(v % 2 for v in N):
        raise ValueError(f"half_grid needs even grid sizes, got {N}")
    n = tuple(v // 2 for v in N)
    dev = problem.eps_tensor.device
    st = _lib.stream_handle()
    chi = torch.empty((1, 3, 3) + n, dtype=torch.complex64, device=dev)
    _lib.call("em3d_fno_downsample2", _native(problem.eps_tensor), 9, *n, problem.eps_tensor.contiguous().data_ptr(),
              chi.data_ptr(), st)
    wc = w.contiguous()
    wv = torch.empty((1, 3) + n, dtype=torch.complex64, device=dev)
    _lib.call("em3d_fno_downsample2", _native(wc), 3, *n, wc.data_ptr(), wv.data_ptr(), st)
    u = net.forward(chi, wv, train=False)[0].contiguous()
    out = torch.empty((3,) + N, dtype=problem.wave.dtype, device=dev)
    _lib.call("em3d_fno_upsample2", _native(out), 3, *n, u.data_ptr(), out.data_ptr(), st)
    return out


def _native(t) -> int:
    import torch

    if t.dtype == torch.complex64:
        return _lib.EM3D_C64
    if t.dtype == torch.complex128:
        return _lib.EM3D_C128
    raise TypeError(f"expected complex64 or complex128, got {t.dtype}")


# ----------------------------------------------------------- evaluation
@dataclass
class EvalRecord:
    seed: int
    N: int
    k0: float
    shapes: int
    guess_error: float              # ||u_nn - u*|| / ||u*||
    guess_residual: float           # ||f - A u_nn|| / ||f||
    born_residual: float            # ||f - A f|| / ||f||
    nn_ms: float
    runs: dict = field(default_factory=dict)   # mode -> {iterations, ms, true_residual, ...}


def _timed(fn, reps: int):
    """Run ``fn`` ``reps`` times; CUDA-event time of the last run (ms) and its result."""
    import torch

    out = None
    ms = 0.0
    for _ in range(reps):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        out = fn()
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
    return out, ms


def evaluate(net: FNO, seeds: Sequence[int], N: int, *, rtol: float = 1e-6, max_iter: int = 4000,
             reps: int = 2, device_index: int = 0, log_every: int = 0, half_grid: bool = False) -> List[EvalRecord]:
    """Per held-out scene: FP64 BiCGStab and the mixed solve (FP32 BiCGStab with
    FP64 reliable updates, ``MixedBiCGStab``), each from the zero guess and from
    the network's guess, to a TRUE relative residual of ``rtol``; ``reps`` runs
    per solve, the last one timed (graphs captured)."""
    import torch

    grid = unit_grid(N, Precision.DOUBLE, device_index)
    out = []
    for i, seed in enumerate(seeds):
        sc = random_scene(seed)
        prob = scene_problem(sc, grid)
        op64 = Operator(prob)
        op32 = op64.with_precision(Precision.SINGLE)
        f = prob.wave
        u_nn, nn_ms = _timed(lambda: guess(net, prob, half_grid=half_grid), reps)
        u_nn = u_nn.clone()
        cfg = SolverConfig(max_iter=max_iter, rtol=rtol)
        runs = {}
        bic = BiCGStab(cfg)
        dc = MixedBiCGStab(SolverConfig(max_iter=max_iter, rtol=rtol))
        plans = {
            "fp64_zero": lambda: bic.solve(op64, f),
            "fp64_nn": lambda: bic.solve(op64, f, x0=u_nn),
            "mixed_zero": lambda: dc.solve(op64, f, operator_low=op32),
            "mixed_nn": lambda: dc.solve(op64, f, x0=u_nn, operator_low=op32),
        }
        ustar = None
        for name, fn in plans.items():
            res, ms = _timed(fn, reps)
            tr = true_relative_residual(op64, res.u, f)
            entry = {"iterations": int(res.iterations), "matvecs": int(res.matvec_count), "ms": float(ms),
                     "true_residual": float(tr), "status": res.status}
            if name.startswith("mixed"):
                entry.update(outer=int(res.outer_iterations), fp32_matvecs=int(res.fp32_matvecs),
                             fp64_matvecs=int(res.fp64_matvecs), guess_rejected=bool(res.guess_rejected))
            if name == "mixed_nn":
                entry["ms_with_nn"] = float(ms + nn_ms)
            runs[name] = entry
            if name == "fp64_zero":
                ustar = res.u.clone()
        gerr = float(torch.linalg.vector_norm(u_nn - ustar) / torch.linalg.vector_norm(ustar))
        out.append(EvalRecord(seed=int(seed), N=N, k0=sc.k0, shapes=len(sc.shapes), guess_error=gerr,
                              guess_residual=float(true_relative_residual(op64, u_nn, f)),
                              born_residual=float(true_relative_residual(op64, f, f)), nn_ms=float(nn_ms),
                              runs=runs))
        if log_every and (i + 1) % log_every == 0:
            print(f"[warmstart] evaluated {i + 1}/{len(seeds)} at {N}^3", flush=True)
    return out


def summarize(records: Sequence[EvalRecord]) -> dict:
    """Means over the held-out scenes (and the median speed-ups)."""
    if not records:
        return {}
    modes = list(records[0].runs)
    s = {"scenes": len(records), "N": records[0].N,
         "guess_error_mean": float(np.mean([r.guess_error for r in records])),
         "guess_residual_mean": float(np.mean([r.guess_residual for r in records])),
         "born_residual_mean": float(np.mean([r.born_residual for r in records])),
         "nn_ms_mean": float(np.mean([r.nn_ms for r in records]))}
    for m in modes:
        its = [r.runs[m]["iterations"] for r in records]
        ms = [r.runs[m].get("ms_with_nn", r.runs[m]["ms"]) for r in records]
        s[m] = {"iterations_mean": float(np.mean(its)), "ms_mean": float(np.mean(ms)),
                "converged": int(sum(r.runs[m]["status"] == "converged" for r in records)),
                "true_residual_max": float(max(r.runs[m]["true_residual"] for r in records))}
    base = np.array([r.runs["fp64_zero"]["ms"] for r in records])
    for m in modes:
        t = np.array([r.runs[m].get("ms_with_nn", r.runs[m]["ms"]) for r in records])
        s[m]["speedup_vs_fp64_zero_median"] = float(np.median(base / t))
        s[m]["speedup_vs_fp64_zero_total"] = float(base.sum() / t.sum())
    s["mixed_nn"]["guess_rejected"] = int(sum(r.runs["mixed_nn"].get("guess_rejected", False) for r in records))
    return s


def iterations_vs_guess_error(seeds: Sequence[int], N: int = 128, *,
                              errors=(1.0, 0.5, 0.3, 0.2, 0.1, 0.05, 0.02, 0.01, 3e-3, 1e-3, 1e-4),
                              rtol: float = 1e-6, device_index: int = 0, noise_seed: int = 0) -> list:
    """What a guess of a given accuracy saves: for each scene, the mixed
    solve (FP32 BiCGStab, FP64 reliable updates) to true ``rtol`` from
    ``x0 = u* - e ||u*|| d`` for every relative error ``e``, with ``u*`` the
    FP64 solution (true residual 1e-10) and ``d`` a unit direction of two
    kinds: ``"scattered"`` (along the scattered field ``u* - f``, the error a
    network that under- or over-shoots the scattering makes; ``e`` equal to
    ``||u* - f|| / ||u*||`` is the guess ``u = f``) and ``"white"`` (complex
    Gaussian noise, every mode of the grid).  Rows: seed, kind, e, the guess's
    true residual, iterations, matvecs and ms (CUDA events), beside the
    zero-guess solve."""
    import torch

    grid = unit_grid(N, Precision.DOUBLE, device_index)
    solver = MixedBiCGStab(SolverConfig(max_iter=4000, rtol=rtol))
    gen = torch.Generator(device=grid.backend.torch_device).manual_seed(noise_seed)
    rows = []
    for seed in seeds:
        prob = scene_problem(random_scene(seed), grid)
        op64 = Operator(prob)
        op32 = op64.with_precision(Precision.SINGLE)
        f = prob.wave
        ustar = BiCGStab(SolverConfig(max_iter=4000, rtol=1e-10)).solve(op64, f).u
        un = torch.linalg.vector_norm(ustar)
        scat = ustar - f
        dirs = {"scattered": scat / torch.linalg.vector_norm(scat)}
        w = torch.randn(ustar.shape, dtype=ustar.dtype, device=ustar.device, generator=gen)
        dirs["white"] = w / torch.linalg.vector_norm(w)
        solver.solve(op64, f, operator_low=op32)  # warm the engines and graphs
        res, ms = _timed(lambda: solver.solve(op64, f, operator_low=op32), 1)
        rows.append({"seed": int(seed), "kind": "zero", "error": 1.0, "guess_residual": 1.0,
                     "iterations": int(res.iterations), "matvecs": int(res.matvec_count), "ms": ms,
                     "scattered_error_of_f": float(torch.linalg.vector_norm(scat) / un)})
        for kind, d in dirs.items():
            for e in errors:
                x0 = (ustar - (float(e) * un) * d).contiguous()
                r0 = true_relative_residual(op64, x0, f)
                solver.solve(op64, f, x0=x0, operator_low=op32)
                res, ms = _timed(lambda: solver.solve(op64, f, x0=x0, operator_low=op32), 1)
                rows.append({"seed": int(seed), "kind": kind, "error": float(e), "guess_residual": float(r0),
                             "iterations": int(res.iterations), "matvecs": int(res.matvec_count), "ms": ms,
                             "converged": bool(res.converged), "guess_rejected": bool(res.guess_rejected)})
        del op64, op32, ustar
        torch.cuda.empty_cache()
    return rows


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--train", type=int, default=len(TRAIN_SEEDS), help="training scenes (seeds 0..)")
    ap.add_argument("--n", type=int, default=64, help="training grid edge")
    ap.add_argument("--epochs", type=int, default=8)
    ap.add_argument("--batch", type=int, default=4)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--width", type=int, default=32)
    ap.add_argument("--modes", type=int, default=12)
    ap.add_argument("--layers", type=int, default=4)
    ap.add_argument("--eval", type=int, default=len(EVAL_SEEDS), help="held-out scenes (seeds 10000..)")
    ap.add_argument("--eval-n", default="64,128")
    ap.add_argument("--data-rtol", type=float, default=1e-4)
    ap.add_argument("--half-grid", action="store_true",
                    help="evaluate the network on the half-resolution grid and interpolate its output")
    ap.add_argument("--out", default=None, help="JSON summary path")
    ap.add_argument("--save", default=None, help="weights .npz path")
    a = ap.parse_args(argv)
    t0 = time.perf_counter()
    data = generate(range(a.train), a.n, data_rtol=a.data_rtol, log_every=max(a.train // 10, 1))
    gen_s = time.perf_counter() - t0
    net = FNO(width=a.width, modes=a.modes, layers=a.layers, act="bf16", seed=0)
    t1 = time.perf_counter()
    hist = train(net, data, epochs=a.epochs, batch=a.batch, lr=a.lr, log_every=200)
    train_s = time.perf_counter() - t1
    if a.save:
        save(net, a.save)
    summary = {"train": {"scenes": a.train, "N": a.n, "usable": int(len(data.usable)),
                         "data_iterations_mean": float(data.iterations.mean()), "generate_s": gen_s,
                         "epochs": a.epochs, "batch": a.batch, "train_s": train_s, "loss_per_epoch": hist,
                         "parameters": net.num_parameters(), "width": a.width, "modes": a.modes,
                         "layers": a.layers}}
    print(json.dumps(summary["train"]), flush=True)
    del data
    for n in (int(v) for v in a.eval_n.split(",") if v):
        recs = evaluate(net, list(EVAL_SEEDS)[:a.eval], n, log_every=max(a.eval // 4, 1), half_grid=a.half_grid)
        summary[f"eval_{n}"] = summarize(recs)
        print(json.dumps({f"eval_{n}": summary[f"eval_{n}"]}), flush=True)
    summary["total_s"] = time.perf_counter() - t0
    if a.out:
        with open(a.out, "w") as fh:
            json.dump(summary, fh, indent=1)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())

"""What the trained warm start gains over the solve without it.

A small network (4 layers, width 32, 8 modes) is trained on the GPU with the
library's own kernels on 400 solver-generated 32^3 scenes, then compared on 24
held-out scenes against the zero guess (the reference solvers' only start),
against u = f, and against the same network untrained.  The solves started
from the guess stop on the true residual, so accuracy is the same either way.
"""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_trained_warm_start_gains_over_zero_guess():
    from em3d_b200 import warmstart as ws
    from em3d_b200.fno import FNO

    data = ws.generate(range(400), 32, data_rtol=1e-5)
    assert data.converged.all()
    net = FNO(width=32, modes=8, layers=4, act="bf16", seed=0)
    hist = ws.train(net, data, epochs=10, batch=4, lr=2e-3)
    assert hist[-1] < 0.4 * hist[0]

    held_out = range(10000, 10024)
    trained = ws.summarize(ws.evaluate(net, held_out, 32, reps=1, rtol=1e-8))
    untrained = ws.summarize(ws.evaluate(FNO(width=32, modes=8, layers=4, act="bf16", seed=0), held_out, 32,
                                         reps=1, rtol=1e-8))
    print("trained", {k: trained[k] for k in ("guess_error_mean", "guess_residual_mean", "born_residual_mean")},
          "iterations zero/nn", trained["fp64_zero"]["iterations_mean"], trained["fp64_nn"]["iterations_mean"])

    # the gain: the starting residual drops from 1 (zero guess) to well below
    # that of u = f, and training is what brings it there
    assert trained["guess_residual_mean"] < 0.75 * trained["born_residual_mean"]
    assert trained["born_residual_mean"] < 0.6
    assert trained["guess_residual_mean"] < 0.75 * untrained["guess_residual_mean"]
    assert trained["guess_error_mean"] < 0.35
    # every solve from the guess reaches the true residual, and the guess does
    # not cost iterations on average
    for mode in ("fp64_zero", "fp64_nn", "mixed_zero", "mixed_nn"):
        assert trained[mode]["converged"] == 24
    assert trained["fp64_nn"]["true_residual_max"] < 1e-8
    assert trained["mixed_nn"]["true_residual_max"] < 1e-8
    # a guess whose true residual is not below ||f|| falls back to the zero
    # guess; that is rare and those solves converge like the others
    assert trained["mixed_nn"]["guess_rejected"] <= 3
    # what the guess saves: iterations (no slack); the solve time including
    # the network's forward is reported, not asserted (at this scene
    # distribution a 20-25% accurate guess is worth about one iteration, see
    # iterations_vs_guess_error; the untrained network's output is close to
    # u = f, itself a guess of that class)
    assert trained["fp64_nn"]["iterations_mean"] <= trained["fp64_zero"]["iterations_mean"]
    print("ms fp64 zero / nn incl. forward", trained["fp64_zero"]["ms_mean"],
          trained["fp64_nn"]["ms_mean"] + trained["nn_ms_mean"])
    assert np.isfinite(trained["nn_ms_mean"])


def test_solve_time_falls_with_guess_error():
    """The mechanism a warm start relies on: the mixed solve from a guess of
    relative error e needs fewer iterations the smaller e is, and a guess as
    coarse as the network's (e ~ 0.2) saves about one iteration."""
    from em3d_b200 import warmstart as ws

    rows = ws.iterations_vs_guess_error([10000, 10001], 32, errors=(0.2, 1e-2, 1e-4))
    for seed in (10000, 10001):
        its = {(r["kind"], r["error"]): r["iterations"] for r in rows if r["seed"] == seed}
        zero = its[("zero", 1.0)]
        for kind in ("scattered", "white"):
            assert its[(kind, 0.2)] <= zero + 1
            assert its[(kind, 1e-4)] < its[(kind, 1e-2)] <= its[(kind, 0.2)]
    assert all(r.get("converged", True) for r in rows)

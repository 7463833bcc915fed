"""FNO warm-start kernels: forward and hand-written gradients against the
CPU oracle (torch float64 autograd), and a short training run."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _gpu_layout(p):
    """oracle parameter arrays -> GPU names and layouts (W stored ci, co, kx, ky, kz)."""
    out = {"P": p["P"], "pb": p["pb"], "Q": p["Q"], "qb": p["qb"]}
    for l in range(len(p["A"])):
        out[f"A{l}"] = p["A"][l]
        out[f"a{l}"] = p["a"][l]
        out[f"Wre{l}"] = np.ascontiguousarray(p["Wre"][l].transpose(3, 4, 0, 1, 2))
        out[f"Wim{l}"] = np.ascontiguousarray(p["Wim"][l].transpose(3, 4, 0, 1, 2))
    return out


def _oracle_grads(tp):
    g = {"P": tp["P"].grad, "pb": tp["pb"].grad, "Q": tp["Q"].grad, "qb": tp["qb"].grad}
    for l in range(len(tp["A"])):
        g[f"A{l}"] = tp["A"][l].grad
        g[f"a{l}"] = tp["a"][l].grad
        g[f"Wre{l}"] = tp["Wre"][l].grad.permute(3, 4, 0, 1, 2)
        g[f"Wim{l}"] = tp["Wim"][l].grad.permute(3, 4, 0, 1, 2)
    return {k: v.detach().numpy() for k, v in g.items()}


def _rand(rng, shape):
    return (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)) * 0.5


@pytest.mark.parametrize("act,ftol,gtol", [("float", 2e-5, 2e-4), ("bf16", 3e-2, 8e-2)])
def test_fno_forward_and_gradients_match_oracle(act, ftol, gtol):
    import torch

    from em3d_b200.fno import FNO
    from oracle import fno as ofno

    W, m, L, B, N = 6, 2, 2, 2, (8, 6, 8)
    rng = np.random.default_rng(3)
    p = ofno.init_params(W, m, L, seed=4)
    chi = _rand(rng, (B, 3, 3) + N)
    wave = _rand(rng, (B, 3) + N)
    target = _rand(rng, (B, 3) + N) + wave
    net = FNO(width=W, modes=m, layers=L, act=act)
    net.set_params(_gpu_layout(p))
    dchi = torch.as_tensor(chi.astype(np.complex64), device="cuda")
    dwave = torch.as_tensor(wave.astype(np.complex64), device="cuda")
    dtarget = torch.as_tensor(target.astype(np.complex64), device="cuda")
    net.zero_grad()
    pred = net.forward(dchi, dwave, train=True)
    loss, du = net.loss_and_grad(pred, dtarget)
    net.backward(du)
    torch.cuda.synchronize()

    tp = ofno.to_torch(p)
    tchi = torch.as_tensor(chi.astype(np.complex64).astype(np.complex128))
    twave = torch.as_tensor(wave.astype(np.complex64).astype(np.complex128))
    ttarget = torch.as_tensor(target.astype(np.complex64).astype(np.complex128))
    opred = ofno.forward(tp, tchi, twave, m)
    oloss = ofno.relative_l2_loss(opred, ttarget)
    oloss.backward()

    got = pred.cpu().numpy()
    ref = opred.detach().numpy()
    assert np.linalg.norm(got - ref) / np.linalg.norm(ref) < ftol
    assert abs(loss - oloss.item()) < ftol * abs(oloss.item()) * 5
    og = _oracle_grads(tp)
    for k, gref in og.items():
        gg = net.grads[k].cpu().numpy()
        err = np.linalg.norm(gg - gref) / max(np.linalg.norm(gref), 1e-30)
        assert err < gtol, (k, err)


def test_fno_training_reduces_loss():
    """A few Adam steps on a fixed small batch lower the loss (bf16 training)."""
    import torch

    from em3d_b200.fno import FNO

    rng = np.random.default_rng(0)
    B, N = 4, (16, 16, 16)
    chi = torch.as_tensor((_rand(rng, (B, 3, 3) + N) * 0.3).astype(np.complex64), device="cuda")
    wave = torch.as_tensor(_rand(rng, (B, 3) + N).astype(np.complex64), device="cuda")
    target = wave + 0.8 * wave + 0.5 * chi[:, 0, 0].unsqueeze(1)  # linear in the features
    net = FNO(width=8, modes=4, layers=2, act="bf16", seed=1)
    losses = [net.train_step(chi, wave, target, lr=1e-2) for _ in range(60)]
    assert np.all(np.isfinite(losses))
    assert losses[-1] < 0.5 * losses[0], losses[::10]

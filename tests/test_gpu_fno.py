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


@pytest.mark.parametrize("act,tol", [("float", 2e-5), ("bf16", 3e-2)])
@pytest.mark.parametrize("N,W,m", [((16, 12, 32), 32, 5), ((8, 10, 128), 7, 3), ((6, 6, 6), 32, 3)])
def test_fused_row_forward_matches_separate_passes(act, tol, N, W, m):
    """The fused z-row forward (lift + z-DFT, layer + next z-DFT, last layer +
    projection) gives the same u and stored activations as the pass-by-pass
    kernels, in inference and in training mode."""
    import torch

    from em3d_b200.fno import FNO

    rng = np.random.default_rng(11)
    B = 2
    chi = torch.as_tensor((_rand(rng, (B, 3, 3) + N) * 0.3).astype(np.complex64), device="cuda")
    wave = torch.as_tensor(_rand(rng, (B, 3) + N).astype(np.complex64), device="cuda")
    net = FNO(width=W, modes=m, layers=3, act=act, seed=5)
    for train in (False, True):
        a = net._forward_rows(chi, wave, train).clone()
        acts = [t.float().clone() for t in net._buffers(B, N, train)["v"]] if train else []
        b = net._forward_passes(chi, wave, train).clone()
        torch.cuda.synchronize()
        err = float(torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b))
        assert err < tol, (train, err)
        if train:
            for x, y in zip(acts, net._buffers(B, N, train)["v"]):
                e = float(torch.linalg.vector_norm(x - y.float()) / torch.linalg.vector_norm(y.float()))
                assert e < tol * 4, e


@pytest.mark.parametrize("N,m", [((10, 12, 32), 5), ((24, 26, 64), 12), ((24, 24, 128), 12), ((32, 33, 128), 16)])
def test_tensor_core_row_pass_matches_cuda_core_pass(N, m):
    """bf16, width 32: the mma.sync row kernel against the CUDA-core one (the
    twiddles and mode coefficients enter the tensor cores as bf16)."""
    import torch

    from em3d_b200 import _lib
    from em3d_b200.fno import FNO

    rng = np.random.default_rng(12)
    B = 2
    chi = torch.as_tensor((_rand(rng, (B, 3, 3) + N) * 0.3).astype(np.complex64), device="cuda")
    wave = torch.as_tensor(_rand(rng, (B, 3) + N).astype(np.complex64), device="cuda")
    net = FNO(width=32, modes=m, layers=3, act="bf16", seed=2)
    out = {}
    for simt in (1, 0):
        _lib.call("em3d_set_tuning", _lib.EM3D_TUNE_FNO_SIMT, simt)
        for train in (False, True):
            u = net.forward(chi, wave, train).clone()
            acts = [t.float().clone() for t in net._buffers(B, N, train)["v"]] if train else []
            out[(simt, train)] = (u, acts)
    _lib.call("em3d_set_tuning", _lib.EM3D_TUNE_FNO_SIMT, 0)
    torch.cuda.synchronize()
    for train in (False, True):
        a, b = out[(0, train)][0], out[(1, train)][0]
        corr_a, corr_b = a - wave, b - wave   # the network's output proper
        assert float(torch.linalg.vector_norm(corr_a - corr_b) / torch.linalg.vector_norm(corr_b)) < 3e-2
        for x, y in zip(out[(0, train)][1], out[(1, train)][1]):
            assert float(torch.linalg.vector_norm(x - y) / torch.linalg.vector_norm(y)) < 3e-2


@pytest.mark.parametrize("N,m", [((7, 9, 32), 3), ((24, 26, 64), 12), ((24, 24, 128), 12), ((32, 33, 128), 16)])
def test_tcgen05_row_pass_matches_mma_sync_pass(N, m):
    """bf16, width 32: the layer pass on tcgen05 (TMEM accumulators, block-
    diagonal DFT tables as MMA operands) against the mma.sync one, in
    inference and training mode (the last tile of (7, 9, 32) is partial);
    no bounded wait gives up."""
    import torch

    from em3d_b200 import _lib
    from em3d_b200.fno import FNO

    rng = np.random.default_rng(13)
    B = 2
    chi = torch.as_tensor((_rand(rng, (B, 3, 3) + N) * 0.3).astype(np.complex64), device="cuda")
    wave = torch.as_tensor(_rand(rng, (B, 3) + N).astype(np.complex64), device="cuda")
    net = FNO(width=32, modes=m, layers=3, act="bf16", seed=3)
    _lib.load().em3d_fno_failures(1)
    out = {}
    try:
        for mode in (3, 2):
            _lib.call("em3d_set_tuning", _lib.EM3D_TUNE_FNO_SIMT, mode)
            for train in (False, True):
                u = net.forward(chi, wave, train).clone()
                bufs = net._buffers(B, N, train)
                acts = [t.float().clone() for t in bufs["v"]] if train else []
                pre = [t.float().clone() for t in bufs["pre"]] if train else []
                out[(mode, train)] = (u, acts, pre)
    finally:
        _lib.call("em3d_set_tuning", _lib.EM3D_TUNE_FNO_SIMT, 0)
    torch.cuda.synchronize()
    assert _lib.load().em3d_fno_failures(1) == 0
    for train in (False, True):
        a, b = out[(2, train)][0] - wave, out[(3, train)][0] - wave   # the network's output proper
        assert float(torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b)) < 2e-3
        for x, y in zip(out[(2, train)][1] + out[(2, train)][2], out[(3, train)][1] + out[(3, train)][2]):
            assert float(torch.linalg.vector_norm(x - y) / torch.linalg.vector_norm(y)) < 2e-3


@pytest.mark.parametrize("src", ["complex64", "complex128"])
def test_half_grid_resampling_matches_torch(src):
    """2x2x2 means and trilinear interpolation between cell centres against
    torch's avg_pool3d / interpolate(align_corners=False) in FP32."""
    import torch
    import torch.nn.functional as F

    from em3d_b200 import _lib

    dt = getattr(torch, src)
    n = (5, 6, 7)
    C = 4
    x = torch.randn((C,) + tuple(2 * v for v in n), dtype=dt, device="cuda")
    down = torch.empty((C,) + n, dtype=torch.complex64, device="cuda")
    _lib.call("em3d_fno_downsample2", _lib.EM3D_C64 if src == "complex64" else _lib.EM3D_C128, C, *n, x.data_ptr(),
              down.data_ptr(), _lib.stream_handle())
    xr = torch.view_as_real(x.to(torch.complex64)).permute(0, 4, 1, 2, 3).reshape(1, 2 * C, *(2 * v for v in n))
    ref = F.avg_pool3d(xr, 2).reshape(C, 2, *n).permute(0, 2, 3, 4, 1)
    assert torch.allclose(torch.view_as_real(down), ref, atol=1e-6, rtol=1e-5)

    up = torch.empty((C,) + tuple(2 * v for v in n), dtype=dt, device="cuda")
    _lib.call("em3d_fno_upsample2", _lib.EM3D_C64 if src == "complex64" else _lib.EM3D_C128, C, *n, down.data_ptr(),
              up.data_ptr(), _lib.stream_handle())
    dr = torch.view_as_real(down).permute(0, 4, 1, 2, 3).reshape(1, 2 * C, *n)
    ref_up = F.interpolate(dr, scale_factor=2, mode="trilinear", align_corners=False)
    ref_up = ref_up.reshape(C, 2, *(2 * v for v in n)).permute(0, 2, 3, 4, 1)
    assert torch.allclose(torch.view_as_real(up).float(), ref_up, atol=1e-6, rtol=1e-5)


def test_half_grid_guess_composes_the_resampling():
    """guess(..., half_grid=True) is the network on the 2x2x2-averaged inputs,
    interpolated back."""
    import torch

    import em3d_b200 as e
    from em3d_b200 import warmstart as ws
    from em3d_b200.fno import FNO

    net = FNO(width=32, modes=4, layers=2, act="bf16", seed=1)
    prob = ws.scene_problem(ws.random_scene(3), ws.unit_grid(32, e.Precision.DOUBLE, 0))
    got = ws.guess(net, prob, half_grid=True)
    assert got.shape == prob.wave.shape and got.dtype == prob.wave.dtype
    # inputs of the half grid: the means of the fine grid's inputs (in FP64,
    # then rounded to complex64 as the kernel does)
    import torch.nn.functional as F

    def avg(t):
        r = torch.view_as_real(t.to(torch.complex128)).movedim(-1, 0)
        lead = r.shape[:-3]
        y = F.avg_pool3d(r.reshape(-1, 1, 32, 32, 32), 2).reshape(lead + (16, 16, 16))
        return torch.view_as_complex(y.movedim(0, -1).contiguous()).to(torch.complex64)

    u = net.forward(avg(prob.eps_tensor).unsqueeze(0), avg(prob.wave).unsqueeze(0), train=False)[0]
    ur = torch.view_as_real(u).permute(0, 4, 1, 2, 3).reshape(1, 6, 16, 16, 16)
    ref = F.interpolate(ur, scale_factor=2, mode="trilinear", align_corners=False)
    ref = torch.view_as_complex(ref.reshape(3, 2, 32, 32, 32).permute(0, 2, 3, 4, 1).contiguous())
    assert float((got.to(torch.complex64) - ref).abs().max()) < 1e-4 * float(ref.abs().max())

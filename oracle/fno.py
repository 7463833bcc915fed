"""CPU restatement (torch, float64, autograd) of the Fourier-neural-operator
warm start, used to check the GPU forward pass and its hand-written gradients.

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).  The network is not
part of the reference; this file states the architecture that
``em3d_b200/csrc/fno.cu`` implements, from the FNO equations:

  features (24 per cell) = Re/Im of chi_ab (a, b = 0..2, row-major), then
                           Re/Im of the incident field f_c (c = 0..2)
  v0   = P feat + pb                                  (lift to `width`)
  for l in 0..L-1:
      V    = DFT_trunc(v_l)                           (modes kx, ky in [0,m) U [N-m,N), kz in [0,m))
      U    = W_l[mode] V[mode]                        (complex width x width per mode)
      s    = Re(IDFT_trunc(U)),  IDFT weights c_kz / (X Y Z), c_0 = 1, c_kz>0 = 2
      pre  = A_l v_l + a_l + s
      v_l+1 = GELU(pre)  (no activation after the last layer)
  out  = Q v_L + qb                                   (6 channels)
  u    = f + (out_0 + i out_1, out_2 + i out_3, out_4 + i out_5)
"""
from __future__ import annotations

import math

import numpy as np
import torch


def mode_lists(N, m):
    """Retained wave numbers per axis: x and y both signs, z non-negative."""
    X, Y, Z = N
    kx = list(range(m)) + list(range(X - m, X))
    ky = list(range(m)) + list(range(Y - m, Y))
    kz = list(range(m))
    return kx, ky, kz


def dft_matrices(N, m, dtype=torch.complex128):
    """Forward (L x K) and inverse (K x L) truncated DFT matrices per axis."""
    kx, ky, kz = mode_lists(N, m)
    out = []
    for L, ks in zip(N, (kx, ky, kz)):
        n = torch.arange(L, dtype=torch.float64)[:, None]
        k = torch.tensor(ks, dtype=torch.float64)[None, :]
        ang = 2.0 * math.pi * n * k / L
        fwd = torch.exp(-1j * ang).to(dtype)      # (L, K)
        inv = torch.exp(1j * ang).T.to(dtype)     # (K, L)
        out.append((fwd, inv))
    return out


def features(chi, wave):
    """(B, 24, X, Y, Z) real features from chi (B,3,3,X,Y,Z) and wave (B,3,X,Y,Z)."""
    B = chi.shape[0]
    c = chi.reshape(B, 9, *chi.shape[-3:])
    f = torch.stack([c.real, c.imag], dim=2).reshape(B, 18, *chi.shape[-3:])
    w = torch.stack([wave.real, wave.imag], dim=2).reshape(B, 6, *wave.shape[-3:])
    return torch.cat([f, w], dim=1)


def gelu(x):
    return 0.5 * x * (1.0 + torch.erf(x / math.sqrt(2.0)))


def spectral(v, Wre, Wim, mats, m):
    """Re(IDFT_trunc(W . DFT_trunc(v))) for v (B, C, X, Y, Z) real."""
    (fx, ix), (fy, iy), (fz, iz) = mats
    X, Y, Z = v.shape[-3:]
    vc = v.to(torch.complex128)
    V = torch.einsum("bcxyz,zk->bcxyk", vc, fz)
    V = torch.einsum("bcxyk,yj->bcxjk", V, fy)
    V = torch.einsum("bcxjk,xi->bcijk", V, fx)
    W = torch.complex(Wre, Wim)                                  # (2m, 2m, m, Cin, Cout)
    U = torch.einsum("bcijk,ijkcd->bdijk", V, W)
    U = torch.einsum("bdijk,ix->bdxjk", U, ix)
    U = torch.einsum("bdxjk,jy->bdxyk", U, iy)
    ck = torch.full((m,), 2.0, dtype=torch.float64)
    ck[0] = 1.0
    izw = iz * (ck[:, None] / (X * Y * Z))
    return torch.einsum("bdxyk,kz->bdxyz", U, izw.to(torch.complex128)).real


def forward(params, chi, wave, m):
    """``u`` predicted by the network (B,3,X,Y,Z) complex128."""
    N = tuple(chi.shape[-3:])
    mats = dft_matrices(N, m)
    x = features(chi, wave)
    v = torch.einsum("of,bfxyz->boxyz", params["P"], x) + params["pb"][None, :, None, None, None]
    nl = len(params["A"])
    for l in range(nl):
        s = spectral(v, params["Wre"][l], params["Wim"][l], mats, m)
        pre = torch.einsum("oc,bcxyz->boxyz", params["A"][l], v) + params["a"][l][None, :, None, None, None] + s
        v = gelu(pre) if l < nl - 1 else pre
    out = torch.einsum("oc,bcxyz->boxyz", params["Q"], v) + params["qb"][None, :, None, None, None]
    B = out.shape[0]
    o = out.reshape(B, 3, 2, *N)
    return wave + torch.complex(o[:, :, 0], o[:, :, 1])


def relative_l2_loss(pred, target):
    """mean over the batch of ||pred - target||^2 / ||target||^2."""
    B = pred.shape[0]
    d = (pred - target).reshape(B, -1)
    t = target.reshape(B, -1)
    return ((d.abs() ** 2).sum(1) / (t.abs() ** 2).sum(1)).mean()


def init_params(width, modes, layers, seed=0):
    """Random parameters as float64 numpy arrays (names as in the GPU model)."""
    rng = np.random.default_rng(seed)
    m2 = 2 * modes
    p = {
        "P": rng.standard_normal((width, 24)) / math.sqrt(24),
        "pb": rng.standard_normal(width) * 0.1,
        "A": [rng.standard_normal((width, width)) / math.sqrt(width) for _ in range(layers)],
        "a": [rng.standard_normal(width) * 0.1 for _ in range(layers)],
        "Wre": [rng.uniform(-1, 1, (m2, m2, modes, width, width)) / width for _ in range(layers)],
        "Wim": [rng.uniform(-1, 1, (m2, m2, modes, width, width)) / width for _ in range(layers)],
        "Q": rng.standard_normal((6, width)) / math.sqrt(width),
        "qb": rng.standard_normal(6) * 0.1,
    }
    return p


def to_torch(p, requires_grad=True):
    def t(a):
        x = torch.tensor(a, dtype=torch.float64)
        return x.requires_grad_(requires_grad)

    return {k: ([t(a) for a in v] if isinstance(v, list) else t(v)) for k, v in p.items()}

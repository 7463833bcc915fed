"""Fourier-neural-operator warm start for the EM solve (``em3d_b200/csrc/fno.cu``).

The network maps (chi, incident field f) on a grid to a guess of the total
field u; the Krylov solver starts from that guess (``x0``) and the true
residual decides convergence, so accuracy never depends on the network.
Architecture: lift 24 -> width, ``layers`` Fourier layers (truncated
separable DFT with ``modes`` wave numbers per axis and sign, per-mode complex
channel mixing, pointwise linear, GELU), projection width -> 6, and
u = f + (out_0 + i out_1, ...).  Forward, backward and Adam run in the
library's own kernels with bf16 activations and weights (FP32 master weights
and FP32 accumulation); ``act="float"`` keeps everything in FP32 (used to
check the gradients against the CPU oracle).
"""
from __future__ import annotations

import ctypes
import math

import numpy as np

from . import _lib

ACT_BF16, ACT_F32 = 0, 1


def _c(p):
    return ctypes.c_void_p(p)


class FNO:
    """Parameters, forward/backward and optimiser state of one network."""

    def __init__(self, width: int = 32, modes: int = 12, layers: int = 4, act: str = "bf16", seed: int = 0,
                 device=None):
        import torch

        if not (1 <= width <= 32):
            raise ValueError("width must be in [1, 32]")
        self.W, self.m, self.L = int(width), int(modes), int(layers)
        self.act = ACT_BF16 if act == "bf16" else ACT_F32
        self.adt = torch.bfloat16 if act == "bf16" else torch.float32
        self.dev = device or torch.device("cuda")
        self.lib = _lib.load()
        rng = np.random.default_rng(seed)
        W, m2, m = self.W, 2 * self.m, self.m
        init = {
            "P": rng.standard_normal((W, 24)) / math.sqrt(24),
            "pb": np.zeros(W),
            "Q": rng.standard_normal((6, W)) / math.sqrt(W) * 0.1,
            "qb": np.zeros(6),
        }
        for l in range(self.L):
            init[f"A{l}"] = rng.standard_normal((W, W)) / math.sqrt(W)
            init[f"a{l}"] = np.zeros(W)
            init[f"Wre{l}"] = rng.uniform(-1, 1, (W, W, m2, m2, m)) / (W * W)
            init[f"Wim{l}"] = rng.uniform(-1, 1, (W, W, m2, m2, m)) / (W * W)
        self.set_params(init)
        self._bufs = {}
        self._mats = {}
        self.step_count = 0

    # ------------------------------------------------------------------ params
    def set_params(self, arrays: dict) -> None:
        """Load float64/float32 arrays (names P pb A{l} a{l} Wre{l} Wim{l} Q qb)."""
        import torch

        self.master = {k: torch.as_tensor(np.asarray(v, dtype=np.float32), device=self.dev).contiguous()
                       for k, v in arrays.items()}
        self.actw = {}
        for k, v in self.master.items():
            if k in ("pb", "qb") or k.startswith("a"):
                continue
            t = torch.empty(v.shape, dtype=self.adt, device=self.dev)
            _lib.call("em3d_fno_cast", self.act, v.numel(), v.data_ptr(), t.data_ptr(), _lib.stream_handle())
            self.actw[k] = t
        self.grads = {k: torch.zeros_like(v) for k, v in self.master.items()}
        self.m1 = {k: torch.zeros_like(v) for k, v in self.master.items()}
        self.m2 = {k: torch.zeros_like(v) for k, v in self.master.items()}

    def params_numpy(self) -> dict:
        return {k: v.detach().cpu().numpy().astype(np.float64) for k, v in self.master.items()}

    def num_parameters(self) -> int:
        return int(sum(v.numel() for v in self.master.values()))

    def _w(self, k):
        return self.actw[k] if k in self.actw else self.master[k]

    # ---------------------------------------------------------------- matrices
    def _matrices(self, N):
        import torch

        key = tuple(N)
        if key not in self._mats:
            X, Y, Z = key
            m = self.m
            if min(X, Y) < 2 * m or Z < 2 * m:
                raise ValueError(f"grid {key} too small for {m} modes per axis")
            kx = np.array(list(range(m)) + list(range(X - m, X)))
            ky = np.array(list(range(m)) + list(range(Y - m, Y)))
            kz = np.arange(m)

            def fwd(L, ks):
                n = np.arange(L)[:, None]
                return np.exp(-2j * np.pi * n * ks[None, :] / L)       # (L, K)

            mats = {"fz": fwd(Z, kz), "fy": fwd(Y, ky), "fx": fwd(X, kx)}
            mats["iz"] = np.conj(mats["fz"]).T                        # (K, L) = e^{+i}
            mats["iy"] = np.conj(mats["fy"]).T
            mats["ix"] = np.conj(mats["fx"]).T
            self._mats[key] = {k: torch.as_tensor(v.astype(np.complex64), device=self.dev).contiguous()
                               for k, v in mats.items()}
        return self._mats[key]

    def _buffers(self, B, N, train):
        import torch

        key = (B, tuple(N), bool(train))
        if key in self._bufs:
            return self._bufs[key]
        X, Y, Z = N
        W, m = self.W, self.m
        nc = X * Y * Z
        nm = 4 * m * m * m
        f32, c64 = torch.float32, torch.complex64
        d = {
            "v": [torch.empty((B, W, X, Y, Z), dtype=self.adt, device=self.dev) for _ in range(self.L + 1 if train else 2)],
            "pre": [torch.empty((B, W, X, Y, Z), dtype=self.adt, device=self.dev) for _ in range(self.L if train else 1)],
            "Vz": torch.empty((B, W, X, Y, m), dtype=c64, device=self.dev),
            "Vy": torch.empty((B, W, X, 2 * m, m), dtype=c64, device=self.dev),
            "V": [torch.empty((B, W, nm), dtype=c64, device=self.dev) for _ in range(self.L if train else 1)],
            "U": torch.empty((B, W, nm), dtype=c64, device=self.dev),
            "Ux": torch.empty((B, W, X, 2 * m * m), dtype=c64, device=self.dev),
            "Uxy": torch.empty((B, W, X, Y, m), dtype=c64, device=self.dev),
            "u": torch.empty((B, 3, X, Y, Z), dtype=c64, device=self.dev),
        }
        if train:
            d.update({
                "g": torch.empty((B, W, X, Y, Z), dtype=f32, device=self.dev),
                "g2": torch.empty((B, W, X, Y, Z), dtype=f32, device=self.dev),
                "gpre": torch.empty((B, W, X, Y, Z), dtype=f32, device=self.dev),
                "du": torch.empty((B, 3, X, Y, Z), dtype=c64, device=self.dev),
                "terms": torch.empty(2 * B, dtype=torch.float64, device=self.dev),
            })
        del nc
        self._bufs[key] = d
        return d

    # ------------------------------------------------------------------ passes
    def _contract(self, kind, act, outer, L, J, inner, X, M, Y):
        _lib.call("em3d_fno_contract", kind, act, ctypes.c_size_t(outer), L, J, inner, X.data_ptr(), M.data_ptr(),
                  Y.data_ptr(), _lib.stream_handle())

    def forward(self, chi, wave, train: bool = False):
        """u = network(chi, wave): chi (B,3,3,X,Y,Z), wave (B,3,X,Y,Z) complex64 device tensors."""
        Z = wave.shape[-1]
        if 4 <= Z <= 128 and 2 * self.m <= Z and self.m <= 16:
            return self._forward_rows(chi, wave, train)
        return self._forward_passes(chi, wave, train)

    # the y and x DFTs of a layer in one launch each way (em3d_fno_spectral);
    # False: two contractions each way (em3d_fno_contract)
    fused_spectral = True

    def _spectral(self, l, B, N, buf, mats, V):
        """Vz (truncated z-DFT of the layer input) -> Uxy (modes mixed, x and y inverted)."""
        X, Y, Z = N
        W, m = self.W, self.m
        nm = 4 * m * m * m
        st = _lib.stream_handle()
        fused = self.fused_spectral and 8 * (X * (Y + 1) + 6 * m * max(X, Y) + 4 * m * m) <= 227 * 1024
        if fused:
            # y and x DFTs in one launch (one CTA per channel slice and kz mode)
            _lib.call("em3d_fno_spectral", 0, B * W, m, X, Y, buf["Vz"].data_ptr(), mats["fx"].data_ptr(),
                      mats["fy"].data_ptr(), V.data_ptr(), st)
        else:
            self._contract(1, 0, B * W * X, Y, 2 * m, m, buf["Vz"], mats["fy"], buf["Vy"])
            self._contract(1, 0, B * W, X, 2 * m, 2 * m * m, buf["Vy"], mats["fx"], V)
        _lib.call("em3d_fno_modemix", self.act, B, W, nm, V.data_ptr(), self._w(f"Wre{l}").data_ptr(),
                  self._w(f"Wim{l}").data_ptr(), buf["U"].data_ptr(), st)
        if fused:
            _lib.call("em3d_fno_spectral", 1, B * W, m, X, Y, buf["U"].data_ptr(), mats["ix"].data_ptr(),
                      mats["iy"].data_ptr(), buf["Uxy"].data_ptr(), st)
        else:
            self._contract(1, 0, B * W, 2 * m, X, 2 * m * m, buf["U"], mats["ix"], buf["Ux"])
            self._contract(1, 0, B * W * X, 2 * m, Y, m, buf["Ux"], mats["iy"], buf["Uxy"])

    def _forward_rows(self, chi, wave, train):
        """Forward with the fused z-row kernel: lift + first z-DFT, then per
        layer the y/x contractions, mode mixing and inverse, and one row pass
        that applies the layer and produces the next layer's z-DFT (or, after
        the last layer, the projection)."""
        B = wave.shape[0]
        N = tuple(wave.shape[-3:])
        X, Y, Z = N
        W, m, Lyr = self.W, self.m, self.L
        mats = self._matrices(N)
        buf = self._buffers(B, N, train)
        st = _lib.stream_handle()
        chi = chi.contiguous()
        wave = wave.contiguous()
        v = buf["v"]

        def ptr(t):
            return None if t is None else t.data_ptr()

        _lib.call("em3d_fno_row_forward", self.act, 1, B, W, X, Y, Z, m, chi.data_ptr(), wave.data_ptr(), None, None,
                  self._w("P").data_ptr(), self.master["pb"].data_ptr(), 0, None, v[0].data_ptr(),
                  buf["Vz"].data_ptr(), None, None, None, st)
        for l in range(Lyr):
            last = l == Lyr - 1
            vin = v[l] if train else v[l % 2]
            vout = v[l + 1] if train else (None if last else v[(l + 1) % 2])
            V = buf["V"][l] if train else buf["V"][0]
            self._spectral(l, B, N, buf, mats, V)
            _lib.call("em3d_fno_row_forward", self.act, 0, B, W, X, Y, Z, m, None, wave.data_ptr(), vin.data_ptr(),
                      buf["Uxy"].data_ptr(), self._w(f"A{l}").data_ptr(), self.master[f"a{l}"].data_ptr(),
                      int(not last), ptr(buf["pre"][l]) if train else None, ptr(vout),
                      None if last else buf["Vz"].data_ptr(), self._w("Q").data_ptr() if last else None,
                      self.master["qb"].data_ptr() if last else None, buf["u"].data_ptr() if last else None, st)
        self._last = (chi, wave, B, N)
        return buf["u"]

    def _forward_passes(self, chi, wave, train: bool = False):
        """Forward as separate passes (any Z up to 1024)."""
        B = wave.shape[0]
        N = tuple(wave.shape[-3:])
        X, Y, Z = N
        W, m, Lyr = self.W, self.m, self.L
        nm = 4 * m * m * m
        nc = X * Y * Z
        mats = self._matrices(N)
        buf = self._buffers(B, N, train)
        st = _lib.stream_handle()
        chi = chi.contiguous()
        wave = wave.contiguous()
        v = buf["v"]
        _lib.call("em3d_fno_lift", self.act, B, ctypes.c_size_t(nc), W, chi.data_ptr(), wave.data_ptr(),
                  self._w("P").data_ptr(), self.master["pb"].data_ptr(), v[0].data_ptr(), st)
        for l in range(Lyr):
            vin = v[l] if train else v[l % 2]
            vout = v[l + 1] if train else v[(l + 1) % 2]
            pre = buf["pre"][l] if train else buf["pre"][0]
            V = buf["V"][l] if train else buf["V"][0]
            self._contract(0, self.act, B * W * X * Y, Z, m, 1, vin, mats["fz"], buf["Vz"])
            self._contract(1, 0, B * W * X, Y, 2 * m, m, buf["Vz"], mats["fy"], buf["Vy"])
            self._contract(1, 0, B * W, X, 2 * m, 2 * m * m, buf["Vy"], mats["fx"], V)
            _lib.call("em3d_fno_modemix", self.act, B, W, nm, V.data_ptr(), self._w(f"Wre{l}").data_ptr(),
                      self._w(f"Wim{l}").data_ptr(), buf["U"].data_ptr(), st)
            self._contract(1, 0, B * W, 2 * m, X, 2 * m * m, buf["U"], mats["ix"], buf["Ux"])
            self._contract(1, 0, B * W * X, 2 * m, Y, m, buf["Ux"], mats["iy"], buf["Uxy"])
            _lib.call("em3d_fno_layer_out", self.act, B, W, X, Y, Z, m, vin.data_ptr(), buf["Uxy"].data_ptr(),
                      self._w(f"A{l}").data_ptr(), self.master[f"a{l}"].data_ptr(), int(l < Lyr - 1),
                      pre.data_ptr(), vout.data_ptr(), st)
        vlast = v[Lyr] if train else v[Lyr % 2]
        _lib.call("em3d_fno_project", self.act, B, ctypes.c_size_t(nc), W, vlast.data_ptr(), self._w("Q").data_ptr(),
                  self.master["qb"].data_ptr(), wave.data_ptr(), buf["u"].data_ptr(), st)
        self._last = (chi, wave, B, N)
        return buf["u"]

    def zero_grad(self):
        for g in self.grads.values():
            g.zero_()

    def backward(self, du):
        """Accumulate parameter gradients for dL/du = ``du`` (complex64, dL/dRe + i dL/dIm)."""
        chi, wave, B, N = self._last
        X, Y, Z = N
        W, m, Lyr = self.W, self.m, self.L
        nm = 4 * m * m * m
        nc = X * Y * Z
        mats = self._matrices(N)
        buf = self._buffers(B, N, True)
        st = _lib.stream_handle()
        g, g2 = buf["g"], buf["g2"]
        G = self.grads
        _lib.call("em3d_fno_project_bwd", self.act, B, ctypes.c_size_t(nc), W, buf["v"][Lyr].data_ptr(),
                  self._w("Q").data_ptr(), du.data_ptr(), g.data_ptr(), G["Q"].data_ptr(), G["qb"].data_ptr(), st)
        for l in reversed(range(Lyr)):
            # g: gradient wrt v[l+1] -> g2: gradient wrt v[l]
            _lib.call("em3d_fno_layer_out_bwd", self.act, B, W, X, Y, Z, m, g.data_ptr(), buf["pre"][l].data_ptr(),
                      self._w(f"A{l}").data_ptr(), int(l < Lyr - 1), buf["gpre"].data_ptr(), g2.data_ptr(),
                      buf["Uxy"].data_ptr(), st)
            _lib.call("em3d_fno_pointwise_wgrad", self.act, B, ctypes.c_size_t(nc), W, buf["gpre"].data_ptr(),
                      buf["v"][l].data_ptr(), G[f"A{l}"].data_ptr(), G[f"a{l}"].data_ptr(), st)
            # spectral path: adjoints in reverse order (Uxy holds dL/dUxy); the
            # adjoint of a contraction with M is the contraction with conj(M)^T
            self._contract(1, 0, B * W * X, Y, 2 * m, m, buf["Uxy"], mats["fy"], buf["Ux"])
            self._contract(1, 0, B * W, X, 2 * m, 2 * m * m, buf["Ux"], mats["fx"], buf["U"])
            dV = self._dv(buf)
            _lib.call("em3d_fno_modemix_bwd", self.act, B, W, nm, buf["V"][l].data_ptr(), buf["U"].data_ptr(),
                      self._w(f"Wre{l}").data_ptr(), self._w(f"Wim{l}").data_ptr(), dV.data_ptr(),
                      G[f"Wre{l}"].data_ptr(), G[f"Wim{l}"].data_ptr(), st)
            self._contract(1, 0, B * W, 2 * m, X, 2 * m * m, dV, mats["ix"], buf["Vy"])
            self._contract(1, 0, B * W * X, 2 * m, Y, m, buf["Vy"], mats["iy"], buf["Vz"])
            self._contract(2, 0, B * W * X * Y, m, Z, 1, buf["Vz"], mats["iz"], g2)
            g, g2 = g2, g
        _lib.call("em3d_fno_lift_bwd", B, ctypes.c_size_t(nc), W, chi.data_ptr(), wave.data_ptr(), g.data_ptr(),
                  G["P"].data_ptr(), G["pb"].data_ptr(), st)

    def _dv(self, buf):
        import torch

        if "dV" not in buf:
            buf["dV"] = torch.empty_like(buf["U"])
        return buf["dV"]

    def loss_and_grad(self, pred, target):
        """Relative L2 loss (mean over the batch) and its gradient wrt ``pred``."""
        B = pred.shape[0]
        n = pred[0].numel()
        buf = self._buffers(B, tuple(pred.shape[-3:]), True)
        _lib.call("em3d_fno_loss", B, ctypes.c_size_t(n), pred.data_ptr(), target.contiguous().data_ptr(),
                  buf["terms"].data_ptr(), buf["du"].data_ptr(), _lib.stream_handle())
        t = buf["terms"].view(B, 2)
        loss = float((t[:, 0] / t[:, 1]).mean())
        return loss, buf["du"]

    def adam_step(self, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
        self.step_count += 1
        st = _lib.stream_handle()
        for k, w in self.master.items():
            wact = self.actw.get(k)
            _lib.call("em3d_fno_adam", self.act, ctypes.c_size_t(w.numel()), w.data_ptr(), self.grads[k].data_ptr(),
                      self.m1[k].data_ptr(), self.m2[k].data_ptr(), ctypes.c_float(lr), ctypes.c_float(b1),
                      ctypes.c_float(b2), ctypes.c_float(eps), self.step_count,
                      None if wact is None else wact.data_ptr(), st)

    def train_step(self, chi, wave, target, lr=1e-3):
        self.zero_grad()
        pred = self.forward(chi, wave, train=True)
        loss, du = self.loss_and_grad(pred, target)
        self.backward(du)
        self.adam_step(lr=lr)
        return loss


def predict_x0(net: FNO, problem, dtype=None):
    """Warm start for a solve of ``problem``: the network's u as a tensor of the
    problem's complex dtype (shape (3, Nx, Ny, Nz))."""
    import torch

    chi = problem.eps_tensor.to(torch.complex64)[None]
    wave = problem.wave.to(torch.complex64)[None]
    u = net.forward(chi, wave, train=False)[0]
    out = u.to(dtype or problem.wave.dtype)
    # a tensor of its own: the network's output buffer is reused by its next forward
    return out.clone() if out.data_ptr() == u.data_ptr() else out

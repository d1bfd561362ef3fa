"""Learned control variate for the correlator C(tau) = <|det S_N(tau)|^2>.

A small 3-D convolutional network g(phi) reads the auxiliary-field time
slices of a configuration (block means of phi over (L/G)^3 sites per slice)
and predicts log C(tau) of that configuration.  It is trained on
(field, correlator) pairs the method itself produces, with the library's
hand-written kernels (csrc/cvnet.cu: BF16 conv weights, FP32 accumulation,
forward, backward and Adam), and enters the estimator

    C_cv(tau) = mean_i [ C_i(tau) - c(tau) (g_i(tau) - <g(tau)>) ]

with <g> from many extra field draws (fields only: no propagation), and
c(tau) fixed from the training pairs, so the estimator stays unbiased: E[g_i]
= E[<g>].  The plain estimator mean_i C_i(tau) is the fallback and the yardstick
of the variance reduction.

No counterpart in the reference (its drivers write plain block averages:
production/slater_det/main.C:208-241).
"""
from __future__ import annotations

import ctypes
import math
import time
from dataclasses import dataclass
from typing import Dict, Optional

import numpy as np
import torch

from . import _capi as C
from ._capi import lib
from .api import Context, Ensemble, EnsembleJob, default_context, draw_z2_bits, momenta


def _p(t: Optional[torch.Tensor]):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


@dataclass
class NetShape:
    T: int              # input channels: time slices (and outputs: log C(tau), tau < T)
    G: int = 8          # coarse lattice G^3
    C: int = 16         # conv channels
    H: int = 32         # hidden units of the head

    @property
    def GS(self) -> int:
        return self.G ** 3


class ControlVariateNet:
    """Parameters (FP32 masters + BF16 conv copies), Adam state and the
    forward / backward passes over the device kernels."""

    def __init__(self, shape: NetShape, seed: int = 0, ctx: Optional[Context] = None):
        self.ctx = ctx or default_context()
        self.s = shape
        dev = self.ctx.device
        g = torch.Generator().manual_seed(seed)
        s = shape

        def init(*dims, fan_in):
            return (torch.randn(*dims, generator=g) * (1.0 / math.sqrt(fan_in))).to(dev)

        self.params: Dict[str, torch.Tensor] = {
            "w1": init(s.C, s.T, 27, fan_in=s.T * 27), "b1": torch.zeros(s.C, device=dev),
            "w2": init(s.C, s.C, 27, fan_in=s.C * 27), "b2": torch.zeros(s.C, device=dev),
            "w3": init(s.C, s.C, 27, fan_in=s.C * 27), "b3": torch.zeros(s.C, device=dev),
            "hw": init(s.H, s.C, fan_in=s.C), "hb": torch.zeros(s.H, device=dev),
            "ow": init(s.T, s.H, fan_in=s.H), "ob": torch.zeros(s.T, device=dev),
        }
        for k in self.params:
            self.params[k] = self.params[k].float().contiguous()
        self.bf16 = {k: self.params[k].to(torch.bfloat16).contiguous() for k in ("w1", "w2", "w3")}
        self.m = {k: torch.zeros_like(v) for k, v in self.params.items()}
        self.v = {k: torch.zeros_like(v) for k, v in self.params.items()}
        self.grads = {k: torch.zeros_like(v) for k, v in self.params.items()}
        self.step_count = 0
        self._bufs: Dict[int, Dict[str, torch.Tensor]] = {}
        # target standardisation (log C per tau)
        self.mu = torch.zeros(s.T, dtype=torch.float64)
        self.sigma = torch.ones(s.T, dtype=torch.float64)

    def refresh_bf16(self) -> None:
        for k in ("w1", "w2", "w3"):
            self.bf16[k].copy_(self.params[k].to(torch.bfloat16))

    def _buffers(self, B: int) -> Dict[str, torch.Tensor]:
        if B not in self._bufs:
            s, dev = self.s, self.ctx.device
            act = lambda: torch.empty((B, s.C, s.GS), dtype=torch.bfloat16, device=dev)  # noqa: E731
            pre = lambda: torch.empty((B, s.C, s.GS), dtype=torch.float32, device=dev)  # noqa: E731
            self._bufs[B] = {"z1": pre(), "a1": act(), "z2": pre(), "a2": act(), "z3": pre(), "a3": act(),
                             "p": torch.empty((B, s.C), device=dev), "h": torch.empty((B, s.H), device=dev),
                             "y": torch.empty((B, s.T), device=dev), "dy": torch.empty((B, s.T), device=dev),
                             "dzh": torch.empty((B, s.H), device=dev), "dz3": pre(), "dz2": pre(), "dz1": pre(),
                             "loss": torch.empty(B, device=dev)}
        return self._bufs[B]

    # ------------------------------------------------------------ passes
    def forward(self, x: torch.Tensor) -> torch.Tensor:
        """x [B, T, G^3] BF16 -> standardised predictions [B, T] (FP32 view of a work buffer)."""
        s, L, ctx = self.s, lib(), self.ctx
        B = x.shape[0]
        b = self._buffers(B)
        P = self.params
        ctx.check(L.nrcps_cv_conv_forward(ctx.handle, _p(x), s.T, s.C, s.G, B, _p(self.bf16["w1"]), _p(P["b1"]),
                                          _p(b["z1"]), _p(b["a1"])), "cv conv1")
        ctx.check(L.nrcps_cv_conv_forward(ctx.handle, _p(b["a1"]), s.C, s.C, s.G, B, _p(self.bf16["w2"]),
                                          _p(P["b2"]), _p(b["z2"]), _p(b["a2"])), "cv conv2")
        ctx.check(L.nrcps_cv_conv_forward(ctx.handle, _p(b["a2"]), s.C, s.C, s.G, B, _p(self.bf16["w3"]),
                                          _p(P["b3"]), _p(b["z3"]), _p(b["a3"])), "cv conv3")
        ctx.check(L.nrcps_cv_head_forward(ctx.handle, _p(b["a3"]), s.C, s.G, B, _p(P["hw"]), _p(P["hb"]), s.H,
                                          _p(P["ow"]), _p(P["ob"]), s.T, _p(b["p"]), _p(b["h"]), _p(b["y"])),
                  "cv head")
        return b["y"]

    def tc_inference_supported(self) -> bool:
        s = self.s
        return s.G == 8 and s.T % 16 == 0 and s.T <= 64 and s.C == 16 and s.H <= 64

    def infer(self, x: torch.Tensor) -> torch.Tensor:
        """Standardised predictions [B, T] for inference: one tensor-core kernel
        (nrcps_cv_forward_tc) for the whole network where the shape allows it
        (G = 8, T a multiple of 16 up to 64), else the layer-by-layer kernels
        of forward().  No activations are kept for a backward pass."""
        if not self.tc_inference_supported():
            return self.forward(x)
        s, ctx = self.s, self.ctx
        B = x.shape[0]
        P = self.params
        y = torch.empty((B, s.T), dtype=torch.float32, device=ctx.device)
        W = (ctypes.c_void_p * 3)(*[self.bf16[k].data_ptr() for k in ("w1", "w2", "w3")])
        bias = (ctypes.c_void_p * 3)(*[P[k].data_ptr() for k in ("b1", "b2", "b3")])
        ctx.check(lib().nrcps_cv_forward_tc(ctx.handle, _p(x), s.T, s.G, B, W, bias, _p(P["hw"]), _p(P["hb"]), s.H,
                                            _p(P["ow"]), _p(P["ob"]), s.T, _p(y)), "cv forward (tensor cores)")
        return y

    def backward(self, x: torch.Tensor, target: torch.Tensor) -> float:
        """Gradients of 0.5 mean (y - target)^2 after forward(x); returns the loss."""
        s, L, ctx = self.s, lib(), self.ctx
        B = x.shape[0]
        b = self._buffers(B)
        P, G_ = self.params, self.grads
        ctx.check(L.nrcps_cv_head_backward(ctx.handle, _p(b["y"]), _p(target), s.T, B, _p(b["h"]), s.H, _p(P["ow"]),
                                           _p(P["hw"]), s.C, _p(b["a3"]), s.G, _p(b["p"]), _p(b["dy"]), _p(b["dzh"]),
                                           _p(b["dz3"]), _p(b["loss"]), _p(G_["ow"]), _p(G_["ob"]), _p(G_["hw"]),
                                           _p(G_["hb"])), "cv head backward")
        ctx.check(L.nrcps_cv_conv_backward(ctx.handle, _p(b["dz3"]), _p(b["a2"]), _p(b["a2"]), s.C, s.C, s.G, B,
                                           _p(self.bf16["w3"]), _p(G_["w3"]), _p(G_["b3"]), _p(b["dz2"])),
                  "cv conv3 backward")
        ctx.check(L.nrcps_cv_conv_backward(ctx.handle, _p(b["dz2"]), _p(b["a1"]), _p(b["a1"]), s.C, s.C, s.G, B,
                                           _p(self.bf16["w2"]), _p(G_["w2"]), _p(G_["b2"]), _p(b["dz1"])),
                  "cv conv2 backward")
        ctx.check(L.nrcps_cv_conv_backward(ctx.handle, _p(b["dz1"]), _p(x), None, s.T, s.C, s.G, B,
                                           _p(self.bf16["w1"]), _p(G_["w1"]), _p(G_["b1"]), None),
                  "cv conv1 backward")
        return float(b["loss"].sum().item()) / (B * s.T)

    def adam(self, lr: float = 2e-3, beta1: float = 0.9, beta2: float = 0.999, eps: float = 1e-8) -> None:
        self.step_count += 1
        for k, w in self.params.items():
            bf = self.bf16.get(k)
            self.ctx.check(lib().nrcps_cv_adam(self.ctx.handle, _p(w), _p(self.grads[k]), _p(self.m[k]),
                                               _p(self.v[k]), w.numel(), ctypes.c_float(lr), ctypes.c_float(beta1),
                                               ctypes.c_float(beta2), ctypes.c_float(eps), self.step_count, _p(bf)),
                           "cv adam")

    # -------------------------------------------------------- training
    def fit(self, X: torch.Tensor, logC: torch.Tensor, epochs: int = 20, batch: int = 256, lr: float = 2e-3,
            seed: int = 0) -> list:
        """X [n, T, G^3] BF16 features, logC [n, T] targets (log |det|^2, FP64);
        standardises the targets per tau and trains; returns the epoch losses."""
        self.mu = logC.mean(0).double().cpu()
        self.sigma = logC.std(0).double().cpu().clamp_min(1e-12)
        Yt = ((logC.double().cpu() - self.mu) / self.sigma).float().to(self.ctx.device)
        n = X.shape[0]
        g = torch.Generator().manual_seed(seed)
        losses = []
        for _ in range(epochs):
            perm = torch.randperm(n, generator=g).to(self.ctx.device)
            tot, cnt = 0.0, 0
            for i in range(0, n - batch + 1, batch):
                idx = perm[i:i + batch]
                xb, yb = X[idx].contiguous(), Yt[idx].contiguous()
                self.forward(xb)
                tot += self.backward(xb, yb)
                cnt += 1
                self.adam(lr)
            losses.append(tot / max(cnt, 1))
        return losses

    def predict_logC(self, X: torch.Tensor, chunk: int = 4096) -> torch.Tensor:
        """Predicted log C(tau) [n, T] (FP64, de-standardised)."""
        out = []
        for i in range(0, X.shape[0], chunk):
            y = self.infer(X[i:i + chunk].contiguous()).double().cpu()
            out.append(y * self.sigma + self.mu)
        return torch.cat(out)


# ------------------------------------------------------------------ data
def coarse_fields(bits, bit0: int, L: int, T: int, G: int, n: int, ctx: Context) -> torch.Tensor:
    """Block means [n, T, G^3] BF16 of the Z2 fields of n configurations whose
    slice t of configuration c is bits bit0 + (c T + t) L^3 ... (bits: a
    device tensor or a device address)."""
    x = torch.empty((n, T, G ** 3), dtype=torch.bfloat16, device=ctx.device)
    b = ctypes.c_void_p(bits) if isinstance(bits, int) else _p(bits)
    ctx.check(lib().nrcps_cv_coarse_z2(ctx.handle, b, bit0, L, T, G, n, _p(x)), "cv coarse")
    return x


def sample_z2_features(seed: int, first: int, L: int, T: int, G: int, n: int, ctx: Context) -> torch.Tensor:
    """Block means [n, T, G^3] BF16 of n fresh uniform Z2 fields (numbers
    first .. first + n - 1 of the Philox stream `seed`), drawn directly from
    their exact distribution: the mean of (L/G)^3 independent +-1 sites."""
    x = torch.empty((n, T, G ** 3), dtype=torch.bfloat16, device=ctx.device)
    ctx.check(lib().nrcps_cv_sample_z2_features(ctx.handle, seed, first, L, T, G, n, _p(x)), "cv sample features")
    return x


def generate_pairs(L: int, T: int, fermi_energy: float, seed: int, n_conf: int, first_conf: int = 0,
                   chunk: int = 1024, G: int = 8, precision: str = "f32", qr_period: int = 8,
                   ctx: Optional[Context] = None):
    """(features, C) pairs the method produces: runs the ensemble (Z2 fields,
    a = 0.5, RANLXS2) for configurations [first_conf, first_conf + n_conf) and
    coarse-grains the same stream window.  Returns X [n, T, G^3] BF16 and
    C [n, T] = |det S_N(tau)|^2 (FP64, device)."""
    ctx = ctx or default_context()
    idx, _, _ = momenta((L, L, L), "PERFECT", 1.0, fermi_energy, 2.0)
    V = L ** 3
    Xs, Cs = [], []
    ens = None  # one ensemble per chunk size, run at each chunk's first configuration
    try:
        for c0 in range(first_conf, first_conf + n_conf, chunk):
            m = min(chunk, first_conf + n_conf - c0)
            if ens is None or ens.job.n_conf != m:
                if ens is not None:
                    ens.close()
                ens = Ensemble(EnsembleJob(L=L, T=T, n_conf=m, seed=seed, precision=precision,
                                           fermi_energy=fermi_energy, qr_period=qr_period),
                               plane_wave_index=idx, ctx=ctx)
            d = ens.run(c0)
            Cs.append((d[:, :, -1].abs() ** 2).to(torch.float64))  # a copy: the next run reuses d
            # the features from the run's own fields (the same stream window)
            Xs.append(coarse_fields(ens.field_bits_ptr(), 0, L, T, G, m, ctx))
    finally:
        if ens is not None:
            ens.close()
    return torch.cat(Xs), torch.cat(Cs)


def extra_fields_mean_g(net: ControlVariateNet, L: int, seed: int, first_conf: int, n_fields: int,
                        chunk: int = 8192, ctx: Optional[Context] = None, sampler: str = "philox"):
    """<g(tau)> over n_fields extra field draws (no propagation): mean and
    standard error of exp(predicted log C) per tau, and the GPU seconds.

    sampler "philox" draws the block-mean features directly from their exact
    distribution (sample_z2_features); "ranlux" draws whole RANLXS2 fields
    and coarse-grains them (the generator of the ensemble, 2 M bits per
    field).  Both give independent fields of the same distribution."""
    if sampler not in ("philox", "ranlux"):
        raise ValueError(f"unknown sampler {sampler!r}")
    ctx = ctx or net.ctx
    T, G, V = net.s.T, net.s.G, L ** 3
    # sums on the device: no host round trip per chunk
    s1 = torch.zeros(T, dtype=torch.float64, device=ctx.device)
    s2 = torch.zeros(T, dtype=torch.float64, device=ctx.device)
    mu, sigma = net.mu.to(ctx.device), net.sigma.to(ctx.device)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for c0 in range(first_conf, first_conf + n_fields, chunk):
        m = min(chunk, first_conf + n_fields - c0)
        if sampler == "philox":
            x = sample_z2_features(seed, c0, L, T, G, m, ctx)
        else:
            bits = draw_z2_bits("RANLXS2", seed, c0 * T * V, m * T * V, ctx)
            x = coarse_fields(bits, 0, L, T, G, m, ctx)
        g = torch.exp(net.infer(x).double() * sigma + mu)  # predict_logC, kept on the device
        s1 += g.sum(0)
        s2 += (g ** 2).sum(0)
    torch.cuda.synchronize()
    el = time.perf_counter() - t0
    s1, s2 = s1.cpu(), s2.cpu()
    mean = s1 / n_fields
    var = (s2 / n_fields - mean ** 2).clamp_min(0)
    return mean, (var / n_fields).sqrt(), el


def cv_coefficient(C: torch.Tensor, g: torch.Tensor) -> torch.Tensor:
    """c(tau) = Cov(C, g) / Var(g) from calibration pairs (fixed before the
    estimator uses other samples, so it adds no bias)."""
    Cc, gc = C - C.mean(0), g - g.mean(0)
    return (Cc * gc).mean(0) / (gc * gc).mean(0).clamp_min(1e-300)


def estimators(C: torch.Tensor, g: torch.Tensor, c: torch.Tensor, g_mean: torch.Tensor, g_mean_err: torch.Tensor):
    """Plain and control-variate estimates of <C(tau)> with standard errors."""
    n = C.shape[0]
    plain = C.mean(0)
    plain_err = C.std(0) / math.sqrt(n)
    r = C - c * g
    cv = r.mean(0) + c * g_mean
    cv_err = ((r.std(0) / math.sqrt(n)) ** 2 + (c * g_mean_err) ** 2).sqrt()
    return plain, plain_err, cv, cv_err

"""Times the hot kernels of libnrcps_b200 in isolation (CUDA events on the
context's stream, after warm-up), one JSON line per measurement.

    python -m nrcps_b200.kernel_bench step    --L 32 --orbitals 19456 [--kind K --cluster C] [--precision f32]
    python -m nrcps_b200.kernel_bench overlap --L 32 --ns 19 --nconf 1024 [--tc 1|0]
    python -m nrcps_b200.kernel_bench dets    --N 19 --nconf 4096
    python -m nrcps_b200.kernel_bench cv      --T 64 --batch 256
    python -m nrcps_b200.kernel_bench qr      --L 32 --N 19 --nconf 1024 [--precision f32] [--gram-tc 1|0]
    python -m nrcps_b200.kernel_bench rng     --L 32 --T 64 --nconf 1024
    python -m nrcps_b200.kernel_bench pair    --L 48 --N 10 --nconf 1024 [--precision f32] [--pair-tile 0]

step:    one transfer-matrix step (nrcps_propagate, Z2 field, a = 0.5) over
         `orbitals` orbitals in batches of 19; GB/s counts one read and one
         write of every orbital.
overlap: S = <src|psi> for FP32 orbitals with dense FP64 sources
         (nrcps_overlap); GB/s counts one read of psi, TFLOP/s the useful
         8 ns nt V complex multiply-adds per configuration.
dets:    determinants of all N leading minors of nconf FP64 matrices.
cv:      one training step (forward, backward, Adam) and one inference pass
         of the control-variate network on random inputs; TFLOP/s counts the
         conv multiply-adds (2 flops each; backward twice the forward).
qr:      one CholeskyQR re-orthonormalisation (nrcps_reorthonormalise) of
         nconf configurations of N orbitals; GB/s counts the algorithmic
         three passes over the orbitals (Gram read, apply read + write).
rng:     the Z2 field bits of nconf configurations x T slices of L^3 sites
         from RANLXS2 (nrcps_draw_z2_bits): uniforms per second and the
         output bits' GB/s.
pair:    the TwoBody pair matrices phi_st = sum_p w(p) psi_s(p) psi_t(-p) of
         nconf configurations of N orbitals (nrcps_pair_matrix); GB/s counts
         one read of the orbitals.
"""
from __future__ import annotations

import argparse
import ctypes
import json

import numpy as np
import torch

from . import _capi as C
from ._capi import lib
from .api import Context, draw_z2_bits, kinetic_table, overlap, reorthonormalise, slater_dets


def _time(fn, reps: int, warmup: int = 2) -> float:
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def bench_step(ctx: Context, L: int, orbitals: int, precision: str, kind: int, cluster: int, reps: int,
               field: str = "z2") -> dict:
    dims = (L, L, L)
    batch = 19
    nconf = max(1, orbitals // batch)
    psi = torch.randn((nconf * batch,) + dims, dtype=torch.complex64 if precision == "f32" else torch.complex128,
                      device=ctx.device)
    kinv = torch.from_numpy(1.0 / kinetic_table(dims, "PERFECT", 1.0, 0.5, 2.0)).to(ctx.device)
    pf = C.PositionFactor()
    if field in ("gauss", "wtab"):  # Gaussian phi, a = 0.3: the general position-factor path
        from .api import draw_fields
        fld, _ = draw_fields("RANLXS2", 7, "GAUSS", L ** 3, nconf, 0, ctx)
        pf.field_mode, pf.dev_field, pf.bit0, pf.conf_stride = 2, fld.data_ptr(), 0, L ** 3
        pf.a, pf.dev_pos = 0.3, None
        if field == "wtab":  # the same field as one FP32 weight (1 + a phi)/V per site
            fld = ((1.0 + 0.3 * fld.reshape(-1, 2)[:, 0]) / L ** 3).to(torch.float32).contiguous()
            pf.field_mode, pf.dev_field = 3, fld.data_ptr()
    else:
        fld = draw_z2_bits("RANLXS2", 7, 0, nconf * L ** 3, ctx)
        pf.field_mode, pf.dev_field, pf.bit0, pf.conf_stride = 1, fld.data_ptr(), 0, L ** 3
        pf.a, pf.dev_pos = 0.5, None
    d3 = np.array(dims, dtype=np.int32)
    ctx.set_option("fused.kind", kind)
    ctx.set_option("fused.cluster", cluster)

    def run():
        ctx.check(lib().nrcps_propagate(ctx.handle, ctypes.c_void_p(psi.data_ptr()), batch, nconf,
                                        d3.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                        ctypes.c_void_p(kinv.data_ptr()), ctypes.byref(pf),
                                        C.F32 if precision == "f32" else C.F64), "propagate")

    try:
        ms = _time(run, reps)
        ctx.synchronize()
    finally:
        ctx.set_option("fused.kind", -1)
        ctx.set_option("fused.cluster", 0)
    esize = 8 if precision == "f32" else 16
    return {"kernel": "step", "field": field, "L": L, "orbitals": nconf * batch, "precision": precision, "kind": kind,
            "cluster": cluster, "ms": round(ms, 4), "GBps": round(2.0 * L ** 3 * esize * nconf * batch / ms / 1e6, 1)}


def bench_overlap(ctx: Context, L: int, ns: int, nconf: int, tc: int, reps: int) -> dict:
    V = L ** 3
    g = torch.Generator(device=ctx.device).manual_seed(1)
    src = torch.randn((ns, V), dtype=torch.complex128, device=ctx.device, generator=g) / V ** 0.5
    psi = torch.randn((nconf, ns, V), dtype=torch.complex64, device=ctx.device, generator=g)
    ctx.set_option("overlap.tc", tc)
    try:
        ms = _time(lambda: overlap(src, psi, ctx), reps)
        ctx.synchronize()
    finally:
        ctx.set_option("overlap.tc", 1)
    return {"kernel": "overlap", "L": L, "ns": ns, "nconf": nconf, "tc": tc, "ms": round(ms, 4),
            "GBps": round(psi.numel() * 8 / ms / 1e6, 1),
            "useful_TFLOPs": round(8.0 * ns * ns * V * nconf / ms / 1e9, 2)}


def bench_dets(ctx: Context, N: int, nconf: int, reps: int) -> dict:
    g = torch.Generator(device=ctx.device).manual_seed(2)
    S = torch.randn((nconf, N, N), dtype=torch.complex128, device=ctx.device, generator=g)
    ms = _time(lambda: slater_dets(S, ctx=ctx), reps)
    ctx.synchronize()
    return {"kernel": "dets", "N": N, "nconf": nconf, "ms": round(ms, 4),
            "matrices_per_s": round(nconf / ms * 1e3, 1)}


def bench_cv(ctx: Context, T: int, batch: int, reps: int) -> dict:
    from .cv import ControlVariateNet, NetShape
    s = NetShape(T=T, G=8)
    net = ControlVariateNet(s, seed=0, ctx=ctx)
    g = torch.Generator(device=ctx.device).manual_seed(3)
    x = (torch.rand((batch, T, s.GS), device=ctx.device, generator=g) * 2 - 1).to(torch.bfloat16)
    y = torch.randn((batch, T), device=ctx.device, generator=g)

    def train():
        net.forward(x)
        net.backward(x, y)
        net.adam()

    ms_train = _time(train, reps)
    ms_fwd = _time(lambda: net.forward(x), reps)
    ms_tc = _time(lambda: net.infer(x), reps)
    # feature extraction at L = 32: Z2 bits of `batch` configurations, then block means
    from .api import draw_z2_bits
    from .cv import coarse_fields
    L = 32
    nbits = batch * T * L ** 3
    bits = draw_z2_bits("RANLXS2", 1, 0, nbits, ctx)
    ms_draw = _time(lambda: draw_z2_bits("RANLXS2", 1, 0, nbits, ctx), reps)
    ms_coarse = _time(lambda: coarse_fields(bits, 0, L, T, s.G, batch, ctx), reps)
    ctx.synchronize()
    macs = batch * s.GS * s.C * 27 * (T + 2 * s.C)  # three conv layers
    return {"kernel": "cv", "T": T, "batch": batch, "train_step_ms": round(ms_train, 4),
            "forward_ms": round(ms_fwd, 4), "forward_TFLOPs": round(2 * macs / ms_fwd / 1e9, 2),
            "infer_tc_ms": round(ms_tc, 4), "infer_tc_TFLOPs": round(2 * macs / ms_tc / 1e9, 2),
            "train_TFLOPs": round(6 * macs / ms_train / 1e9, 2), "z2_draw_ms": round(ms_draw, 4),
            "coarse_ms": round(ms_coarse, 4), "coarse_GBs": round(nbits / 8 / ms_coarse / 1e6, 1)}


def bench_qr(ctx: Context, L: int, N: int, nconf: int, precision: str, reps: int) -> dict:
    dt = torch.complex64 if precision == "f32" else torch.complex128
    g = torch.Generator(device=ctx.device).manual_seed(11)
    psi = torch.randn((nconf, N, L ** 3), dtype=dt, device=ctx.device, generator=g)
    logR = torch.zeros((nconf, N), dtype=torch.float64, device=ctx.device)
    ms = _time(lambda: reorthonormalise(psi, logR, ctx), reps)
    nbytes = 3 * psi.numel() * psi.element_size()
    return {"kernel": "qr", "L": L, "N": N, "nconf": nconf, "precision": precision, "ms": round(ms, 4),
            "GBps": round(nbytes / ms / 1e6, 1)}


def bench_rng(ctx: Context, L: int, T: int, nconf: int, reps: int) -> dict:
    count = nconf * T * L ** 3
    ms = _time(lambda: draw_z2_bits("RANLXS2", 7, 0, count, ctx), reps)
    ctx.synchronize()
    return {"kernel": "rng", "generator": "RANLXS2", "L": L, "T": T, "nconf": nconf, "uniforms": count,
            "ms": round(ms, 4), "uniforms_per_s": round(count / ms * 1e3, 1),
            "out_GBps": round(count / 8 / ms / 1e6, 1)}


def bench_pair(ctx: Context, L: int, N: int, nconf: int, precision: str, reps: int) -> dict:
    from .api import TwoBody
    dims = (L, L, L)
    dt = torch.complex64 if precision == "f32" else torch.complex128
    g = torch.Generator(device=ctx.device).manual_seed(13)
    psi = torch.randn((nconf, N, L ** 3), dtype=dt, device=ctx.device, generator=g)
    tb = TwoBody(dims, "TGND", "STANDARD", 1.0, 0.176776695, 2.0, ctx)
    ms = _time(lambda: tb.run_matrix(psi, psi), reps)
    ctx.synchronize()
    return {"kernel": "pair", "L": L, "N": N, "nconf": nconf, "precision": precision, "ms": round(ms, 4),
            "GBps": round(psi.numel() * psi.element_size() / ms / 1e6, 1)}


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("what", choices=["step", "overlap", "dets", "cv", "qr", "rng", "pair"])
    ap.add_argument("--gram-tc", type=int, default=0)
    ap.add_argument("--pair-tile", type=int, default=1)
    ap.add_argument("--field", default="z2", choices=["z2", "gauss", "wtab"],
                    help="step: Z2 bits, Gaussian phi, or the Gaussian field as FP32 weights per site")
    ap.add_argument("--L", type=int, default=32)
    ap.add_argument("--orbitals", type=int, default=19456)
    ap.add_argument("--precision", default="f32", choices=["f32", "f64"])
    ap.add_argument("--kind", type=int, default=-1)
    ap.add_argument("--cluster", type=int, default=0)
    ap.add_argument("--ns", type=int, default=19)
    ap.add_argument("--nconf", type=int, default=1024)
    ap.add_argument("--tc", type=int, default=1)
    ap.add_argument("--N", type=int, default=19)
    ap.add_argument("--reps", type=int, default=5)
    ap.add_argument("--T", type=int, default=64)
    ap.add_argument("--batch", type=int, default=256)
    a = ap.parse_args(argv)
    ctx = Context(0)
    if a.what == "step":
        r = bench_step(ctx, a.L, a.orbitals, a.precision, a.kind, a.cluster, a.reps, a.field)
    elif a.what == "overlap":
        r = bench_overlap(ctx, a.L, a.ns, a.nconf, a.tc, a.reps)
    elif a.what == "cv":
        r = bench_cv(ctx, a.T, a.batch, a.reps)
    elif a.what == "qr":
        ctx.set_option("qr.gram_tc", a.gram_tc)
        r = bench_qr(ctx, a.L, a.N, a.nconf, a.precision, a.reps)
        r["gram_tc"] = a.gram_tc
    elif a.what == "rng":
        r = bench_rng(ctx, a.L, a.T, a.nconf, a.reps)
    elif a.what == "pair":
        ctx.set_option("pair.tile", a.pair_tile)
        r = bench_pair(ctx, a.L, a.N, a.nconf, a.precision, a.reps)
        r["pair_tile"] = a.pair_tile
    else:
        r = bench_dets(ctx, a.N, a.nconf, a.reps)
    print(json.dumps(r), flush=True)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())

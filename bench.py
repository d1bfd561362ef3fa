"""Benchmark: batched auxiliary-field transfer-matrix ensemble on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Workload (the batched precision form): L=32^3 periodic lattice, T=64 time
slices, N=19 plane-wave orbitals (E_F = 0.045, closed shells |n|^2 <= 2),
Z2 fields with a = 0.5 (C0 = 0.25/(4 pi)) drawn on the device from RANLXS2
seed 7 (+491*rank), 4096 configurations per step, complex FP32 propagation,
FP64 LU of every leading minor.  One step = one pass of the production loop
over the 4096 configurations: field draw, 64 x (measure all N minors + one
transfer-matrix step), and the reference's per-block sum of |det|^2 over
configurations (and over ranks, as Comms::GlobalSum does).

Metric: config*slices/s (whole job).  Inputs: none but seeds and the source
list, so the orbitals (20 GB) and fields (1 GB) are generated on the device
and exceed L2 (126 MB) every step.

The default line also carries, as extra keys, the other workloads measured
in the same process (rank 0): the trapped few-body workload at its full shape
(L=48, T=128, SHO N=10, [K,V,I,V,K], pair sink, 1024 configurations), the
uneven batch (512 jobs of random L, N, T in one graph launch), the learned
control variate at a reduced training set (stated in its key), and the FP64
mode of the default workload batched the same way.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

METRIC = "L=32³ N=19+19 config·slices/s vs plain FP64; stat. error per GPU-second"
UNIT = "config·slices/s"
REF_BIN = os.path.join(REPO, "oracle", "_ref", "nrcps_ref")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--L", type=int, default=32)
    ap.add_argument("--T", type=int, default=64)
    ap.add_argument("--ef", type=float, default=0.045)
    ap.add_argument("--configs", type=int, default=4096)
    ap.add_argument("--precision", default="f32", choices=["f32", "f64"])
    ap.add_argument("--seed", type=int, default=7)
    ap.add_argument("--cpu-sample-slices", type=int, default=32, help="slices per host process for cpu_baseline")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cluster", type=int, default=0, help="force the fused kernel's cluster size (0: autotuned)")
    ap.add_argument("--no-fused", action="store_true", help="pencil passes instead of the fused kernel")
    ap.add_argument("--split", type=int, default=-1, help="fused kernel lane split: -1 autotuned, 0, 1")
    ap.add_argument("--kind", type=int, default=-1, help="fused kernel kind: -1 autotuned, 0 peer access, 1 split, 2 bulk staged, 3 bulk L2, 4-6 packed 0/2/3, 7/8 peer access L2, 9/10 kinds 6/3 with k(p) in shared memory, 11/12 kinds 7/8 with st.async write-backs")
    ap.add_argument("--no-plain", action="store_true", help="skip the plain FP64 GPU path measurement")
    ap.add_argument("--qr", type=int, default=-1, help="re-orthonormalise every k slices (-1: 8 for f32, 0 for f64)")
    ap.add_argument("--workload", default="batched", choices=["batched", "uneven", "cv", "trapped"],
                    help="batched: the L=32 ensemble (default); uneven: 512 jobs of random (L, N, T) in one launch; "
                         "cv: the learned control variate against the plain estimator; trapped: L=48 T=128 SHO "
                         "N=10 in a harmonic trap with the pair sink")
    ap.add_argument("--no-extras", action="store_true",
                    help="default workload only: skip the trapped, uneven, control-variate and batched-FP64 keys")
    ap.add_argument("--trapped-configs", type=int, default=1024, help="configurations of the trapped workload")
    ap.add_argument("--extras-cv-train", type=int, default=8192,
                    help="training pairs of the control-variate key of the default line")
    ap.add_argument("--cv-train", type=int, default=65536, help="cv: training pairs (seeds 1000.. in blocks of 1024)")
    ap.add_argument("--cv-eval", type=int, default=8192, help="cv: evaluation configurations")
    ap.add_argument("--cv-extra", type=int, default=1 << 20, help="cv: extra field draws for <g>")
    ap.add_argument("--cv-epochs", type=int, default=6)
    ap.add_argument("--jobs", type=int, default=512, help="jobs of the uneven workload")
    ap.add_argument("--real-weights", type=int, default=1, choices=[0, 1],
                    help="uneven, FP32: 1 steps on one FP32 weight per site made once per run, 0 forms "
                         "(1 + a phi)/V from phi per site and orbital")
    ap.add_argument("--uneven-groups", action="store_true",
                    help="uneven: also time every (L, N) group alone and the field draw alone")
    ap.add_argument("--precision-configs", type=int, default=64,
                    help="configurations of the FP32-vs-FP64 precision report (0: skip)")
    return ap.parse_args()


def qr_period(a):
    # FP32 orbitals are re-orthonormalised every 8 slices, as the batched L=32
    # workload prescribes (--qr changes it: at L=32, T=64, N=19 the FP32-vs-FP64
    # error of C_n(tau) is 1.2e-6 every 8, 1.9e-6 every 16, 1.5e-6 every 32 and
    # 1.7e-6 never)
    return a.qr if a.qr >= 0 else (8 if a.precision == "f32" else 0)


def workload(a, n_orb):
    return {"workload": f"batched ensemble L={a.L}^3 T={a.T} N={n_orb} Z2 a=0.5 RANLXS2 seed {a.seed}, "
                        f"{a.configs} configs/step, {a.precision} propagation + FP64 LU, QR every {qr_period(a)}",
            "L": a.L, "T": a.T, "N": n_orb, "configs_per_step": a.configs, "field": "ZTWO", "rng": "RANLXS2",
            "seed": a.seed, "precision": a.precision, "qr_period": qr_period(a),
            "sources": "plane waves (Fermi sea E_F=%g)" % a.ef,
            "l2": "inputs larger than L2 (orbitals %.1f GB)" % (a.configs * n_orb * a.L ** 3 * (8 if a.precision == "f32" else 16) / 1e9)}


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, local: int):
        self.index = self.smi_id(local)
        self.samples = []
        self.proc = None
        self.thread = None

    @staticmethod
    def smi_id(local: int) -> str:
        """nvidia-smi's id of CUDA device `local`: its UUID (CUDA ordinals are
        renumbered under CUDA_VISIBLE_DEVICES, nvidia-smi's are not), else the
        CUDA_VISIBLE_DEVICES entry, else the ordinal itself."""
        cands = []
        try:
            import torch
            u = str(torch.cuda.get_device_properties(local).uuid)
            cands.append(u if u.startswith("GPU-") else "GPU-" + u)
        except Exception:
            pass
        vis = [v.strip() for v in os.environ.get("CUDA_VISIBLE_DEVICES", "").split(",") if v.strip()]
        if local < len(vis):
            cands.append(vis[local])
        cands.append(str(local))
        for c in cands:
            try:
                r = subprocess.run(["nvidia-smi", "-i", c, "--query-gpu=index", "--format=csv,noheader"],
                                   capture_output=True, text=True, timeout=20)
                if r.returncode == 0 and r.stdout.strip():
                    return c
            except (OSError, subprocess.TimeoutExpired):
                break
        return str(local)

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.samples.append([x.strip() for x in line.split(",")])

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            if self.thread:
                self.thread.join(timeout=2)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(s[1]) for s in self.samples if len(s) > 8 and s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if len(s) > 8 and s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples if len(s) > 8 for i in range(4) if s[5 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples), "gpu": self.index}


# ------------------------------------------------------------ cpu baseline
def cpu_baseline(a, slices_per_proc: int, n_orb: int):
    """The reference's CPU path (oracle/_ref, built from its own sources) on
    every host core: one single-threaded process per core, seeds seed+491*r
    as the reference's MPI ranks (src/random/random.C:88)."""
    cores = os.cpu_count() or 1
    if os.path.exists(REF_BIN):
        procs = [subprocess.Popen([REF_BIN, "bench", f"L={a.L}", f"T={a.T}", f"ef={a.ef}", f"seed={a.seed + 491 * r}",
                                   "rng=RANLXS2", "field=ZTWO", f"max_slices={slices_per_proc}", "cutoff=2.0"],
                                  stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True) for r in range(cores)]
        rates = []
        for p in procs:
            out, _ = p.communicate()
            rates.append(json.loads(out.strip().splitlines()[-1])["config_slices_per_s"])
        return {"value": sum(rates), "unit": UNIT, "cores": cores, "kind": "reference",
                "sample": f"{slices_per_proc} slices of one L={a.L}^3 N={n_orb} configuration per process, "
                          f"{cores} processes (reference CPU FP64 path, FFTW replaced by the oracle's FFT)"}
    # fall back to the oracle port, single thread
    from oracle import oracle as O
    import numpy as np
    idx, _, _ = O.momenta((a.L,) * 3, "PERFECT", 1.0, a.ef, (2 * O.PI) ** 2)
    job = O.Job(L=a.L, T=min(a.T, 4), configs=1, seed=a.seed)
    t = time.perf_counter()
    O.run_ensemble(job, O.plane_wave_sources(job.dims, idx))
    el = time.perf_counter() - t
    return {"value": job.T / el, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": f"{job.T} slices of one configuration, oracle restatement, 1 thread"}


def run_reference(a):
    """--impl reference: the reference's own CPU implementation timed on the host."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    import numpy as np  # noqa: F401
    n_orb = 19
    samples = []
    for i in range(a.warmup + a.steps):
        t = time.perf_counter()
        cb = cpu_baseline(a, max(4, a.cpu_sample_slices // 4), n_orb)
        el = time.perf_counter() - t
        if i >= a.warmup:
            samples.append((cb, el))
    vals = [s[0]["value"] for s in samples]
    v = statistics.median(vals)
    cb = dict(samples[-1][0])
    cb["value"] = v
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": a.gpus, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": 1000 * statistics.median([s[1] for s in samples]),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload(a, n_orb), "cpu_baseline": cb,
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


# ------------------------------------------------------------- helpers
# DRAM bytes per orbital of the fused step from one ncu capture of the
# variant (dram__bytes_read.sum + dram__bytes_write.sum of one launch divided
# by the orbitals it processed), keyed (precision, L, kind, cluster): the
# line's roofline.traffic scales it to the timed launch.
NCU_TRAFFIC_PER_ORBITAL = {
    ("f32", 32, 7, 8): ((645.4e6 + 583.7e6) / 2432,
                        "ncu, kind 7 cluster 8, 2432 orbitals: 645.4 MB read + 583.7 MB written, scaled by orbitals "
                        "(profiles/fused_step_L32_f32.md)"),
    ("f32", 32, 11, 8): ((640.81e6 + 577.95e6) / 2432,
                         "ncu, kind 11 cluster 8, 2432 orbitals: 640.8 MB read + 577.9 MB written, scaled by orbitals "
                         "(profiles/fused_step_async_L32_f32.md)"),
    ("f32", 48, 11, 12): ((898.52e6 + 840.19e6) / 1007,
                          "ncu, kind 11 cluster 12, 1007 orbitals: 898.5 MB read + 840.2 MB written, scaled by "
                          "orbitals (profiles/fused_step_async_L48_f32_trapped.md)"),
}
# FP32-pipe figures of the same captures (FMA pipe and issue active, % of peak)
NCU_PIPES = {
    ("f32", 32, 7, 8): {"fma_pipe_pct": 41.1, "issue_active_pct": 49.0, "warps_per_sm": 15.4,
                        "source": "profiles/fused_step_L32_f32.md"},
    ("f32", 32, 11, 8): {"fma_pipe_pct": 41.7, "issue_active_pct": 51.3, "warps_per_sm": 15.0,
                         "source": "profiles/fused_step_async_L32_f32.md"},
    ("f32", 48, 11, 12): {"fma_pipe_pct": 36.8, "issue_active_pct": 43.3, "warps_per_sm": 11.3,
                          "source": "profiles/fused_step_async_L48_f32_trapped.md"},
}


def cuda_ms(fn, reps: int) -> float:
    """Milliseconds per call of fn() on the current stream (the library's):
    CUDA events around `reps` calls after one untimed call, synchronised on
    both sides."""
    import torch
    fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def measured_peaks():
    try:
        return json.load(open(os.path.join(REPO, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        return {}


def hbm_peak():
    p = measured_peaks()
    return (p["hbm_gbs"], "measured") if "hbm_gbs" in p else (6650.0, "fallback")


def fp32_peak_tflops(sm_count: int, sm_mhz) -> float:
    """FP32 CUDA-core peak: 128 FMA lanes per SM, 2 flops each, at the SM
    clock sampled during the run (the nominal 1965 MHz if none)."""
    return sm_count * 128 * 2 * (sm_mhz or 1965.0) * 1e6 / 1e12


def fft_flops_per_orbital_step(L: int) -> float:
    """The conventional count of one transfer-matrix step of one orbital: a
    forward and a backward complex 3-D FFT at 5 V log2 V real flops each
    (the pointwise factors are not counted)."""
    import math
    V = L ** 3
    return 2 * 5 * V * math.log2(V)


def ctx_sm_count(ctx) -> int:
    import torch
    return torch.cuda.get_device_properties(ctx.device).multi_processor_count


# ------------------------------------------------------- trapped workload
TRAPPED = dict(L=48, T=128, N=10, seed=31, kappa=0.005, lam=4.0, a=0.5)
SHO_JSON = os.path.join(REPO, "tests", "golden", "sho_coefficients.json")


def trapped_job(nb, precision: str, n_conf: int, qr_period: int = 8):
    """The trapped few-body workload (production/slater_det2_trapped/main-no_cum.C:90-128):
    [K, V, I, V, K] with a harmonic EXP trap kappa = 0.005 (Potential(arg, 0.5)),
    Z2 fields a = 0.5 from RANLXS2 seed 31, SlaterDet2 on the TGND pair sink.
    The orbitals are re-orthonormalised every 8 slices (unstabilised, the 10
    trap orbitals align over 128 slices and the pair-matrix minors lose
    precision, FP64 included); the determinants are rescaled to the
    unstabilised ones."""
    return nb.EnsembleJob(L=TRAPPED["L"], T=TRAPPED["T"], n_conf=n_conf, seed=TRAPPED["seed"], precision=precision,
                          potential=True, kappa=TRAPPED["kappa"], pot_type="EXP", pot_dt=0.5, mode="slater2",
                          wavefunc="TGND", wf_disp="STANDARD", wf_lambda=0.176776695, cutoff=2.0,
                          qr_period=qr_period)


def trapped_sources(nb):
    """The 10 lowest 3-D oscillator states of production/slater_det2_trapped/sources/source.{0..9}
    (coefficients as committed in tests/golden), built by OneBody::Set's rule with lambda = 4."""
    import numpy as np
    sho = json.load(open(SHO_JSON))
    L, lam = TRAPPED["L"], TRAPPED["lam"]
    return np.stack([nb.sho_source((L,) * 3, (lam,) * 3, sho[str(n)]) for n in range(TRAPPED["N"])])


def trapped_cpu_baseline(slices_per_proc: int):
    """The reference's CPU path (oracle/_ref) at the trapped shape: one
    single-threaded process per host core, seeds 31 + 491 r."""
    import tempfile
    if not os.path.exists(REF_BIN):
        return None
    cores = os.cpu_count() or 1
    sho = json.load(open(SHO_JSON))
    with tempfile.TemporaryDirectory() as d:
        for n, lines in sho.items():
            with open(os.path.join(d, f"source.{n}"), "w") as f:
                for l in lines:
                    f.write(f"{l[0]} {l[1]} {l[2]} {l[3]!r} {l[4]!r}\n")
        lam = TRAPPED["lam"]
        procs = [subprocess.Popen([REF_BIN, "bench", f"L={TRAPPED['L']}", f"T={TRAPPED['T']}", "sources=sho",
                                   f"N={TRAPPED['N']}", f"sho_dir={d}", f"lambda1={lam}", f"lambda2={lam}",
                                   f"lambda3={lam}", "mode=slater2", "potential=1", f"kappa={TRAPPED['kappa']}",
                                   "ptype=EXP", "wavefunc=TGND", "tb_disp=STANDARD", "tb_lambda=0.176776695",
                                   f"seed={TRAPPED['seed'] + 491 * r}", "rng=RANLXS2", "field=ZTWO",
                                   "couplings=0.019894367886486918", "cutoff=2.0", f"max_slices={slices_per_proc}"],
                                  stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True) for r in range(cores)]
        rates = []
        for p in procs:
            out, _ = p.communicate()
            rates.append(json.loads(out.strip().splitlines()[-1])["config_slices_per_s"])
    return {"value": sum(rates), "unit": UNIT, "cores": cores, "kind": "reference",
            "sample": f"{slices_per_proc} slices of one trapped L=48^3 configuration per process, {cores} processes "
                      f"(reference CPU FP64 path, FFTW replaced by the oracle's FFT)"}


def trapped_core(ctx, n_conf: int, steps: int, warmup: int, cpu_slices: int, precision_configs: int = 64,
                 sm_mhz=None):
    """The trapped workload: throughput (device-timed and end to end), the
    step's kernels alone at the same size, FP32-vs-FP64 correlators, and the
    reference's CPU path at the same shape."""
    import ctypes

    import numpy as np
    import torch

    import nrcps_b200 as nb
    from nrcps_b200 import _capi as C
    L, T, N = TRAPPED["L"], TRAPPED["T"], TRAPPED["N"]
    dims, V = (L,) * 3, L ** 3
    dev = ctx.device
    src = trapped_sources(nb)
    ens = nb.Ensemble(trapped_job(nb, "f32", n_conf), sources=src, ctx=ctx)
    for i in range(warmup):
        ens.run(i * n_conf)
    conf0 = warmup * n_conf
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for i in range(steps):
        ens.run(conf0 + i * n_conf)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    value = n_conf * T / (ms / 1000.0)
    # end to end: every step sends the sources from pinned host memory (the
    # propagator's Set of OneBody::Get) and reads the raw determinants back
    src_host = torch.from_numpy(np.ascontiguousarray(src)).pin_memory()
    dets_host = torch.empty(ens.dets.shape, dtype=ens.dets.dtype).pin_memory()
    conf0 += steps * n_conf
    torch.cuda.synchronize()
    e0.record()
    for i in range(steps):
        ens.set_sources(src_host)
        d = ens.run(conf0 + i * n_conf)
        dets_host.copy_(d, non_blocking=True)
    e1.record()
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1) / steps
    kind, cluster = ctx.fused_choice("f32", L)
    launches = ens.launches()
    ens.close()
    # the step's kernels alone on the same orbitals (FP32, n_conf x N)
    psi = torch.randn((n_conf * N,) + dims, dtype=torch.complex64, device=dev)
    bits = nb.draw_z2_bits("RANLXS2", TRAPPED["seed"], 0, n_conf * V, ctx)
    kinv = torch.from_numpy(1.0 / nb.kinetic_table(dims, "PERFECT", 1.0, 0.5, 2.0)).to(dev)
    pot = nb.potential_table(dims, TRAPPED["kappa"], 0.5, "EXP")
    posf = torch.from_numpy((V * pot) ** 2).to(dev)  # [K,V,I,V,K] = K B diag(V^2 v^2 w) F K
    pf = C.PositionFactor()
    pf.field_mode, pf.dev_field, pf.bit0, pf.conf_stride = 1, bits.data_ptr(), 0, V
    pf.a, pf.dev_pos = TRAPPED["a"], posf.data_ptr()
    d3 = np.array(dims, dtype=np.int32)

    def prop():
        ctx.check(nb.lib().nrcps_propagate(ctx.handle, ctypes.c_void_p(psi.data_ptr()), N, n_conf,
                                           d3.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                           ctypes.c_void_p(kinv.data_ptr()), ctypes.byref(pf), C.F32), "propagate")

    kms = cuda_ms(prop, 3)
    peak, peak_src = hbm_peak()
    step_bytes = 2.0 * V * 8 * n_conf * N
    step_gbs = step_bytes / (kms / 1000.0) / 1e9
    src_d = torch.from_numpy(src).to(dev)
    orbs = psi.view(n_conf, N, V)
    oms = cuda_ms(lambda: nb.overlap(src_d, orbs, ctx), 3)
    tb = nb.TwoBody(dims, "TGND", "STANDARD", 1.0, 0.176776695, 2.0, ctx)
    pms = cuda_ms(lambda: tb.run_matrix(orbs, orbs), 3)
    read_bytes = V * 8.0 * n_conf * N  # one read of every orbital
    overlap_flops = 8.0 * N * N * V * n_conf  # complex MACs of S = src^H psi, one precision pass
    del psi, orbs, bits
    torch.cuda.empty_cache()
    # FP32 propagation against the FP64 mode on the same fields
    prec = {}
    if precision_configs > 0:
        for p in ("f32", "f64"):
            e = nb.Ensemble(trapped_job(nb, p, precision_configs), sources=src, ctx=ctx)
            prec[p] = e.run(0).mean(0).cpu().numpy()
            e.close()
        rel = np.max(np.abs(prec["f32"] - prec["f64"]) / np.abs(prec["f64"]), axis=1)
    fp32_tflops = fft_flops_per_orbital_step(L) * n_conf * N / (kms / 1000) / 1e12
    fp32_peak = fp32_peak_tflops(ctx_sm_count(ctx), sm_mhz)
    traffic = NCU_TRAFFIC_PER_ORBITAL.get(("f32", L, kind, cluster))
    out = {"metric": "trapped config·slices/s", "value": value, "unit": UNIT, "ms_per_step": ms, "steps": steps,
           "warmup": warmup, "dtype": "f32",
           "config": {"workload": f"trapped few-body L={L}^3 T={T}, SHO N={N}+{N} (lambda 4), [K,V,I,V,K] harmonic "
                                  f"EXP trap kappa={TRAPPED['kappa']}, Z2 a=0.5 RANLXS2 seed {TRAPPED['seed']}, "
                                  f"SlaterDet2 on the TGND pair sink, {n_conf} configs/step, FP32 propagation, "
                                  f"TF32-split tensor-core overlap, FP64 LU, QR every 8",
                      "configs_per_step": n_conf, "l2": "orbitals %.1f GB (larger than L2)" % (n_conf * N * V * 8 / 1e9)},
           "e2e": {"value": n_conf * T / (e2e_ms / 1000.0), "unit": UNIT,
                   "h2d_bytes_per_step": src_host.numel() * 16, "d2h_bytes_per_step": dets_host.numel() * 16},
           "gpu_launches_per_step": launches + 1,
           "roofline": {"bound": "hbm", "achieved": round(step_gbs, 1), "peak": peak, "unit": "GB/s",
                        "frac": round(step_gbs / peak, 4),
                        "traffic": round(traffic[0] * n_conf * N) if traffic else None,
                        "traffic_source": traffic[1] if traffic else "no ncu capture of this variant",
                        "peak_source": peak_src,
                        "kernel": "fused transfer-matrix step with the trap folded in (kind %d, cluster %d), "
                                  "%d configs x %d orbitals, %.3f ms/launch" % (kind, cluster, n_conf, N, kms),
                        "fp32": {"convention": "10 V log2 V flops per orbital-step",
                                 "achieved_tflops": round(fp32_tflops, 2), "peak_tflops": round(fp32_peak, 1),
                                 "frac": round(fp32_tflops / fp32_peak, 4)}},
           "overlap": {"kernel": "tcgen05 TF32 hi/lo overlap S = src^H psi (incl. the source split)",
                       "ms": round(oms, 3), "achieved_gbs": round(read_bytes / (oms / 1000) / 1e9, 1),
                       "frac_hbm": round(read_bytes / (oms / 1000) / 1e9 / peak, 4),
                       "useful_tflops": round(overlap_flops / (oms / 1000) / 1e12, 2)},
           "pair_matrix": {"kernel": "TwoBody pair matrix sum_p w(p) psi_s(p) psi_t(-p)", "ms": round(pms, 3),
                           "achieved_gbs": round(read_bytes / (pms / 1000) / 1e9, 1),
                           "frac_hbm": round(read_bytes / (pms / 1000) / 1e9 / peak, 4)}}
    if prec:
        out["precision_report"] = {"configs": precision_configs,
                                   "compare": "FP32 vs FP64 mode (both QR every 8), C_m(tau) = <det S2_m(tau)>",
                                   "max_rel_err_C": float(rel.max()),
                                   "rel_err_C_per_tau": [float("%.2e" % v) for v in rel[::8]],
                                   "per_tau_stride": 8, "target": 1e-5}
    if cpu_slices > 0:
        out["cpu_baseline"] = trapped_cpu_baseline(cpu_slices)
    return out


# ------------------------------------------------------- plain FP64 GPU path
def plain_fp64_gpu(a, ctx, idx, configs: int = 2, slices: int = 8):
    """The reference's GPU call structure through the class API, in FP64:
    one configuration at a time, Propagator::Run over [K, I, K] as separate
    Kinetic / Interaction (FFT, multiply, FFT) launches, fields drawn per
    slice by Lattice::Refresh, the Slater matrix by one overlap per slice and
    the determinants of all leading minors -- the 'plain FP64 GPU path' the
    batched FP32 path is compared with."""
    import torch
    import nrcps_b200 as nb

    dims = (a.L,) * 3
    vol = a.L ** 3
    n = len(idx)
    rng = nb.Random("RANLXS2", a.seed)
    lat = nb.Lattice(dims, rng, "ZTWO", ctx)
    inter = nb.Interaction(lat, 1.0, [0.019894367886486918], 1.0, 2.0)
    kin = nb.Kinetic(dims, "PERFECT", 1.0, 0.5, 2.0, ctx)
    prop = nb.Propagator(n, dims, "f64", ctx)
    src = torch.zeros((n, vol), dtype=torch.complex128, device=ctx.device)
    src[torch.arange(n), torch.as_tensor(idx, dtype=torch.long)] = 1
    ham = [kin, inter, kin]

    def one_config():
        prop.get().b.copy_(src.reshape(prop.get().b.shape))
        for _ in range(slices):
            S = nb.overlap(src, prop.get().b.reshape(1, n, vol), ctx)
            nb.slater_dets(S, ctx=ctx)
            for h in ham:
                h.initialize()
            prop.run(ham)
            lat.refresh()

    one_config()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(configs):
        one_config()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    return {"value": configs * slices / (ms / 1000.0), "unit": UNIT,
            "sample": f"{configs} configurations x {slices} slices, L={a.L}^3 N={n}, FP64, class-API call structure"}


def fp64_batched(a, ctx, idx, configs: int = 256):
    """The default workload in the library's FP64 mode, batched and
    graph-captured like the FP32 line (no re-orthonormalisation): separates
    the gain from batching from the gain from FP32."""
    import nrcps_b200 as nb
    job = nb.EnsembleJob(L=a.L, T=a.T, n_conf=configs, seed=a.seed, precision="f64", fermi_energy=a.ef,
                         qr_period=0)
    ens = nb.Ensemble(job, plane_wave_index=idx, ctx=ctx)
    ens.run(0)
    k = [0]

    def run():
        k[0] += 1
        ens.run(k[0] * configs)

    ms = cuda_ms(run, 2)
    kind, cluster = ctx.fused_choice("f64", a.L)
    ens.close()
    return {"value": configs * a.T / (ms / 1000.0), "unit": UNIT, "ms_per_step": ms,
            "sample": f"{configs} configurations x {a.T} slices per step, L={a.L}^3 N={len(idx)}, FP64 orbitals and "
                      f"determinants, fused step kind {kind} cluster {cluster}"}


# ------------------------------------------------- precision and statistics
def stat_error(a, ctx, dets, ms_per_step, world):
    """The second metric: statistical error of <C_N(tau)> = <|det S_N(tau)|^2>
    from one step's configurations (binned jackknife on the device), scaled to
    one GPU-second of this throughput (error ~ 1/sqrt(time))."""
    import torch
    import nrcps_b200 as nb
    x = (dets[:, :, -1].abs() ** 2).to(torch.float64).contiguous()  # [n_conf, T]
    mean, err, em, ee = nb.jackknife(x, 32, True, ctx)
    mean, err, em, ee = (t.cpu().numpy() for t in (mean, err, em, ee))
    t_mid = a.T // 2
    rel = float(err[t_mid] / abs(mean[t_mid]))
    gpu_s = ms_per_step / 1000.0 / world
    return {"observable": f"C_N(tau) = <|det S_N(tau)|^2>, N={dets.shape[-1]}, tau={t_mid}",
            "estimator": "plain", "configs": int(dets.shape[0]), "jackknife_bins": 32,
            "rel_err": rel, "gpu_seconds": gpu_s, "rel_err_per_gpu_second": rel * gpu_s ** 0.5,
            "E_eff_tau_mid": float(em[t_mid]), "E_eff_err_tau_mid": float(ee[t_mid])}


def precision_report(a, ctx, idx):
    """FP32 propagation (QR as the bench runs it) against the FP64 mode on the
    same fields and configurations: per-slice relative error of
    C_n(tau) = <|det S_n(tau)|^2> (max over n) and of the effective energy
    E(tau) = log(C_N(tau)/C_N(tau+1)).  The FP64 mode is the one the parity
    tests hold to 1e-12 of the oracle."""
    import numpy as np
    import nrcps_b200 as nb
    n = a.precision_configs
    out = {}
    for prec, qr in (("f32", qr_period(a) if a.precision == "f32" else 8), ("f64", 0)):
        job = nb.EnsembleJob(L=a.L, T=a.T, n_conf=n, seed=a.seed, precision=prec, fermi_energy=a.ef, qr_period=qr)
        ens = nb.Ensemble(job, plane_wave_index=idx, ctx=ctx)
        d = ens.run(0).cpu().numpy()
        ens.close()
        out[prec] = (np.abs(d) ** 2).mean(0)  # [T, N]
    c32, c64 = out["f32"], out["f64"]
    rel_tau = np.max(np.abs(c32 - c64) / np.abs(c64), axis=1)
    e32 = np.log(c32[:-1, -1] / c32[1:, -1])
    e64 = np.log(c64[:-1, -1] / c64[1:, -1])
    e_rel = np.abs(e32 - e64) / np.maximum(np.abs(e64), 1e-300)
    return {"configs": n, "compare": "FP32 propagation (QR every %d) vs FP64 mode" % (qr_period(a) or 8),
            "max_rel_err_C": float(rel_tau.max()), "rel_err_C_per_tau": [float("%.3e" % v) for v in rel_tau],
            "max_rel_err_E_eff": float(e_rel.max()), "target": 1e-5}


# -------------------------------------------------------------------- b200
def run_b200(a):
    import ctypes

    import numpy as np
    import torch
    import torch.distributed as dist

    import nrcps_b200 as nb
    from nrcps_b200 import _capi as C
    from nrcps_b200 import parallel

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    dev = torch.device("cuda", local)
    ctx = nb.Context(local)
    if a.no_fused:
        ctx.set_option("propagate.fused", 0)
    if a.cluster:
        ctx.set_option("fused.cluster", a.cluster)
    if a.split >= 0:
        ctx.set_option("fused.split", a.split)
    if a.kind >= 0:
        ctx.set_option("fused.kind", a.kind)

    dims = (a.L,) * 3
    idx, _, _ = nb.momenta(dims, "PERFECT", 1.0, a.ef, 2.0)
    n_orb = len(idx)
    # each rank runs its own stream, seeded seed + 491 * rank (src/random/random.C:88)
    job = nb.EnsembleJob(L=a.L, T=a.T, n_conf=a.configs, seed=a.seed, rank=rank, precision=a.precision,
                         fermi_energy=a.ef, qr_period=qr_period(a))
    ens = nb.Ensemble(job, plane_wave_index=idx, ctx=ctx)
    corr = torch.zeros((a.T, n_orb), dtype=torch.float64, device=dev)

    def step(i):
        dets = ens.run(i * a.configs)
        # production/slater_det/main.C:208-211 and :226: corr[n][t] += |det|^2, summed over ranks
        c = parallel.accumulate(dets, "slater")
        parallel.global_sum(c)
        corr.copy_(c.real.T)
        return dets

    def barrier():
        torch.cuda.synchronize(dev)
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize(dev)

    for i in range(a.warmup):
        last_dets = step(i)
    barrier()
    clocks = ClockSampler(local)
    clocks.start()
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    launches0 = ctx_launches = None
    start.record()
    for i in range(a.steps):
        last_dets = step(a.warmup + i)
    stop.record()
    barrier()
    clocks.stop()
    ms = start.elapsed_time(stop)
    t = torch.tensor([ms], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms = float(t.item())
    launches_per_step = ens.launches() + 1  # graph body + field draw
    value = world * a.configs * a.T * a.steps / (ms / 1000.0)

    # ---- roofline of the dominant kernel: the fused transfer-matrix step
    # (psi <- K B w F K psi), algorithmic bytes = one read + one write of every
    # orbital = 2 * V * sizeof(complex) per orbital.
    rconf = min(a.configs, 1024)
    esize = 8 if a.precision == "f32" else 16
    psi = torch.randn((rconf * n_orb,) + dims, dtype=torch.complex64 if a.precision == "f32" else torch.complex128,
                      device=dev)
    bits = nb.draw_z2_bits("RANLXS2", a.seed, 0, rconf * a.L ** 3, ctx)
    kinv = torch.from_numpy(1.0 / nb.kinetic_table(dims, "PERFECT", 1.0, 0.5, 2.0)).to(dev)
    pf = C.PositionFactor()
    pf.field_mode, pf.dev_field, pf.bit0, pf.conf_stride = 1, bits.data_ptr(), 0, a.L ** 3
    pf.a, pf.dev_pos = 0.5, None
    d3 = np.array(dims, dtype=np.int32)
    prec = C.F32 if a.precision == "f32" else C.F64

    def prop():
        ctx.check(nb.lib().nrcps_propagate(ctx.handle, ctypes.c_void_p(psi.data_ptr()), n_orb, rconf,
                                           d3.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                           ctypes.c_void_p(kinv.data_ptr()), ctypes.byref(pf), prec), "propagate")

    for _ in range(3):
        prop()
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    reps = 5
    e0.record()
    for _ in range(reps):
        prop()
    e1.record()
    torch.cuda.synchronize(dev)
    kms = e0.elapsed_time(e1) / reps
    alg_bytes = 2.0 * a.L ** 3 * esize * rconf * n_orb
    achieved = alg_bytes / (kms / 1000.0) / 1e9
    peak, peak_src = hbm_peak()
    kind, cluster = ctx.fused_choice(a.precision, a.L)
    traffic = NCU_TRAFFIC_PER_ORBITAL.get((a.precision, a.L, kind, cluster))
    roofline = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4),
                "traffic": round(traffic[0] * rconf * n_orb) if traffic else None,
                "traffic_source": traffic[1] if traffic else "no ncu capture of this variant",
                "kernel": "fused transfer-matrix step (nrcps_propagate), kind %d, cluster %d, %d configs x %d "
                          "orbitals, %.3f ms/launch" % (kind, cluster, rconf, n_orb, kms),
                "peak_source": peak_src}
    del psi, bits

    # ---- end to end through the public API with host buffers: every step
    # sends the source list from pinned host memory into the ensemble (which
    # starts every configuration from it, as Propagator::Set does) and reads
    # the raw determinants back into pinned memory.
    idx_host = torch.from_numpy(np.asarray(idx, dtype=np.int32)).pin_memory()
    dets_host = torch.empty(ens.dets.shape, dtype=ens.dets.dtype).pin_memory()
    barrier()
    e0.record()
    for i in range(a.steps):
        ens.set_sources(plane_wave_index=idx_host)
        dets = step(a.warmup + a.steps + i)
        dets_host.copy_(dets, non_blocking=True)
    e1.record()
    barrier()
    ems = e0.elapsed_time(e1)
    t = torch.tensor([ems], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    e2e = {"value": world * a.configs * a.T * a.steps / (float(t.item()) / 1000.0), "unit": UNIT,
           "h2d_bytes_per_step": idx_host.numel() * 4, "d2h_bytes_per_step": dets_host.numel() * 16}
    clk = clocks.summary()
    fp32_tflops = fft_flops_per_orbital_step(a.L) * rconf * n_orb / (kms / 1000) / 1e12
    fp32_peak = fp32_peak_tflops(ctx_sm_count(ctx), clk.get("sm_mhz"))
    roofline["fp32"] = {"convention": "10 V log2 V flops per orbital-step (two complex 3-D FFTs)",
                        "achieved_tflops": round(fp32_tflops, 2), "peak_tflops": round(fp32_peak, 1),
                        "frac": round(fp32_tflops / fp32_peak, 4)}
    ncu = NCU_PIPES.get((a.precision, a.L, kind, cluster))
    if ncu:
        roofline["fp32"]["ncu"] = ncu

    plain = plain_fp64_gpu(a, ctx, idx) if rank == 0 and not a.no_plain else None
    stat = stat_error(a, ctx, last_dets, ms / a.steps, world) if rank == 0 else None
    del last_dets
    prec_report = precision_report(a, ctx, idx) if rank == 0 and a.precision_configs > 0 else None
    ens.close()
    extras = {}
    if rank == 0 and not a.no_extras:
        torch.cuda.empty_cache()
        extras["fp64_batched"] = fp64_batched(a, ctx, idx)
        extras["trapped"] = trapped_core(ctx, a.trapped_configs, 2, 1, 0 if a.no_cpu_baseline else 4,
                                         sm_mhz=clk.get("sm_mhz"))
        extras["uneven"] = uneven_core(ctx, a.jobs, 2, 1)
        extras["control_variate"] = cv_core(ctx, a, a.extras_cv_train, a.cv_eval, a.cv_extra, a.cv_epochs)
        extras["control_variate"]["reduced"] = (f"{a.extras_cv_train} training pairs instead of the workload's "
                                                f"65536 (python bench.py --workload cv runs the full set)")

    if rank == 0:
        cb = None if a.no_cpu_baseline else cpu_baseline(a, a.cpu_sample_slices, n_orb)
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps,
                "warmup": a.warmup, "ms_per_step": ms / a.steps, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": a.precision, "data": "synthetic (device-drawn fields, plane-wave sources)",
                "config": workload(a, n_orb), "roofline": roofline, "cpu_baseline": cb, "e2e": e2e,
                "gpu_launches": launches_per_step * a.steps, "clocks": clk,
                "plain_fp64_gpu": plain, "precision_report": prec_report, "stat_error": stat,
                "speedup_vs_plain_fp64_gpu": (value / world / plain["value"]) if plain else None}
        if extras.get("fp64_batched"):
            line["speedup_vs_batched_fp64_gpu"] = value / world / extras["fp64_batched"]["value"]
        line.update(extras)
        print(json.dumps(line))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


# ------------------------------------------------------------ uneven batch
def uneven_jobs(n_jobs: int, seed: int = 99):
    """The uneven workload: per job L in {16, 24, 32, 48}, N in {7, 19, 33}
    (closed shells |n|^2 <= 1, 2, 4) and T in {32, 64, 128}, each drawn
    uniformly from `seed`; one configuration per job."""
    import numpy as np
    import nrcps_b200 as nb
    rs = np.random.default_rng(seed)
    shell = {7: 1.5, 19: 2.5, 33: 4.5}  # E_F between shells, in units of (2 pi / L)^2 / 2
    jobs = []
    for _ in range(n_jobs):
        L = int(rs.choice([16, 24, 32, 48]))
        N = int(rs.choice([7, 19, 33]))
        T = int(rs.choice([32, 64, 128]))
        ef = 0.5 * (2 * np.pi / L) ** 2 * shell[N]
        jobs.append(nb.BatchJob(L=L, T=T, n_conf=1, fermi_energy=ef))
    return jobs


def uneven_core(ctx, n_jobs: int, steps: int, warmup: int, precision: str = "f32"):
    """512 jobs of uneven (L, N, T), Gaussian fields a = 0.3, FP32 orbitals and
    FP64 determinants, every time loop in one graph launch per run."""
    import nrcps_b200 as nb
    jobs = uneven_jobs(n_jobs)
    b = nb.Batch(jobs, seed=99, field="GAUSS", a=0.3, precision=precision, ctx=ctx)
    slices = sum(j.T * j.n_conf for j in jobs)
    for _ in range(warmup):
        b.run()
    ms = cuda_ms(b.run, steps) if steps > 0 else 0.0
    shapes = sorted({(j.L, n, ) for j, n in zip(jobs, b.n_orb)})
    orb_steps = sum(j.T * j.n_conf * n for j, n in zip(jobs, b.n_orb))
    alg_bytes = sum(j.T * j.n_conf * n * 2 * 8 * j.L ** 3 for j, n in zip(jobs, b.n_orb))
    peak, peak_src = hbm_peak()
    out = {"metric": "uneven batch config·slices/s", "value": slices / (ms / 1000.0), "unit": UNIT,
           "ms_per_step": ms, "steps": steps, "warmup": warmup, "dtype": precision,
           "config": {"workload": f"{len(jobs)} jobs, L in 16/24/32/48, N in 7/19/33, T in 32/64/128 drawn from "
                                  f"seed 99, Gaussian phi a=0.3, one graph launch per step (fields drawn before it)",
                      "jobs": len(jobs), "config_slices_per_step": slices, "orbital_steps_per_step": orb_steps,
                      "groups": len(shapes)},
           "gpu_launches_in_graph": b.launches(),
           # the whole step (propagation, measurement, LU, field draw) against the
           # propagation's algorithmic bytes: a lower bound of its HBM fraction
           "step_hbm": {"algorithmic_bytes": alg_bytes, "achieved_gbs": round(alg_bytes / (ms / 1000) / 1e9, 1),
                        "peak": peak, "frac": round(alg_bytes / (ms / 1000) / 1e9 / peak, 4),
                        "peak_source": peak_src}}
    b.close()
    return out


def uneven_breakdown(ctx, n_jobs: int, precision: str = "f32"):
    """Where the uneven step goes: every (L, N) group run alone as its own
    batch (its own field draw included) and the whole step's Gaussian field
    draw alone; a sum of the groups close to the whole step means the groups'
    launches already fill the GPU one after another."""
    import nrcps_b200 as nb
    jobs = uneven_jobs(n_jobs)
    full = nb.Batch(jobs, seed=99, field="GAUSS", a=0.3, precision=precision, ctx=ctx)
    n_orb = full.n_orb
    full.run()
    full_ms = cuda_ms(full.run, 2)
    full.close()
    sites = sum(j.T * j.L ** 3 for j in jobs)
    draw_ms = cuda_ms(lambda: nb.draw_fields("RANLXS2", 99, "GAUSS", sites // 8, 8, 0, ctx), 1)
    groups = {}
    for j, n in zip(jobs, n_orb):
        groups.setdefault((j.L, n), []).append(j)
    out = {}
    for (L, N), js in sorted(groups.items()):
        b = nb.Batch(js, seed=99, field="GAUSS", a=0.3, precision=precision, ctx=ctx)
        b.run()
        ms = cuda_ms(b.run, 2)
        b.close()
        out[f"L{L}_N{N}"] = {"jobs": len(js), "config_slices": sum(j.T for j in js),
                             "orbital_steps": sum(j.T for j in js) * N, "ms_alone": round(ms, 2)}
    return {"whole_step_ms": round(full_ms, 1), "field_draw_ms": round(draw_ms, 1),
            "sum_of_groups_alone_ms": round(sum(v["ms_alone"] for v in out.values()), 1), "groups": out}


def run_uneven(a):
    import nrcps_b200 as nb
    if int(os.environ.get("RANK", "0")) != 0:
        return 0
    ctx = nb.Context(0)
    ctx.set_option("batch.real_weights", a.real_weights)
    line = uneven_core(ctx, a.jobs, a.steps, a.warmup, a.precision)
    line["config"]["field_weights"] = ("one FP32 weight per site, made once per run"
                                       if a.real_weights and a.precision == "f32" else "formed from phi per site")
    if a.uneven_groups:
        line["breakdown"] = uneven_breakdown(ctx, a.jobs, a.precision)
    line.update({"n_gpus": 1, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                 "data": "synthetic (device-drawn Gaussian fields)"})
    print(json.dumps(line))
    return 0


# ------------------------------------------------------- control variate
def cv_core(ctx, a, cv_train: int, cv_eval: int, cv_extra: int, cv_epochs: int):
    """The learned control variate at the batched shape (L=32, T=64, N=19,
    Z2 a=0.5): training pairs from seeds 1000.. (1024 configurations per
    seed), a calibration block for c(tau), an evaluation block from a fresh
    seed, <g> from extra field draws; statistical error of <C_N(tau)> per
    GPU-second for the plain and the control-variate estimators."""
    import math
    import time as _t
    import torch
    import nrcps_b200 as nb
    from nrcps_b200 import cv
    L, T, ef, G = a.L, a.T, a.ef, 8

    def timed(fn):
        torch.cuda.synchronize()
        t0 = _t.perf_counter()
        r = fn()
        torch.cuda.synchronize()
        return r, _t.perf_counter() - t0

    # training pairs: 1024 configurations per seed, seeds 1000, 1001, ...
    Xs, Cs, t_gen = [], [], 0.0
    for i in range(0, cv_train, 1024):
        (X, C), el = timed(lambda: cv.generate_pairs(L, T, ef, 1000 + i // 1024, min(1024, cv_train - i),
                                                     chunk=1024, G=G, precision=a.precision,
                                                     qr_period=qr_period(a), ctx=ctx))
        Xs.append(X)
        Cs.append(C)
        t_gen += el
    X, C = torch.cat(Xs), torch.cat(Cs)
    n_cal = max(1024, X.shape[0] // 8)
    net = cv.ControlVariateNet(cv.NetShape(T=T, G=G), seed=0, ctx=ctx)
    losses, t_train = timed(lambda: net.fit(X[:-n_cal], torch.log(C[:-n_cal]), epochs=cv_epochs, batch=256,
                                            lr=2e-3))
    c = cv.cv_coefficient(C[-n_cal:].cpu(), torch.exp(net.predict_logC(X[-n_cal:])))
    del X, Xs
    # evaluation block: a seed never used for training
    # (4096 configurations per ensemble run, as the batched workload; each
    # configuration's determinants do not depend on the chunking)
    (Xe, Ce), t_eval = timed(lambda: cv.generate_pairs(L, T, ef, 2000, cv_eval, chunk=4096, G=G,
                                                       precision=a.precision, qr_period=qr_period(a), ctx=ctx))
    ge, t_inf = timed(lambda: torch.exp(net.predict_logC(Xe)))
    gm, gm_err, t_extra = cv.extra_fields_mean_g(net, L, 3000, 0, cv_extra, chunk=32768, ctx=ctx)
    Ce = Ce.cpu()
    plain, plain_err, est, est_err = cv.estimators(Ce, ge, c, gm, gm_err)
    var_ratio = (Ce - c * ge).var(0) / Ce.var(0)
    t_plain = t_eval                           # propagation + measurement of the evaluation block
    t_cv = t_eval + t_inf + t_extra            # + inference on it + the extra draws for <g>
    tau = T // 2
    rel_plain = float(plain_err[tau] / plain[tau])
    rel_cv = float(est_err[tau] / est[tau])
    z = ((est - plain).abs() / (plain_err ** 2 + est_err ** 2).sqrt())[1:]
    line = {"metric": "statistical error of <C_N(tau)> per GPU-second (control variate vs plain)",
            "value": rel_cv * math.sqrt(t_cv), "unit": "relative error x sqrt(GPU s)", "higher_is_better": False,
            "n_gpus": 1, "dtype": a.precision, "data": "synthetic (device-drawn fields)",
            "config": {"workload": f"L={L}^3 T={T} N={len(nb.momenta((L,) * 3, 'PERFECT', 1.0, ef, 2.0)[0])} "
                                   f"Z2 a=0.5; train {cv_train} pairs "
                                   f"(seeds 1000..), eval {cv_eval} configs (seed 2000), <g> from {cv_extra} "
                                   f"extra fields (block means drawn directly, Philox4x32-10 seed 3000), net 3x conv3d(16, k3) on {G}^3 block means + MLP",
                       "tau": tau},
            "plain": {"rel_err": rel_plain, "gpu_seconds": t_plain, "rel_err_per_gpu_second": rel_plain *
                      math.sqrt(t_plain)},
            "control_variate": {"rel_err": rel_cv, "gpu_seconds": t_cv, "rel_err_per_gpu_second": rel_cv *
                                math.sqrt(t_cv)},
            "variance_ratio_median_over_tau": float(var_ratio[1:].median()),
            "variance_ratio_tau_mid": float(var_ratio[tau]),
            "unbiasedness_max_z_over_tau": float(z.max()),
            "training": {"pairs": int(C.shape[0]), "epochs": cv_epochs, "loss_first": losses[0],
                         "loss_last": losses[-1], "generation_s": t_gen, "training_s": t_train},
            "extra_fields": {"count": cv_extra, "gpu_seconds": t_extra, "sampler": "philox block means"},
            # the one-off costs (training pairs, training) charged to this single evaluation block
            "control_variate_with_one_off_costs": {"gpu_seconds": t_cv + t_gen + t_train,
                                                   "rel_err_per_gpu_second": rel_cv * math.sqrt(t_cv + t_gen + t_train)}}
    return line


def run_cv(a):
    import nrcps_b200 as nb
    if int(os.environ.get("RANK", "0")) != 0:
        return 0
    print(json.dumps(cv_core(nb.Context(0), a, a.cv_train, a.cv_eval, a.cv_extra, a.cv_epochs)))
    return 0


def run_trapped(a):
    """--workload trapped: the trapped few-body workload at its full shape."""
    import nrcps_b200 as nb
    if int(os.environ.get("RANK", "0")) != 0:
        return 0
    ctx = nb.Context(0)
    if a.cluster:
        ctx.set_option("fused.cluster", a.cluster)
    if a.kind >= 0:
        ctx.set_option("fused.kind", a.kind)
    line = trapped_core(ctx, a.trapped_configs, a.steps, a.warmup, 0 if a.no_cpu_baseline else 4)
    line.update({"n_gpus": 1, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                 "data": "synthetic (device-drawn fields, SHO sources)"})
    print(json.dumps(line))
    return 0


def main():
    a = parse()
    if a.impl == "reference":
        return run_reference(a)
    if a.workload == "uneven":
        return run_uneven(a)
    if a.workload == "cv":
        return run_cv(a)
    if a.workload == "trapped":
        return run_trapped(a)
    return run_b200(a)


if __name__ == "__main__":
    sys.exit(main())

"""Generates the golden fixtures in tests/golden/ from the reference itself.

Run here (where the reference tree and its CPU build exist), never on a GPU
box:

    make -C oracle/ref_build REF=<reference tree>
    python tests/golden/make_golden.py --ref <reference tree> [--only GROUP]

Sources of truth:
  * ranlx_kat.npz      -- Luscher's published ranlxs/ranlxd sequences, parsed
                          from the reference's own test (tests/ranlx/main.C).
  * ludcmp_kat.json    -- the reference's 10x10 Hilbert LU test
                          (tests/ludcmp_test/main.C) as printed by its binary.
  * batch_large.npz    -- the oracle's batch runner (o_run_batch) at the
                          uneven workload's largest shapes; the reference has
                          no batch driver, and the oracle is pinned to it by
                          the ensemble fixtures.
  * everything else    -- outputs of the reference's CPU path compiled from
                          its unchanged sources (oracle/_ref/nrcps_ref, see
                          oracle/ref_build/ref_driver.cc).
"""
from __future__ import annotations

import argparse
import json
import os
import re
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
REF_BIN = os.path.join(REPO, "oracle", "_ref", "nrcps_ref")


def run_ref(*args: str) -> str:
    out = subprocess.run([REF_BIN, *args], check=True, capture_output=True, text=True)
    return out.stdout


def parse_ranlx_kat(ref: str) -> dict:
    src = open(os.path.join(ref, "tests", "ranlx", "main.C")).read()
    xs = {int(k): float(v) for k, v in re.findall(r"xsn\[(\d+)\]=([0-9.]+)f;", src)}
    xd = {int(k): float(v) for k, v in re.findall(r"xdn\[(\d+)\]=([0-9.]+);", src)}
    assert sorted(xs) == list(range(96)) and sorted(xd) == list(range(48))
    return {
        # ranlxs lux 0 seed 32767: 20 blocks of 204 draws, compare xs[k+60]
        # of the last block -> 0-based stream outputs 19*204+60 .. +155.
        "ranlxs0_seed32767_first_index": np.int64(19 * 204 + 60),
        "ranlxs0_seed32767_times_2p24": np.array([xs[k] for k in range(96)]),
        # ranlxd lux 1 seed 32767: 20 blocks of 99 draws, compare xd[k+39].
        "ranlxd1_seed32767_first_index": np.int64(19 * 99 + 39),
        "ranlxd1_seed32767_times_2p48": np.array([xd[k] for k in range(48)]),
    }


def parse_ludcmp_kat(ref: str) -> dict:
    out = subprocess.run([os.path.join(REPO, "oracle", "_ref", "kat_ludcmp")], check=True,
                         capture_output=True, text=True).stdout
    det = re.search(r"^det = \(([-0-9.e+]+), ([-0-9.e+]+)\)", out, re.M)
    ldet = re.search(r"^log\(det\) = \(([-0-9.e+]+), ([-0-9.e+]+)\)", out, re.M)
    src = open(os.path.join(ref, "tests", "ludcmp_test", "main.C")).read()
    mdet = re.search(r"det = ([0-9.]+) \* 10\^(-?\d+) \(Mathematica", src)
    mldet = re.search(r"ldet = (-?[0-9.]+) \(Mathematica", src)
    return {
        "n": 10,
        "reference_det_printed": [float(det.group(1)), float(det.group(2))],
        "reference_logdet_printed": [float(ldet.group(1)), float(ldet.group(2))],
        "mathematica_det": float(mdet.group(1)) * 10.0 ** int(mdet.group(2)),
        "mathematica_logdet": float(mldet.group(1)),
    }


def rng_streams(tmp: str) -> dict:
    out = {}
    for kind in ["RANLXS0", "RANLXS1", "RANLXS2", "RANLXD1", "RANLXD2", "RAN2"]:
        for skip, count in [(0, 600), (200_000, 200)]:
            fn = os.path.join(tmp, f"{kind}_{skip}.bin")
            run_ref("rng", f"rng={kind}", "seed=1234", f"skip={skip}", f"count={count}", f"out={fn}")
            out[f"{kind}_seed1234_skip{skip}"] = np.fromfile(fn)
    fn = os.path.join(tmp, "gauss.bin")
    run_ref("gauss", "rng=RANLXS2", "seed=99", "skip=0", "count=400", f"out={fn}")
    out["gauss_RANLXS2_seed99"] = np.fromfile(fn)
    return out


def fields(tmp: str) -> dict:
    out = {}
    cases = [("ZTWO", "RANLXS2", 1234, 4, 3), ("ZTWO", "RANLXD1", 7, 6, 2), ("GAUSS", "RANLXS2", 99, 4, 2),
             ("COMPLEXGAUSS", "RANLXS1", 5, 4, 1), ("ZTHREE", "RANLXS0", 11, 4, 2), ("ZTWO", "RAN2", 3, 4, 2)]
    for field, kind, seed, L, slices in cases:
        fn = os.path.join(tmp, "f.bin")
        run_ref("field", f"field={field}", f"rng={kind}", f"seed={seed}", f"L={L}", f"slices={slices}",
                f"out={fn}")
        out[f"{field}_{kind}_seed{seed}_L{L}"] = np.fromfile(fn).reshape(slices, L ** 3, 2)
    return out


# Keys passed to the reference binary that name a path of the generating
# machine; they are left out of the stored arguments.
_LOCAL_KEYS = ("sho_dir", "out")

# Above this many source entries only every SOURCE_STRIDE-th entry of the
# sources is stored (sources_sample); the tests rebuild the full sources with
# the library's own builders and check them against the sample.
SOURCE_FULL_MAX = 1 << 16
SOURCE_STRIDE = 61


def ensemble(tmp: str, name: str, **kv) -> dict:
    d = os.path.join(tmp, name)
    os.makedirs(d, exist_ok=True)
    args = [f"{k}={v}" for k, v in kv.items()] + [f"out={d}"]
    info = json.loads(run_ref("ensemble", *args).strip().splitlines()[-1])
    L, T = int(kv["L"]), int(kv["T"])
    N = info["N"]
    nmeas = 2 * N if kv.get("mode") == "slater2" else N
    sources = np.fromfile(os.path.join(d, "sources.bin"), dtype=np.complex128).reshape(N, L ** 3)
    res = {
        "dets": np.fromfile(os.path.join(d, "dets.bin"), dtype=np.complex128).reshape(-1, T, nmeas),
        "args": json.dumps({k: v for k, v in kv.items() if k not in _LOCAL_KEYS}),
    }
    if sources.size <= SOURCE_FULL_MAX:
        res["sources"] = sources
    else:
        res["sources_sample"] = sources[:, ::SOURCE_STRIDE].copy()
        res["sources_stride"] = np.int64(SOURCE_STRIDE)
    if os.path.exists(os.path.join(d, "momenta.txt")):
        res["momenta"] = np.loadtxt(os.path.join(d, "momenta.txt"), dtype=np.int64).reshape(-1, 4)
    if os.path.exists(os.path.join(d, "props.bin")):
        res["props"] = np.fromfile(os.path.join(d, "props.bin"), dtype=np.complex128).reshape(-1, N, L ** 3)
    if os.path.exists(os.path.join(d, "fields.bin")):
        res["fields"] = np.fromfile(os.path.join(d, "fields.bin")).reshape(-1, L ** 3, 2)
    return res


def lu_cases(tmp: str) -> dict:
    rs = np.random.default_rng(20251203)
    mats, dets = [], []
    for n in range(1, 13):
        for _ in range(2):
            m = rs.standard_normal((n, n)) + 1j * rs.standard_normal((n, n))
            if _ == 1 and n > 2:
                m[1] = m[0] * (1 + 1e-9)  # nearly singular: pivoting matters
            fn = os.path.join(tmp, "m.bin")
            with open(fn, "wb") as f:
                np.array([1, n], dtype=np.int32).tofile(f)
                m.astype(np.complex128).tofile(f)
            run_ref("lu", f"in={fn}", f"out={fn}.det")
            dets.append(np.fromfile(fn + ".det", dtype=np.complex128)[0])
            mats.append(m)
    out = {f"m{i}": m for i, m in enumerate(mats)}
    out["dets"] = np.array(dets)
    return out


def sho_coefficients(ref: str) -> dict:
    d = os.path.join(ref, "production", "slater_det2_trapped", "sources")
    out = {}
    for n in range(10):
        lines = []
        for line in open(os.path.join(d, f"source.{n}")):
            p = line.split()
            if len(p) == 5:
                lines.append([int(p[0]), int(p[1]), int(p[2]), float(p[3]), float(p[4])])
        out[str(n)] = lines
    return out


# GeneralizedTwoBody (src/two_body/two_body.C:209-288) cases: L, distinct
# vector, wave function, lambda, seed of the random propagators
OHPAIR_CASES = [(8, (1, 0, 0), "TGND", 0.25, 3), (8, (1, 1, 2), "PAIR1", 0.5, 4), (6, (1, 2, 3), "TGND", 0.3, 5),
                (8, (0, 0, 0), "UNIFORM", 0.1, 6)]


def ohpair_cases(tmp: str) -> dict:
    """Tables, random propagators and Run / Run2 for every OctahedralRep,
    from the reference's GeneralizedTwoBody (oracle/ref_build/ohpair_dump.cc)."""
    out = {}
    for k, (L, vec, wf, lam, seed) in enumerate(OHPAIR_CASES):
        path = os.path.join(tmp, f"oh{k}.bin")
        subprocess.run([os.path.join(REPO, "oracle", "_ref", "ohpair_dump"), f"L={L}", "vec=%d,%d,%d" % vec,
                        f"wf={wf}", f"lambda={lam!r}", f"seed={seed}", f"out={path}"], check=True,
                       capture_output=True)
        b = open(path, "rb").read()
        nt, vol = np.frombuffer(b[:8], np.int32)
        o = 8
        take = lambda dt, n: (np.frombuffer(b[o:o + n * np.dtype(dt).itemsize], dt).copy(),  # noqa: E731
                              o + n * np.dtype(dt).itemsize)
        opp, o = take(np.int32, vol)
        shift, o = take(np.int32, nt * vol)
        hsw, o = take(np.float64, nt * vol)
        wts, o = take(np.float64, nt * 10)
        props, o = take(np.float64, 4 * vol)
        run, o = take(np.float64, 20)
        run2, o = take(np.float64, 20)
        out[f"c{k}_L"] = np.int64(L)
        out[f"c{k}_opp"] = opp
        out[f"c{k}_shift"] = shift.reshape(nt, vol)
        out[f"c{k}_hsw"] = hsw.reshape(nt, vol)
        out[f"c{k}_weights"] = wts.reshape(nt, 10)
        out[f"c{k}_props"] = props.view(np.complex128).reshape(2, vol)
        out[f"c{k}_run"] = run.view(np.complex128)
        out[f"c{k}_run2"] = run2.view(np.complex128)
    out["cases"] = np.int64(len(OHPAIR_CASES))
    return out


def result_files(tmp: str, name: str, sho: dict, **kv) -> dict:
    """The drivers' own result files for a small run: the reference's
    accumulation and Fprintf rows (one row per block of `unload`
    configurations), next to the raw determinants they were made from."""
    d = os.path.join(tmp, name)
    os.makedirs(d, exist_ok=True)
    if kv.get("sources") == "sho":
        write_sho_dir(sho, os.path.join(d, "sho"))
        kv["sho_dir"] = os.path.join(d, "sho")
    res = ensemble(tmp, name, results=d, **kv)
    texts = {}
    for fn in sorted(os.listdir(d)):
        if fn.startswith("slater.") or (fn.startswith("z") and "." in fn):
            texts[fn] = open(os.path.join(d, fn)).read()
    res["result_files"] = json.dumps(texts)
    res["args"] = json.dumps({k: v for k, v in json.loads(str(res["args"])).items() if k != "results"})
    return res


# Multilevel branching trees (production/two_body-branched/main.C:23-80 over
# the current classes, oracle/ref_build/ref_driver.cc run_branch): L, levels,
# branches, steps, trees, field, seed; plane-wave sources at p = 0, TGND sink.
BRANCH_CASES = [(8, 3, 2, 2, 2, "ZTWO", 11), (8, 2, 3, 3, 2, "GAUSS", 11), (4, 4, 2, 1, 2, "ZTWO", 11),
                (8, 10, 2, 2, 1, "ZTWO", 7)]


def branching_cases(tmp: str) -> dict:
    out = {}
    for k, (L, levels, branches, steps, trees, field, seed) in enumerate(BRANCH_CASES):
        fn = os.path.join(tmp, f"br{k}.bin")
        run_ref("branch", f"L={L}", f"levels={levels}", f"branches={branches}", f"steps={steps}",
                f"trees={trees}", f"field={field}", f"seed={seed}", "rng=RANLXS2",
                "couplings=0.019894367886486918", "cutoff=2.0", f"out={fn}")
        out[f"c{k}_params"] = np.array([L, levels, branches, steps, trees, seed], dtype=np.int64)
        out[f"c{k}_field"] = np.array(field)
        out[f"c{k}_corr"] = np.fromfile(fn, dtype=np.complex128)
    out["cases"] = np.int64(len(BRANCH_CASES))
    out["couplings"] = np.array([0.019894367886486918])
    return out


def write_sho_dir(sho: dict, shodir: str) -> None:
    os.makedirs(shodir, exist_ok=True)
    for n, lines in sho.items():
        with open(os.path.join(shodir, f"source.{n}"), "w") as f:
            for l in lines:
                f.write(f"{l[0]} {l[1]} {l[2]} {l[3]!r} {l[4]!r}\n")


# The uneven-batch workload's largest and middle shapes (L, T, n_conf, N) with
# E_F between closed shells; N = 7, 19, 33 are the shells |n|^2 <= 1, 2, 4.
BATCH_LARGE_JOBS = [(48, 128, 1, 33), (24, 64, 1, 19), (16, 32, 2, 7)]
_SHELL = {7: 1.5, 19: 2.5, 33: 4.5}


def batch_large() -> dict:
    """Uneven-batch jobs at the workload's largest shapes through the oracle's
    batch runner (o_run_batch, Gaussian fields a = 0.3, RANLXS2 seed 99).  The
    oracle is pinned to the reference on the ensemble fixtures; the reference
    itself has no batch driver."""
    import sys
    sys.path.insert(0, REPO)
    from oracle import oracle as O
    jobs, meta = [], []
    for L, T, nc, N in BATCH_LARGE_JOBS:
        ef = 0.5 * (2 * np.pi / L) ** 2 * _SHELL[N]
        idx, _, _ = O.momenta((L,) * 3, "PERFECT", 1.0, ef, (2 * O.PI) ** 2)
        assert len(idx) == N
        jobs.append((L, T, nc, list(idx)))
        meta.append([L, T, nc, N])
    outs = O.run_batch(jobs, "RANLXS2", 99, "GAUSS", 0.3)
    res = {f"dets{i}": o for i, o in enumerate(outs)}
    res["jobs"] = np.array(meta, dtype=np.int64)
    res["fermi_energies"] = np.array([0.5 * (2 * np.pi / L) ** 2 * _SHELL[N] for L, _, _, N in BATCH_LARGE_JOBS])
    res["args"] = json.dumps({"rng": "RANLXS2", "seed": 99, "field": "GAUSS", "a": 0.3, "kin_dt": 0.5,
                              "cutoff": 2.0})
    return res


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("NRCPS_REFERENCE", ""),
                    help="the reference tree (or set NRCPS_REFERENCE)")
    ap.add_argument("--only", default="",
                    help="regenerate one group only: ohpair, small, config2, trapped48, results, branching, "
                         "batch_large")
    a = ap.parse_args()
    need_ref = a.only != "batch_large"
    if need_ref and not a.ref:
        ap.error("--ref (or NRCPS_REFERENCE) names the reference tree")
    if need_ref and (not os.path.exists(REF_BIN) or
                     not os.path.exists(os.path.join(REPO, "oracle", "_ref", "ohpair_dump"))):
        subprocess.check_call(["make", "-s", "-C", os.path.join(REPO, "oracle", "ref_build"), f"REF={a.ref}"])
    if a.only in ("", "ohpair"):
        with tempfile.TemporaryDirectory() as tmp:
            np.savez_compressed(os.path.join(HERE, "ohpair.npz"), **ohpair_cases(tmp))
    sho = sho_coefficients(a.ref) if need_ref else None
    if a.only in ("", "small"):
        np.savez_compressed(os.path.join(HERE, "ranlx_kat.npz"), **parse_ranlx_kat(a.ref))
        json.dump(parse_ludcmp_kat(a.ref), open(os.path.join(HERE, "ludcmp_kat.json"), "w"), indent=1)
        json.dump(sho, open(os.path.join(HERE, "sho_coefficients.json"), "w"))
        with tempfile.TemporaryDirectory() as tmp:
            np.savez_compressed(os.path.join(HERE, "rng_streams.npz"), **rng_streams(tmp))
            np.savez_compressed(os.path.join(HERE, "fields.npz"), **fields(tmp))
            np.savez_compressed(os.path.join(HERE, "lu_cases.npz"), **lu_cases(tmp))
            # config 1 of the benchmark: L=16, T=32, N=7 (E_F=0.1), Z2 a=0.5, seed 1234
            np.savez_compressed(os.path.join(HERE, "ensemble_config1.npz"), **ensemble(
                tmp, "c1", L=16, T=32, ef=0.1, seed=1234, rng="RANLXS2", field="ZTWO",
                couplings="0.019894367886486918", cutoff=2.0, configs=2, dump_fields=3))
            # small lattice, p-dependent interaction (3 couplings), ranlxd, props dumped
            np.savez_compressed(os.path.join(HERE, "ensemble_multicoupling.npz"), **ensemble(
                tmp, "mc", L=8, T=8, ef=0.35, seed=5, rng="RANLXD1", field="ZTWO",
                couplings="0.02,0.004,0.001", cutoff=0.99999, configs=2, dump_props=4))
            # Gaussian field, a=0.3
            np.savez_compressed(os.path.join(HERE, "ensemble_gauss.npz"), **ensemble(
                tmp, "g", L=8, T=8, ef=0.35, seed=99, rng="RANLXS2", field="GAUSS",
                couplings=repr(0.09 / (4 * np.pi)), cutoff=2.0, configs=2))
            # trapped, SHO sources, pair sink (production/slater_det2_trapped shape)
            shodir = os.path.join(tmp, "sho")
            write_sho_dir(sho, shodir)
            np.savez_compressed(os.path.join(HERE, "ensemble_trapped.npz"), **ensemble(
                tmp, "tr", L=8, T=6, sources="sho", N=4, sho_dir=shodir, lambda1=2.0, lambda2=2.0,
                lambda3=2.0, mode="slater2", potential=1, kappa=0.005, ptype="EXP", wavefunc="TGND",
                tb_disp="STANDARD", tb_lambda=0.176776695, seed=31, rng="RANLXS2", field="ZTWO",
                couplings="0.019894367886486918", cutoff=0.99999, configs=2, dump_props=3))
    if a.only in ("", "config2"):
        # the batched workload's shape: L=32, T=64, N=19 (E_F=0.045), Z2 a=0.5,
        # RANLXS2 seed 7 (production/slater_det/main.C:185-220); 2 configurations
        with tempfile.TemporaryDirectory() as tmp:
            np.savez_compressed(os.path.join(HERE, "ensemble_config2.npz"), **ensemble(
                tmp, "c2", L=32, T=64, ef=0.045, seed=7, rng="RANLXS2", field="ZTWO",
                couplings="0.019894367886486918", cutoff=2.0, configs=2))
    if a.only in ("", "trapped48"):
        # the trapped few-body workload's shape: L=48, T=128, SHO N=10 from
        # production/slater_det2_trapped/sources/source.{0..9} with that
        # production's lambda = 4 (args/one_body.arg), [K,V,I,V,K] with a
        # harmonic EXP trap kappa = 0.005, TGND pair sink, Z2 a=0.5, RANLXS2
        # seed 31 (production/slater_det2_trapped/main-no_cum.C:90-128,185-210)
        with tempfile.TemporaryDirectory() as tmp:
            shodir = os.path.join(tmp, "sho")
            write_sho_dir(sho, shodir)
            np.savez_compressed(os.path.join(HERE, "ensemble_trapped48.npz"), **ensemble(
                tmp, "t48", L=48, T=128, sources="sho", N=10, sho_dir=shodir, lambda1=4.0, lambda2=4.0,
                lambda3=4.0, mode="slater2", potential=1, kappa=0.005, ptype="EXP", wavefunc="TGND",
                tb_disp="STANDARD", tb_lambda=0.176776695, seed=31, rng="RANLXS2", field="ZTWO",
                couplings="0.019894367886486918", cutoff=2.0, configs=2))
    if a.only in ("", "results"):
        # results/slater.<m> of production/slater_det/main.C (|det|^2 rows) and
        # results/slater.<m> + z<k>.<m> of production/slater_det2_trapped/main-cum.C
        # (det rows, Nc = 6 log-det cumulants), 6 configurations in blocks of 2
        with tempfile.TemporaryDirectory() as tmp:
            np.savez_compressed(os.path.join(HERE, "results_slater.npz"), **result_files(
                tmp, "rs", sho, L=8, T=6, ef=0.35, seed=5, rng="RANLXS2", field="ZTWO",
                couplings="0.019894367886486918", cutoff=2.0, configs=6, unload=2))
            np.savez_compressed(os.path.join(HERE, "results_trapped_cum.npz"), **result_files(
                tmp, "rc", sho, L=8, T=6, sources="sho", N=4, lambda1=2.0, lambda2=2.0, lambda3=2.0,
                mode="slater2", potential=1, kappa=0.005, ptype="EXP", wavefunc="TGND", tb_disp="STANDARD",
                tb_lambda=0.176776695, seed=31, rng="RANLXS2", field="ZTWO", couplings="0.019894367886486918",
                cutoff=0.99999, configs=6, unload=2, cumulants=6))
    if a.only in ("", "branching"):
        with tempfile.TemporaryDirectory() as tmp:
            np.savez_compressed(os.path.join(HERE, "branching.npz"), **branching_cases(tmp))
    if a.only in ("", "batch_large"):
        np.savez_compressed(os.path.join(HERE, "batch_large.npz"), **batch_large())
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()

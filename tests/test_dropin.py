"""The drop-in: the reference's own class layer (src/*/*.C compiled in its GPU
configuration) with nrcps_b200/shim in place of its CUDA units, driven by the
same production loop as the CPU reference, must reproduce the reference's CPU
determinants.  Binary: oracle/_ref/nrcps_dropin (built where the reference
tree is present, by `make -C nrcps_b200/shim` and `make -C oracle/ref_build dropin`).
"""
import json
import os
import subprocess

import numpy as np
import pytest

from conftest import GOLDEN, REPO

pytestmark = pytest.mark.gpu

DROPIN = os.path.join(REPO, "oracle", "_ref", "nrcps_dropin")


def _run(tmp_path, args: dict) -> np.ndarray:
    if not os.path.exists(DROPIN):
        pytest.skip("drop-in binary not built (needs the reference tree at build time)")
    out = tmp_path / "out"
    out.mkdir()
    cmd = [DROPIN, "ensemble"] + [f"{k}={v}" for k, v in args.items()] + [f"out={out}"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    return np.fromfile(out / "dets.bin", dtype=np.complex128)


def _rel(a, b):
    return np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-300))


@pytest.mark.parametrize("name", ["ensemble_config1.npz", "ensemble_multicoupling.npz"])
def test_dropin_reproduces_reference(tmp_path, golden, name):
    g = golden(name)
    args = json.loads(str(g["args"]))
    args = {k: v for k, v in args.items() if not k.startswith("dump_")}
    dets = _run(tmp_path, args).reshape(g["dets"].shape)
    assert _rel(dets, g["dets"]) < 1e-12


def test_dropin_trapped_pair_sink(tmp_path, golden):
    """SlaterDet2 + TwoBody + Potential + SHO sources through the shims."""
    g = golden("ensemble_trapped.npz")
    args = json.loads(str(g["args"]))
    args = {k: v for k, v in args.items() if not k.startswith("dump_")}
    sho = json.load(open(os.path.join(GOLDEN, "sho_coefficients.json")))
    d = tmp_path / "sho"
    d.mkdir()
    for n, lines in sho.items():
        with open(d / f"source.{n}", "w") as f:
            for l in lines:
                f.write(f"{l[0]} {l[1]} {l[2]} {l[3]!r} {l[4]!r}\n")
    args["sho_dir"] = str(d)
    dets = _run(tmp_path, args).reshape(g["dets"].shape)
    assert _rel(dets, g["dets"]) < 1e-12

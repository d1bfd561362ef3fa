"""Block accumulators, cumulant sums, their result rows and the jackknife.

CPU: the oracle's restatement of the drivers' accumulation against a
vectorised numpy form, and the result-file rows.  GPU: the device kernels
(nrcps_accumulate, nrcps_jackknife) against the oracle and a direct numpy
jackknife.
"""
import json

import numpy as np
import pytest

from oracle import oracle as O
from nrcps_b200 import parallel


def _dets(n_conf, T, nmeas, seed):
    rs = np.random.default_rng(seed)
    return rs.standard_normal((n_conf, T, nmeas)) + 1j * rs.standard_normal((n_conf, T, nmeas))


def _np_jackknife(x, n_bins, eff=False):
    per = x.shape[0] // n_bins
    x = x[: per * n_bins]
    tot = x.sum(0)
    loo = (tot[None, :] - x.reshape(n_bins, per, -1).sum(1)) / (x.shape[0] - per)
    mu = tot / x.shape[0]
    f = (n_bins - 1) / n_bins
    err = np.sqrt(f * ((loo - mu) ** 2).sum(0))
    if not eff:
        return mu, err
    e0 = np.log(tot[:-1] / tot[1:])
    bs = x.reshape(n_bins, per, -1).sum(1)
    eb = np.log((tot[None, :-1] - bs[:, :-1]) / (tot[None, 1:] - bs[:, 1:]))
    return mu, err, e0, np.sqrt(f * ((eb - e0) ** 2).sum(0))


def test_oracle_block_sums_match_numpy():
    d = _dets(7, 5, 6, 1)
    corr, z = O.block_sums(d, "slater2", 4)
    assert np.allclose(corr, d.sum(0).T, rtol=1e-14)
    l = np.log(np.abs(d))
    for k in range(4):
        assert np.allclose(z[k], (l ** (k + 1)).sum(0).T, rtol=1e-13)
    corr0, _ = O.block_sums(d, "slater", 0)
    assert np.allclose(corr0.real, (np.abs(d) ** 2).sum(0).T, rtol=1e-14)


def test_cumulant_rows_format():
    z = np.arange(2 * 3 * 4, dtype=float).reshape(2, 3, 4) + 0.5
    rows = parallel.block_rows_cumulants(z, world=2, unload_period=1)
    assert len(rows) == 2 and len(rows[0]) == 3
    assert rows[1][2] == "".join("%.15e " % (v / 2.0) for v in z[1, 2])


@pytest.mark.gpu
@pytest.mark.parametrize("mode,nc", [("slater", 0), ("slater2", 6), ("slater", 3)])
def test_device_accumulate_matches_oracle(mode, nc):
    import torch
    import nrcps_b200 as nb
    ctx = nb.default_context()
    d = _dets(33, 9, 8, 2)
    corr, z = nb.accumulate(torch.from_numpy(d).to(ctx.device), mode, nc, ctx)
    rc, rz = O.block_sums(d, mode, nc)
    assert np.allclose(corr.cpu().numpy(), rc, rtol=1e-13, atol=0)
    if nc:
        assert np.allclose(z.cpu().numpy(), rz, rtol=1e-12, atol=1e-12)


@pytest.mark.gpu
def test_device_jackknife_matches_numpy():
    import torch
    import nrcps_b200 as nb
    ctx = nb.default_context()
    rs = np.random.default_rng(3)
    x = np.exp(-0.1 * np.arange(12))[None, :] * (1.0 + 0.1 * rs.standard_normal((1003, 12)))
    mu, err, em, ee = nb.jackknife(torch.from_numpy(x).to(ctx.device), 17, True, ctx)
    rmu, rerr, rem, ree = _np_jackknife(x, 17, True)
    for a, b in ((mu, rmu), (err, rerr), (em, rem), (ee, ree)):
        assert np.allclose(a.cpu().numpy(), b, rtol=1e-10, atol=0)


# ------------------------------------------------------------ result files
def _blocks(g):
    args = json.loads(str(g["args"]))
    return g["dets"], int(args["unload"]), int(args.get("cumulants", 0)), args.get("mode", "slater")


@pytest.mark.parametrize("name", ["results_slater.npz", "results_trapped_cum.npz"])
def test_result_rows_byte_identical_to_the_reference_files(golden, name):
    """results/slater.<m> (and z<k>.<m>) as written by the reference's own
    accumulation and Fprintf (production/slater_det/main.C:208-247,
    production/slater_det2_trapped/main-cum.C:219-270), from the same raw
    determinants: parallel.accumulate / cumulant_sums + block_rows reproduce
    every file byte for byte."""
    g = golden(name)
    dets, unload, nc, mode = _blocks(g)
    files = json.loads(str(g["result_files"]))
    nmeas = dets.shape[2]
    got = {f"slater.{m + 1}": "" for m in range(nmeas)}
    got.update({f"z{k + 1}.{m + 1}": "" for k in range(nc) for m in range(nmeas)})
    for b in range(dets.shape[0] // unload):
        blk = dets[b * unload:(b + 1) * unload]
        for m, row in enumerate(parallel.block_rows(parallel.accumulate(blk, mode), 1, unload)):
            got[f"slater.{m + 1}"] += row + "\n"
        if nc:
            for k, rows in enumerate(parallel.block_rows_cumulants(parallel.cumulant_sums(blk, nc), 1, unload)):
                for m, row in enumerate(rows):
                    got[f"z{k + 1}.{m + 1}"] += row + "\n"
    assert sorted(got) == sorted(files)
    for fn in files:
        assert got[fn] == files[fn], fn


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["results_slater.npz", "results_trapped_cum.npz"])
def test_device_accumulate_result_rows(golden, name):
    """The device accumulator (nrcps_accumulate) on the reference's raw
    determinants: the slater.<m> rows byte for byte; the cumulant rows, whose
    log and hypot are CUDA's (within an ulp or two of the C library's), within
    1e-13 of the row's largest value (the sums of the odd powers of log|det|
    cancel, so single values can be far smaller than the row)."""
    import torch
    import nrcps_b200 as nb
    ctx = nb.default_context()
    g = golden(name)
    dets, unload, nc, mode = _blocks(g)
    files = json.loads(str(g["result_files"]))
    for b in range(dets.shape[0] // unload):
        blk = torch.from_numpy(np.ascontiguousarray(dets[b * unload:(b + 1) * unload])).to(ctx.device)
        corr, z = nb.accumulate(blk, mode, nc, ctx)
        for m, row in enumerate(parallel.block_rows(corr, 1, unload)):
            assert row == files[f"slater.{m + 1}"].splitlines()[b], (m, b)
        if nc:
            for k, rows in enumerate(parallel.block_rows_cumulants(z, 1, unload)):
                for m, row in enumerate(rows):
                    want = np.array(files[f"z{k + 1}.{m + 1}"].splitlines()[b].split(), dtype=float)
                    got = np.array(row.split(), dtype=float)
                    assert np.allclose(got, want, rtol=0, atol=1e-13 * np.abs(want).max()), (k, m, b)

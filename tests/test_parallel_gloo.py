"""The N > 1 path on CPU: two gloo ranks, each with the reference's per-rank
seed, accumulate their correlators and meet in the GlobalSum; the result
must equal one process computing both ranks' ensembles (the oracle stands in
for the per-rank GPU computation)."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from nrcps_b200 import parallel


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_dets(rank, seed):
    from oracle import oracle as O
    job = O.Job(L=4, T=4, configs=3, seed=parallel.rank_seed(seed, rank))
    idx, _, _ = O.momenta(job.dims, "PERFECT", 1.0, 1.0, job.cutoff_sq)
    return O.run_ensemble(job, O.plane_wave_sources(job.dims, idx))


def _worker(rank, world, port, seed, out_path):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        corr = torch.from_numpy(parallel.accumulate(_rank_dets(rank, seed), "slater"))
        parallel.global_sum(corr)
        if rank == 0:
            np.save(out_path, corr.numpy())
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_two_gloo_ranks_match_single_process(tmp_path):
    seed, world = 1234, 2
    out = str(tmp_path / "corr.npy")
    mp.spawn(_worker, args=(world, _free_port(), seed, out), nprocs=world, join=True)
    got = np.load(out)
    want = sum(parallel.accumulate(_rank_dets(r, seed), "slater") for r in range(world))
    assert np.allclose(got, want, rtol=1e-14, atol=0)
    rows = parallel.block_rows(got, world)
    assert len(rows) == got.shape[0] and len(rows[0].split()) == 2 * got.shape[1]


def test_rank_seed_matches_reference_rule():
    assert parallel.rank_seed(7012, 0) == 7012 and parallel.rank_seed(7012, 3) == 7012 + 3 * 491


def test_accumulate_modes():
    d = np.array([[[1 + 1j, 2]], [[0.5j, -1]]])  # [conf=2, T=1, nmeas=2]
    assert np.allclose(parallel.accumulate(d, "slater"), [[2.25], [5.0]])
    assert np.allclose(parallel.accumulate(d, "slater2"), [[1 + 1.5j], [1.0]])

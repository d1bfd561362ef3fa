"""Configurations sharded over ranks, with the reference's MPI semantics.

The reference runs one independent ensemble per MPI rank and meets only in
``Comms::GlobalSum`` (src/sys/sysfunc.C:114-151):

* rank r seeds its generator with ``seed + 491 * r`` (src/random/random.C:88);
* each rank accumulates, per block of configurations, ``corr[n][t] +=
  |det S_{n+1}(t)|^2`` (production/slater_det/main.C:208-211) or the raw
  determinant (production/slater_det2_trapped/main-no_cum.C:205-207);
* the block's sums are reduced over ranks (MPI_Reduce SUM to rank 0,
  main.C:226) and written as the average over ``size * unload_period``
  configurations (main.C:229-241), one row per block, ``%.*e %.*e`` pairs
  with PREC = 15 (include/config.h:41).

Here one process drives one GPU; the reduction is a ``torch.distributed``
all-reduce (NCCL between GPUs, gloo on CPU), and only rank 0 writes.
"""
from __future__ import annotations

from typing import Iterable, List, Optional

import numpy as np
import torch

PREC = 15  # include/config.h:41


def rank_seed(seed: int, rank: int) -> int:
    """Random::Random's per-rank seed (src/random/random.C:88)."""
    return seed + 491 * rank


def accumulate(dets, mode: str = "slater"):
    """Sum over configurations of |det|^2 (mode 'slater') or det ('slater2').

    dets: [n_conf, T, nmeas] complex (numpy or torch); returns [nmeas, T] complex128.
    """
    if isinstance(dets, torch.Tensor):
        d = dets.to(torch.complex128)
        s = (d.real ** 2 + d.imag ** 2).sum(0).to(torch.complex128) if mode == "slater" else d.sum(0)
        return s.transpose(0, 1).contiguous()
    d = np.asarray(dets, dtype=np.complex128)
    s = (np.abs(d) ** 2).sum(0).astype(np.complex128) if mode == "slater" else d.sum(0)
    return np.ascontiguousarray(s.T)


def global_sum(corr: torch.Tensor, group=None) -> torch.Tensor:
    """Comms::GlobalSum over ranks (in place; every rank receives the sum)."""
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized() and dist.get_world_size(group) > 1:
        if corr.is_complex():
            v = torch.view_as_real(corr)
            dist.all_reduce(v, group=group)
        else:
            dist.all_reduce(corr, group=group)
    return corr


def block_rows(corr, world: int, unload_period: int = 1) -> List[str]:
    """The reference's result rows for one block: one line per measured minor,
    T pairs 're im ' with %.15e, averaged over world * unload_period."""
    c = corr.cpu().numpy() if isinstance(corr, torch.Tensor) else np.asarray(corr)
    block = float(world * unload_period)
    rows = []
    for n in range(c.shape[0]):
        rows.append("".join("%.*e %.*e " % (PREC, v.real / block, PREC, v.imag / block) for v in c[n]))
    return rows


def block_rows_cumulants(z, world: int, unload_period: int = 1) -> List[List[str]]:
    """The cumulant files' rows for one block (results/z<k+1>.<m+1>,
    production/slater_det2_trapped/main-cum.C:263-270): per cumulant k and
    measured minor m one line of T values '%.15e ' (real part), averaged over
    world * unload_period."""
    zz = z.cpu().numpy() if isinstance(z, torch.Tensor) else np.asarray(z)
    block = float(world * unload_period)
    return [["".join("%.*e " % (PREC, v / block) for v in zz[k, m]) for m in range(zz.shape[1])]
            for k in range(zz.shape[0])]


def write_block(files: Iterable, corr, world: int, unload_period: int = 1) -> None:
    """Appends one block row to each results/slater.<n> stream (rank 0 only)."""
    for f, row in zip(files, block_rows(corr, world, unload_period)):
        f.write(row + "\n")


def shard_first_config(rank: int, n_conf: int, block: int = 0) -> int:
    """First configuration index of this rank's block within its own stream.

    Every rank owns its whole stream (its own seed), so configuration c of
    block b on any rank is stream configuration b * n_conf + c."""
    return block * n_conf

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
    """Sum over configurations of |det|^2 (mode 'slater') or det ('slater2'),
    configuration after configuration as the drivers' `corr[n][t] += ...`
    (|det|^2 as re*re + im*im, the real part of tmp*conj(tmp)), so that the
    sums -- and the result rows printed from them -- are the reference's to
    the bit.

    dets: [n_conf, T, nmeas] complex (numpy or torch); returns [nmeas, T]
    complex128 (a device tensor through the library's kernel for CUDA
    tensors, the same type as the input otherwise)."""
    if isinstance(dets, torch.Tensor) and dets.is_cuda:
        from .api import accumulate as device_accumulate
        corr, _ = device_accumulate(dets, mode, 0)
        return corr
    as_torch = isinstance(dets, torch.Tensor)
    d = np.asarray(dets.numpy() if as_torch else dets, dtype=np.complex128)
    s = np.zeros(d.shape[1:], dtype=np.complex128)
    for c in range(d.shape[0]):
        if mode == "slater":
            s.real += d[c].real * d[c].real + d[c].imag * d[c].imag
        else:
            s += d[c]
    out = np.ascontiguousarray(s.T)
    return torch.from_numpy(out) if as_torch else out


def cumulant_sums(dets, n_cumulants: int):
    """The log-det moments of production/slater_det2_trapped/main-cum.C:219-233
    on the host: cum[0] = log(abs(det)), cum[k] = cum[0] cum[k-1],
    z[k][m][t] += cum[k], configuration after configuration, with the C
    library's log and hypot (math.log, abs of a Python complex) as the
    reference's.  dets [n_conf, T, nmeas] -> z [n_cumulants, nmeas, T]."""
    import math
    d = np.asarray(dets, dtype=np.complex128)
    n_conf, T, nmeas = d.shape
    z = np.zeros((n_cumulants, nmeas, T))
    for c in range(n_conf):
        for t in range(T):
            for m in range(nmeas):
                c0 = math.log(abs(complex(d[c, t, m])))
                p = c0
                for k in range(n_cumulants):
                    z[k, m, t] += p
                    p = c0 * p
    return z


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

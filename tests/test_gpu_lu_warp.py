"""The warp-per-minor determinant kernel against the thread-per-minor kernel
and the oracle's ludcmp restatement (src/utils/ludcmp.C:9-65, driven as
SlaterDet::Run / SlaterDet2::Run, src/slater_det/slater_det.C:59-115).

Both kernels run the same Crout arithmetic in the same order, so they agree
far inside the FP64 tolerance (1e-12 relative) of the parity tests.
"""
import numpy as np
import pytest
import torch

from oracle import oracle as O

pytestmark = pytest.mark.gpu

nb = pytest.importorskip("nrcps_b200")

FP64_REL = 1e-12


@pytest.fixture(scope="module")
def ctx():
    return nb.default_context()


def _dets(ctx, S, P=None, mode=0, log=False, warp=1):
    ctx.set_option("lu.warp", warp)
    try:
        out = nb.slater_dets(S, P, mode=mode, log=log, ctx=ctx)
        ctx.synchronize()
        return out.cpu().numpy()
    finally:
        ctx.set_option("lu.warp", 1)


def _random(nconf, N, seed):
    rs = np.random.default_rng(seed)
    return rs.standard_normal((nconf, N, N)) + 1j * rs.standard_normal((nconf, N, N))


@pytest.mark.parametrize("N,mode,log", [(1, 0, False), (7, 0, False), (19, 0, False), (19, 1, False), (19, 0, True),
                                        (32, 0, False), (32, 1, True), (33, 0, False),
                                        (64, 1, False), (65, 0, False)])
def test_warp_kernel_agrees_with_thread_kernel(ctx, N, mode, log):
    S = torch.from_numpy(_random(37, N, N + 100 * mode)).to(ctx.device)
    P = torch.from_numpy(_random(37, N, N + 7)).to(ctx.device) if mode else None
    a = _dets(ctx, S, P, mode, log, warp=1)
    b = _dets(ctx, S, P, mode, log, warp=0)
    if log:  # compare exp of the log form, branch-free
        a, b = np.exp(a), np.exp(b)
    assert np.max(np.abs(a - b) / np.abs(b)) < FP64_REL


def test_warp_kernel_matches_oracle_minors(ctx):
    S = _random(5, 19, 3)
    got = _dets(ctx, torch.from_numpy(S).to(ctx.device))
    for c in range(S.shape[0]):
        for n in range(1, 20):
            ref = O.minor_det(S[c], n)
            assert abs(got[c, n - 1] - ref) <= FP64_REL * abs(ref)


def test_warp_kernel_exact_ties_and_zero_pivots(ctx):
    """Exact ties and zero pivots: the identity (tau = 0 with plane-wave
    sources) and the all-ones matrix, where every row ties in every column
    and every pivot after the first is an exact zero -- the last-row tie
    rule and ludcmp's 1e-20 substitute decide sign and size."""
    for M in (np.eye(19, dtype=np.complex128), np.ones((19, 19), dtype=np.complex128)):
        got = _dets(ctx, torch.from_numpy(M.reshape(1, 19, 19)).to(ctx.device))[0]
        ref = np.array([O.minor_det(M, n) for n in range(1, 20)])
        assert np.allclose(got, ref, rtol=FP64_REL, atol=0.0)


def test_warp_kernel_large_batch(ctx):
    S = torch.from_numpy(_random(4096, 19, 9)).to(ctx.device)
    a = _dets(ctx, S, warp=1)
    b = _dets(ctx, S, warp=0)
    assert np.max(np.abs(a - b) / np.abs(b)) < FP64_REL

"""The non-allocating determinant entry point, checked against the regular one.

nrcps_slater_dets_noalloc exists for callers that must not have the library
allocate device memory (a host whose memory pool already owns the device, or
measurement between already-queued kernels).  For N <= 64 it runs the
warp-per-minor kernel, which needs no working memory at all; for N > 64 it
draws its working memory from a fixed 16 MiB array inside the library.  This
file is collected last so that a failure here never hides the other GPU
tests.
"""
import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

nb = pytest.importorskip("nrcps_b200")
from nrcps_b200 import _capi as C  # noqa: E402

TOL = 1e-12  # the FP64 determinant tolerance of the parity tests


def _call(fn, ctx, S, psi1, N, nconf, mode, out):
    p1 = ctypes.c_void_p(psi1.data_ptr()) if psi1 is not None else None
    return fn(ctx.handle, ctypes.c_void_p(S.data_ptr()), p1, N, nconf, mode, 0, ctypes.c_void_p(out.data_ptr()))


def _inputs(rs, nconf, N, mode, device):
    S = rs.standard_normal((nconf, N, N)) + 1j * rs.standard_normal((nconf, N, N))
    P1 = rs.standard_normal((nconf, N, N)) + 1j * rs.standard_normal((nconf, N, N))
    return torch.from_numpy(S).to(device), (torch.from_numpy(P1).to(device) if mode else None)


# (N, configurations, mode): the warp kernel (N <= 64) at small and at the
# batched workload's N = 19, and the fixed-array kernel (N > 64) up to a batch
# just under the array's 16 MiB (N = 65, 3 matrices: 13.3 MB)
@pytest.mark.parametrize("N,nconf,mode", [(9, 17, 0), (9, 17, 1), (19, 64, 0), (19, 64, 1), (66, 1, 1), (65, 3, 0)])
def test_noalloc_matches_allocating_entry_point_twice(N, nconf, mode):
    ctx = nb.Context(0)
    L = nb.lib()
    rs = np.random.default_rng(11 + mode + N)
    nmeas = 2 * N if mode else N
    for call in range(2):  # two calls in a row share (and reuse) the fixed array
        S_d, P1_d = _inputs(rs, nconf, N, mode, ctx.device)
        ref = torch.empty((nconf, nmeas), dtype=torch.complex128, device=ctx.device)
        got = torch.full((nconf, nmeas), float("nan"), dtype=torch.complex128, device=ctx.device)
        assert _call(L.nrcps_slater_dets, ctx, S_d, P1_d, N, nconf, mode, ref) == C.OK
        st = _call(L.nrcps_slater_dets_noalloc, ctx, S_d, P1_d, N, nconf, mode, got)
        assert st == C.OK, L.nrcps_last_error(ctx.handle)
        torch.cuda.synchronize()
        r, g = ref.cpu().numpy(), got.cpu().numpy()
        assert np.all(np.abs(g - r) <= TOL * np.abs(r)), call
    ctx.close()


def test_noalloc_rejects_batches_beyond_its_fixed_array():
    ctx = nb.Context(0)
    L = nb.lib()
    N, nconf = 80, 3  # 3 * 80 * (2*6400 + 80) doubles = 24.7 MB > 16 MiB
    S = torch.zeros((1, N, N), dtype=torch.complex128, device=ctx.device)
    out = torch.zeros((1, N), dtype=torch.complex128, device=ctx.device)
    st = _call(L.nrcps_slater_dets_noalloc, ctx, S, None, N, nconf, 0, out)
    assert st == 1  # NRCPS_ERR_INVALID_ARGUMENT
    assert b"fixed" in L.nrcps_last_error(ctx.handle)
    ctx.close()


def test_noalloc_empty_batch_is_a_no_op():
    """An empty batch (a torch tensor with no elements has a null data
    pointer) succeeds without touching any buffer, as nrcps_slater_dets does."""
    ctx = nb.Context(0)
    L = nb.lib()
    for mode in (0, 1):
        assert L.nrcps_slater_dets_noalloc(ctx.handle, None, None, 19, 0, mode, 0, None) == C.OK
        assert L.nrcps_slater_dets_noalloc(ctx.handle, None, None, 80, 0, mode, 0, None) == C.OK
    ctx.close()


def test_noalloc_leaves_device_memory_alone():
    """After the first call on the device (which loads the library's module
    and looks up the fixed array), further calls change the device's free
    memory by nothing, for both kernels -- while the allocating entry point
    grows its context's working memory for the same N > 64 batch."""
    ctx = nb.Context(0)
    L = nb.lib()
    rs = np.random.default_rng(5)
    cases = [(19, 64, 1), (65, 3, 0)]
    bufs = []
    for N, nconf, mode in cases:
        S_d, P1_d = _inputs(rs, nconf, N, mode, ctx.device)
        out = torch.empty((nconf, 2 * N if mode else N), dtype=torch.complex128, device=ctx.device)
        bufs.append((N, nconf, mode, S_d, P1_d, out))
    for N, nconf, mode, S_d, P1_d, out in bufs:  # set-up calls
        assert _call(L.nrcps_slater_dets_noalloc, ctx, S_d, P1_d, N, nconf, mode, out) == C.OK
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info(ctx.device)
    for _ in range(3):
        for N, nconf, mode, S_d, P1_d, out in bufs:
            assert _call(L.nrcps_slater_dets_noalloc, ctx, S_d, P1_d, N, nconf, mode, out) == C.OK
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info(ctx.device)
    assert free1 == free0
    N, nconf, mode, S_d, P1_d, out = bufs[1]
    assert _call(L.nrcps_slater_dets, ctx, S_d, P1_d, N, nconf, mode, out) == C.OK
    torch.cuda.synchronize()
    free2, _ = torch.cuda.mem_get_info(ctx.device)
    assert free2 < free1  # the context's scratch: the measurement sees an allocation
    ctx.close()

"""The non-allocating determinant entry point, checked against the regular one.

nrcps_slater_dets_noalloc exists for callers that must not have the library
allocate device memory (a host whose memory pool already owns the device, or
measurement between already-queued kernels); it draws its working memory
from a fixed array inside the library.  This file is collected last so that
a failure here never hides the other GPU tests.
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


@pytest.mark.parametrize("mode", [0, 1])
def test_noalloc_matches_allocating_entry_point_twice(mode):
    ctx = nb.Context(0)
    L = nb.lib()
    rs = np.random.default_rng(11 + mode)
    N, nconf = 9, 17
    nmeas = 2 * N if mode else N
    for call in range(2):  # two calls in a row share (and reuse) the fixed array
        S = rs.standard_normal((nconf, N, N)) + 1j * rs.standard_normal((nconf, N, N))
        P1 = rs.standard_normal((nconf, N, N)) + 1j * rs.standard_normal((nconf, N, N))
        S_d = torch.from_numpy(S).to(ctx.device)
        P1_d = torch.from_numpy(P1).to(ctx.device) if mode else None
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
    N, nconf = 40, 200  # 200 * 40 * (2*1600 + 40) doubles > 16 MiB
    S = torch.zeros((1, N, N), dtype=torch.complex128, device=ctx.device)
    out = torch.zeros((1, N), dtype=torch.complex128, device=ctx.device)
    st = _call(L.nrcps_slater_dets_noalloc, ctx, S, None, N, nconf, 0, out)
    assert st == 1  # NRCPS_ERR_INVALID_ARGUMENT
    assert b"fixed" in L.nrcps_last_error(ctx.handle)
    ctx.close()

"""CholeskyQR re-orthonormalisation (nrcps_reorthonormalise) against numpy:
after the call every configuration's orbitals are orthonormal and the
accumulated log R_ii reproduce the Gram determinant of the input,
log det(Psi^H Psi) = 2 sum_i log R_ii.  Covers the register-blocked FP32
Gram kernel (N <= 20), the general tiled kernels (N = 33, FP64) and a
ragged site count."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("N,L,prec", [(19, 16, "f32"), (7, 8, "f32"), (20, 12, "f32"), (33, 8, "f32"),
                                      (19, 16, "f64"), (5, 6, "f64")])
def test_reorthonormalise_against_numpy(N, L, prec):
    import nrcps_b200 as nb
    ctx = nb.default_context()
    nconf, V = 3, L ** 3
    rs = np.random.default_rng(N * 100 + L)
    a = rs.standard_normal((nconf, N, V)) + 1j * rs.standard_normal((nconf, N, V))
    a[:, 1:] += 0.9 * a[:, :1]          # correlated orbitals: a conditioned but not trivial Gram matrix
    a *= np.exp(rs.uniform(-3, 3, (nconf, N, 1)))
    dt = torch.complex64 if prec == "f32" else torch.complex128
    psi = torch.from_numpy(a).to(dt).to(ctx.device).contiguous()
    ref = psi.cpu().numpy().astype(np.complex128)
    logR = nb.reorthonormalise(psi, ctx=ctx)
    ctx.synchronize()
    q = psi.cpu().numpy().astype(np.complex128)
    tol_orth = 5e-5 if prec == "f32" else 1e-12
    tol_det = 1e-5 if prec == "f32" else 1e-12
    for c in range(nconf):
        g = q[c].conj() @ q[c].T
        assert np.abs(g - np.eye(N)).max() < tol_orth, c
        want = np.linalg.slogdet(ref[c].conj() @ ref[c].T)[1]
        got = 2 * logR[c].sum().item()
        assert abs(got - want) <= tol_det * abs(want) + tol_det, c


@pytest.mark.parametrize("N,L,nconf", [(19, 32, 5), (10, 48, 2), (32, 16, 4), (1, 8, 9)])
def test_tensor_core_gram_against_cuda_cores(N, L, nconf):
    """The Gram matrices on the tcgen05 tensor cores (TF32 hi/lo, option
    "qr.gram_tc" for FP32 orbitals with N <= 32) against the CUDA-core kernel
    (the default), through a
    whole re-orthonormalisation: the same log R_ii to 2e-5 (FP32 sums over
    2V floats either way) and orthonormal orbitals to the FP32 tolerance of
    the test above (odd configuration counts leave the last tile half
    empty)."""
    import nrcps_b200 as nb
    ctx = nb.default_context()
    V = L ** 3
    rs = np.random.default_rng(N + L)
    a = rs.standard_normal((nconf, N, V)) + 1j * rs.standard_normal((nconf, N, V))
    if N > 1:
        a[:, 1:] += 0.5 * a[:, :1]
    psi0 = torch.from_numpy(a).to(torch.complex64).to(ctx.device).contiguous()
    out = {}
    try:
        for tc in (1, 0):
            ctx.set_option("qr.gram_tc", tc)
            psi = psi0.clone()
            logR = nb.reorthonormalise(psi, ctx=ctx)
            ctx.synchronize()
            out[tc] = (logR.cpu().numpy(), psi.cpu().numpy().astype(np.complex128))
    finally:
        ctx.set_option("qr.gram_tc", 0)
    assert np.max(np.abs(out[1][0] - out[0][0]) / np.maximum(np.abs(out[0][0]), 1.0)) < 2e-5
    for c in range(nconf):
        q = out[1][1][c]
        assert np.abs(q.conj() @ q.T - np.eye(N)).max() < 5e-5, c

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

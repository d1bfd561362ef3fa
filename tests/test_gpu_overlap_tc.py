"""The tensor-core Slater overlap (tcgen05, TF32 hi/lo split, FP32
accumulation) against the FP64 overlap of the same FP32 orbitals.

S[c][s][t] = sum_p conj(src_s(p)) psi_{c,t}(p) (OneBody::Project,
src/one_body/noarch/one_body_project.C:14-27).  Tolerance: 1e-6 of the
largest |S| (the split carries ~22 mantissa bits per operand and the
accumulator is FP32), well inside the 1e-5 FP32-mode target on correlators.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

nb = pytest.importorskip("nrcps_b200")

TC_REL = 1e-6


@pytest.fixture(scope="module")
def ctx():
    return nb.default_context()


def _inputs(L, ns, nt, nconf, seed):
    rs = np.random.default_rng(seed)
    vol = L ** 3
    src = (rs.standard_normal((ns, vol)) + 1j * rs.standard_normal((ns, vol))) / np.sqrt(vol)
    psi = (rs.standard_normal((nconf, nt, vol)) + 1j * rs.standard_normal((nconf, nt, vol))).astype(np.complex64)
    return src, psi


def _overlaps(ctx, src, psi, tc):
    ctx.set_option("overlap.tc", 1 if tc else 0)
    try:
        S = nb.overlap(torch.from_numpy(src).to(ctx.device), torch.from_numpy(psi).to(ctx.device), ctx)
        ctx.synchronize()
        return S.cpu().numpy()
    finally:
        ctx.set_option("overlap.tc", 1)


@pytest.mark.parametrize("L,ns,nt,nconf", [(8, 7, 7, 3), (16, 19, 19, 4), (16, 33, 19, 2), (32, 10, 10, 3),
                                           (24, 19, 5, 40)])
def test_tc_overlap_matches_fp64_reference(ctx, L, ns, nt, nconf):
    src, psi = _inputs(L, ns, nt, nconf, seed=L + ns)
    got = _overlaps(ctx, src, psi, tc=True)
    ref = np.einsum("sp,ctp->cst", src.conj(), psi.astype(np.complex128))
    assert np.max(np.abs(got - ref)) / np.max(np.abs(ref)) < TC_REL


def test_tc_overlap_agrees_with_cuda_core_kernel_large_batch(ctx):
    """A batch large enough that K is not split over CTAs (plain stores)."""
    L, ns, nt, nconf = 16, 19, 19, 2100
    g = torch.Generator(device=ctx.device).manual_seed(11)
    src = torch.randn((ns, L ** 3), dtype=torch.complex128, device=ctx.device, generator=g) / L ** 1.5
    psi = torch.randn((nconf, nt, L ** 3), dtype=torch.complex64, device=ctx.device, generator=g)
    out = []
    for tc in (1, 0):
        ctx.set_option("overlap.tc", tc)
        out.append(nb.overlap(src, psi, ctx))
    ctx.set_option("overlap.tc", 1)
    ctx.synchronize()
    err = (out[0] - out[1]).abs().max() / out[1].abs().max()
    assert float(err) < TC_REL


def test_tc_overlap_two_calls_in_a_row_agree_bitwise(ctx):
    src, psi = _inputs(16, 19, 19, 3, seed=12)
    a = _overlaps(ctx, src, psi, tc=True)
    b = _overlaps(ctx, src, psi, tc=True)
    # the split-K sums are atomic, so the order of the partial sums may vary
    assert np.max(np.abs(a - b)) / np.max(np.abs(a)) < 1e-12


def test_tc_overlap_in_the_ensemble_matches_fp64(ctx):
    """Dense (non-plane-wave) sources through the graph-captured ensemble:
    FP32 orbitals with the tensor-core overlap against the FP64 run."""
    L, T, n_conf = 8, 6, 4
    dims = (L, L, L)
    idx, _, _ = nb.momenta(dims, "PERFECT", 1.0, 0.35, 2.0)
    n = len(idx)
    rs = np.random.default_rng(3)
    # plane waves mixed by a random unitary: a dense source set with the same span
    q, _ = np.linalg.qr(rs.standard_normal((n, n)) + 1j * rs.standard_normal((n, n)))
    pw = np.zeros((n, L ** 3), dtype=np.complex128)
    pw[np.arange(n), idx] = 1.0
    src = q @ pw
    out = {}
    for prec in ("f64", "f32"):
        job = nb.EnsembleJob(L=L, T=T, n_conf=n_conf, seed=99, precision=prec, fermi_energy=0.35)
        ens = nb.Ensemble(job, sources=src, ctx=ctx)
        out[prec] = ens.run(0).cpu().numpy()
        ens.close()
    rel = np.max(np.abs(out["f32"] - out["f64"]) / np.abs(out["f64"]))
    assert rel < 1e-5

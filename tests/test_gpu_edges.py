"""Edge cases a caller of the reference's classes can reach.

Empty batches are no-ops (an empty torch tensor has a null data pointer, so
the C ABI accepts null buffers when the count is zero); lattice extents the
reference's FFTW path would take but this library does not implement, and
malformed arguments, come back as a status with a message (the reference
would call ERR.General and exit, src/utils/error.C:36-46); the context stays
usable after an error.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    import nrcps_b200 as nb
    return nb.default_context()


def _kinv(L, dev):
    """k = 1/xi (Kinetic::Evolve divides by xi)."""
    import nrcps_b200 as nb
    return torch.from_numpy(np.ascontiguousarray(1.0 / nb.kinetic_table((L, L, L)))).to(dev)


def test_empty_batches_are_no_ops(ctx):
    import nrcps_b200 as nb
    from nrcps_b200 import cv
    dev = ctx.device
    L = 16
    bits = torch.zeros(L ** 3 // 32, dtype=torch.int32, device=dev)
    for dt in (torch.complex64, torch.complex128):
        psi = torch.empty((0, L, L, L), dtype=dt, device=dev)
        nb.propagate(psi, 7, _kinv(L, dev), bits, 0.5, ctx=ctx)
    f = nb.Fourier(0, (L, L, L), "f64", ctx)
    f.forward()
    f.backward()
    src = torch.zeros((7, L ** 3), dtype=torch.complex128, device=dev)
    assert nb.overlap(src, torch.empty((0, 7, L ** 3), dtype=torch.complex64, device=dev), ctx).shape == (0, 7, 7)
    assert nb.overlap_planewave(np.arange(7), torch.empty((0, 7, L ** 3), dtype=torch.complex128, device=dev),
                                ctx).shape == (0, 7, 7)
    assert nb.slater_dets(torch.empty((0, 7, 7), dtype=torch.complex128, device=dev), ctx=ctx).shape == (0, 7)
    corr, z = nb.accumulate(torch.empty((0, 4, 7), dtype=torch.complex128, device=dev), n_cumulants=2, ctx=ctx)
    assert torch.count_nonzero(corr).item() == 0 and torch.count_nonzero(z).item() == 0
    assert nb.draw_z2_bits("RANLXS2", 1, 0, 0, ctx).numel() == 0
    assert cv.sample_z2_features(1, 0, 32, 64, 8, 0, ctx).shape == (0, 64, 512)
    ctx.synchronize()


@pytest.mark.parametrize("L", [10, 20, 40])
def test_unsupported_extent_is_a_status_and_the_context_survives(ctx, L):
    """Extents with a prime factor above 3 (FFTW handles them, this library's
    register DFTs do not): UNSUPPORTED with the supported list, then a valid
    call on the same context."""
    import nrcps_b200 as nb
    from nrcps_b200._capi import NrcpsError
    dev = ctx.device
    psi = torch.zeros((2, L, L, L), dtype=torch.complex64, device=dev)
    bits = torch.zeros((L ** 3 + 31) // 32, dtype=torch.int32, device=dev)
    with pytest.raises(NrcpsError, match="UNSUPPORTED"):
        nb.propagate(psi, 2, torch.ones(L ** 3, dtype=torch.float64, device=dev), bits, 0.5, ctx=ctx)
    f = nb.Fourier(1, (L, L, L), "f64", ctx)
    with pytest.raises(NrcpsError, match="not supported"):
        f.forward()
    q = torch.zeros((2, 16, 16, 16), dtype=torch.complex64, device=dev)
    q[:, 0, 0, 0] = 1
    nb.propagate(q, 2, _kinv(16, dev), torch.zeros(128, dtype=torch.int32, device=dev), 0.5, ctx=ctx)
    ctx.synchronize()
    assert torch.isfinite(torch.view_as_real(q)).all()


def test_bad_arguments_are_statuses(ctx):
    import nrcps_b200 as nb
    from nrcps_b200 import cv
    from nrcps_b200._capi import NrcpsError
    dev = ctx.device
    with pytest.raises(NrcpsError, match="INVALID_ARGUMENT"):
        ctx.set_option("fused.kind", 13)
    with pytest.raises(NrcpsError, match="INVALID_ARGUMENT"):
        ctx.set_option("no.such.option", 1)
    bits = torch.zeros(1024, dtype=torch.int32, device=dev)
    with pytest.raises(NrcpsError, match="G must divide L"):
        cv.coarse_fields(bits, 0, 16, 2, 5, 1, ctx)
    with pytest.raises(NrcpsError, match="INVALID_ARGUMENT"):
        nb.jackknife(torch.zeros((3, 4), dtype=torch.float64, device=dev), 8, ctx=ctx)
    net = cv.ControlVariateNet(cv.NetShape(T=12, G=8), ctx=ctx)  # T not a multiple of 16
    assert not net.tc_inference_supported()
    y = net.infer(torch.zeros((2, 12, 512), dtype=torch.bfloat16, device=dev))  # the layer-by-layer kernels
    assert y.shape == (2, 12)
    ctx.synchronize()

"""Learned control variate: the network's kernels against the CPU reference
(forward and every gradient), training, and the estimator it serves.

CPU: the reference's analytic gradients against central finite differences
(FP64).  GPU: forward and gradients of the BF16 device kernels against the
reference with the same BF16 roundings (5e-3 of each tensor's norm: the
device accumulates in FP32); a short training run lowers the loss; on a small
ensemble the control-variate estimator agrees with the plain one within the
errors and has a smaller variance per configuration.
"""
import numpy as np
import pytest

from oracle import cvnet as R


def _params(T, C=16, H=32, seed=0):
    rs = np.random.default_rng(seed)
    p = {}
    p["w1"] = rs.standard_normal((C, T, 27)) / np.sqrt(T * 27)
    p["w2"] = rs.standard_normal((C, C, 27)) / np.sqrt(C * 27)
    p["w3"] = rs.standard_normal((C, C, 27)) / np.sqrt(C * 27)
    for i in (1, 2, 3):
        p[f"b{i}"] = 0.1 * rs.standard_normal(C)
    p["hw"] = rs.standard_normal((H, C)) / np.sqrt(C)
    p["hb"] = 0.1 * rs.standard_normal(H)
    p["ow"] = rs.standard_normal((T, H)) / np.sqrt(H)
    p["ob"] = 0.1 * rs.standard_normal(T)
    return {k: v.astype(np.float32).astype(np.float64) for k, v in p.items()}


def test_reference_gradients_match_finite_differences():
    T, G, B = 3, 4, 2
    rs = np.random.default_rng(1)
    p = _params(T, C=16, H=8, seed=2)
    x = rs.uniform(-1, 1, (B, T, G ** 3))
    tgt = rs.standard_normal((B, T))
    loss, _, g = R.loss_and_grads(p, x, tgt, G, bf16=False)
    for name, idx in (("w1", (3, 1, 13)), ("w2", (0, 5, 26)), ("w3", (7, 7, 0)), ("b2", (4,)), ("hw", (2, 9)),
                      ("ob", (1,))):
        h = 1e-6
        pp = {k: v.copy() for k, v in p.items()}
        pm = {k: v.copy() for k, v in p.items()}
        pp[name][idx] += h
        pm[name][idx] -= h
        fd = (R.loss_and_grads(pp, x, tgt, G, bf16=False)[0] - R.loss_and_grads(pm, x, tgt, G, bf16=False)[0]) / (2 * h)
        assert abs(fd - g[name][idx]) <= 1e-6 * max(1.0, abs(fd)), name


def _norm_err(a, b):
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.mark.gpu
def test_device_forward_and_gradients_match_reference():
    import torch
    import nrcps_b200 as nb
    from nrcps_b200.cv import ControlVariateNet, NetShape
    ctx = nb.default_context()
    T, G, B = 12, 8, 6
    net = ControlVariateNet(NetShape(T=T, G=G), seed=3, ctx=ctx)
    p = {k: v.cpu().numpy().astype(np.float64) for k, v in net.params.items()}
    rs = np.random.default_rng(4)
    x32 = rs.uniform(-1, 1, (B, T, G ** 3)).astype(np.float32)
    x = torch.from_numpy(x32).to(torch.bfloat16).to(ctx.device)
    xr = x.float().cpu().numpy().astype(np.float64)
    tgt = rs.standard_normal((B, T)).astype(np.float32)
    y = net.forward(x).cpu().numpy()
    loss = net.backward(x, torch.from_numpy(tgt).to(ctx.device))
    ctx.synchronize()
    rloss, ry, rg = R.loss_and_grads(p, xr, tgt.astype(np.float64), G, bf16=True)
    assert _norm_err(y, ry) < 5e-3
    assert abs(loss - rloss) <= 5e-3 * abs(rloss)
    for k in rg:
        assert _norm_err(net.grads[k].cpu().numpy(), rg[k]) < 5e-3, k


@pytest.mark.gpu
def test_run_field_bits_are_the_stream_window():
    """nrcps_ensemble_field_bits: after a run at configuration c0 the
    ensemble's bits are the RANLXS2 window of configurations c0.. (the
    control variate takes its features from them): the same words as a fresh
    draw of that window, and the same block means."""
    import torch
    import nrcps_b200 as nb
    from nrcps_b200 import cv
    ctx = nb.default_context()
    L, T, m, seed, c0 = 8, 6, 5, 1234, 7
    V = L ** 3
    idx, _, _ = nb.momenta((L,) * 3, "PERFECT", 1.0, 0.35, 2.0)
    ens = nb.Ensemble(nb.EnsembleJob(L=L, T=T, n_conf=m, seed=seed, precision="f64", fermi_energy=0.35),
                      plane_wave_index=idx, ctx=ctx)
    try:
        ens.run(c0)
        ptr = ens.field_bits_ptr()
        assert ptr
        ref = nb.draw_z2_bits("RANLXS2", seed, c0 * T * V, m * T * V, ctx)
        nwords = (m * T * V) // 32

        class _Words:  # the ensemble's device words as a tensor view
            __cuda_array_interface__ = {"shape": (nwords,), "typestr": "<i4", "data": (ptr, False), "version": 3}

        got = torch.as_tensor(_Words(), device=ctx.device)
        assert torch.equal(got, ref.view(torch.int32)[:nwords])
        xa = cv.coarse_fields(ptr, 0, L, T, 4, m, ctx)
        xb = cv.coarse_fields(ref, 0, L, T, 4, m, ctx)
        assert torch.equal(xa, xb)
    finally:
        ens.close()


@pytest.mark.gpu
def test_training_and_control_variate_on_a_small_ensemble():
    """L=8, T=12, N=7, Z2 a=0.5: train on 3072 configurations, calibrate c on
    1024 more, estimate <C_N(tau)> from 2048 fresh configurations with <g> from
    16384 extra field draws.  The control variate must cut the per-sample
    variance and agree with the plain estimator within 4 sigma."""
    import torch
    import nrcps_b200 as nb
    from nrcps_b200 import cv
    ctx = nb.default_context()
    L, T, ef, seed = 8, 12, 0.35, 1000
    X, C = cv.generate_pairs(L, T, ef, seed, 6144, chunk=2048, G=4, precision="f64", qr_period=0, ctx=ctx)
    net = cv.ControlVariateNet(cv.NetShape(T=T, G=4), seed=0, ctx=ctx)
    losses = net.fit(X[:3072], torch.log(C[:3072]), epochs=8, batch=128, lr=3e-3)
    assert losses[-1] < 0.7 * losses[0]
    g_cal = torch.exp(net.predict_logC(X[3072:4096]))
    c = cv.cv_coefficient(C[3072:4096].cpu(), g_cal)
    g_eval = torch.exp(net.predict_logC(X[4096:]))
    gm, gm_err, _ = cv.extra_fields_mean_g(net, L, seed, 100000, 16384, chunk=4096, ctx=ctx)
    plain, plain_err, est, est_err = cv.estimators(C[4096:].cpu(), g_eval, c, gm, gm_err)
    var_ratio = ((C[4096:].cpu() - c * g_eval).var(0) / C[4096:].cpu().var(0))[1:]
    assert float(var_ratio.median()) < 0.5
    z = (est - plain).abs() / (plain_err ** 2 + est_err ** 2).sqrt()
    assert float(z[1:].max()) < 4.0


@pytest.mark.gpu
@pytest.mark.parametrize("L,G", [(32, 8), (16, 4), (8, 4)])
def test_coarse_field_block_means(L, G):
    """Block means of the Z2 field against numpy (the word-at-a-time kernel
    at L = 32, the per-site kernel otherwise)."""
    import torch
    import nrcps_b200 as nb
    from nrcps_b200 import cv
    ctx = nb.default_context()
    B, T = 2, 3
    bits = nb.draw_z2_bits("RANLXS2", 17, 0, B * T * L ** 3, ctx)
    got = cv.coarse_fields(bits, 0, L, T, G, B, ctx).float().cpu().numpy()
    w = bits.cpu().numpy().astype(np.uint32)
    allbits = np.unpackbits(w.view(np.uint8), bitorder="little")[: B * T * L ** 3].astype(np.float64)
    phi = (2 * allbits - 1).reshape(B, T, L, L, L)
    f = L // G
    ref = phi.reshape(B, T, G, f, G, f, G, f).mean(axis=(3, 5, 7)).reshape(B, T, G ** 3)
    assert np.array_equal(got, ref.astype(np.float32).astype(np.float64))


def test_philox_known_answers():
    """The oracle's Philox4x32-10 against the published known-answer vectors."""
    from oracle import philox
    for ctr, key, want in philox.PHILOX_KATS:
        got = philox.philox4x32_10(*[np.uint32(c) for c in ctr], np.uint32(key[0]), np.uint32(key[1]))
        assert tuple(int(v) for v in got) == want


def test_sampled_features_have_the_block_mean_distribution():
    """Oracle features at L=8, G=4 (8 sites per cell): the counts are
    Binomial(8, 1/2) (chi-square over the 9 values)."""
    from math import comb
    from oracle import philox
    x = philox.z2_block_features(5, 0, 8, 16, 4, 64)
    c = np.rint((x.ravel() * 8 + 8) / 2).astype(int)
    obs = np.bincount(c, minlength=9)
    exp = np.array([comb(8, k) for k in range(9)]) / 256.0 * c.size
    chi2 = float(((obs - exp) ** 2 / exp).sum())
    assert chi2 < 30.0  # 8 degrees of freedom: p ~ 2e-4


@pytest.mark.gpu
@pytest.mark.parametrize("L,G,T,B,first", [(32, 8, 8, 6, 0), (8, 4, 5, 7, 3), (24, 8, 3, 4, 11), (48, 8, 2, 3, 1 << 33)])
def test_device_feature_sampler_matches_oracle(L, G, T, B, first):
    """nrcps_cv_sample_z2_features bit-exact against the oracle (1, 8, 27
    and 216 bits per cell; a field number above 2^32)."""
    import nrcps_b200 as nb
    from nrcps_b200 import cv
    from oracle import philox
    ctx = nb.default_context()
    seed = (7 << 32) | 3000
    got = cv.sample_z2_features(seed, first, L, T, G, B, ctx).float().cpu().numpy()
    want = philox.z2_block_features(seed, first, L, T, G, B)
    assert np.array_equal(got.astype(np.float64), want)


@pytest.mark.gpu
def test_sampled_features_match_coarse_grained_ranlux_fields():
    """The direct draws and the block means of RANLXS2 fields have the same
    distribution at L=32, G=8 (per-cell mean and variance of 4096 x 8 x 512
    values each; variance 1/64 for both)."""
    import nrcps_b200 as nb
    from nrcps_b200 import cv
    ctx = nb.default_context()
    L, T, G, B = 32, 8, 8, 4096
    a = cv.sample_z2_features(11, 0, L, T, G, B, ctx).double()
    bits = nb.draw_z2_bits("RANLXS2", 11, 0, B * T * L ** 3, ctx)
    b = cv.coarse_fields(bits, 0, L, T, G, B, ctx).double()
    n = a.numel()
    for v in (a, b):
        assert abs(float(v.mean())) < 5 * (1 / 64 / n) ** 0.5
        assert abs(float(v.var()) - 1 / 64) < 5 * (2 / 64 ** 2 / n) ** 0.5
    assert set(torch_unique(a)) <= {k / 32 for k in range(-32, 33)}


def torch_unique(t):
    return [float(v) for v in t.unique().cpu()]


@pytest.mark.gpu
@pytest.mark.parametrize("T,B", [(64, 6), (16, 5), (48, 3), (32, 300)])
def test_tensor_core_inference_matches_reference(T, B):
    """nrcps_cv_forward_tc (the whole network in one tcgen05 kernel) against
    the CPU reference with the same BF16 roundings (5e-3 of the norm; FP32
    accumulation in another order) and against the layer-by-layer CUDA-core
    kernels; B = 300 runs several samples per CTA."""
    import torch
    import nrcps_b200 as nb
    from nrcps_b200.cv import ControlVariateNet, NetShape
    ctx = nb.default_context()
    net = ControlVariateNet(NetShape(T=T, G=8), seed=5, ctx=ctx)
    rs = np.random.default_rng(T + B)
    for k in ("b1", "b2", "b3", "hb", "ob"):  # non-zero biases
        net.params[k].copy_(torch.from_numpy(0.1 * rs.standard_normal(net.params[k].shape)).float())
    assert net.tc_inference_supported()
    x = torch.from_numpy(rs.uniform(-1, 1, (B, T, 512)).astype(np.float32)).to(torch.bfloat16).to(ctx.device)
    y_tc = net.infer(x).cpu().numpy().astype(np.float64)
    y_cc = net.forward(x).cpu().numpy().astype(np.float64)
    p = {k: v.cpu().numpy().astype(np.float64) for k, v in net.params.items()}
    n = min(B, 8)
    y_ref, _ = R.forward(p, x[:n].float().cpu().numpy().astype(np.float64), 8, bf16=True)
    assert _norm_err(y_tc[:n], y_ref) < 5e-3
    assert _norm_err(y_tc, y_cc) < 5e-3

"""Uneven batches: jobs of different L, N and T in one graph launch, fields
from one generator stream in job order.

CPU: the oracle's batch runner (o_run_batch) against the oracle's pinned
ensemble driver for one job, and the stream order across jobs.  GPU: the
device batch in FP64 against the oracle within 1e-12, and the FP32 batch at
the uneven-batch shapes against the FP64 batch.
"""
import numpy as np
import pytest

from oracle import oracle as O

FP64_REL = 1e-12


def _rel(a, b):
    """Relative error per (configuration, slice) row of determinants, against
    the row's largest magnitude (a leading minor can be pure cancellation)."""
    return np.max(np.max(np.abs(a - b), axis=-1) / np.max(np.abs(b), axis=-1))


def _pw(L, ef):
    idx, _, _ = O.momenta((L,) * 3, "PERFECT", 1.0, ef, (2 * O.PI) ** 2)
    return list(idx)


def test_oracle_batch_single_job_equals_ensemble_driver():
    """One Z2 job through o_run_batch (local factor (1 + a phi)/V) against
    o_run_ensemble (Interaction::Initialize with one coupling, a = c V)."""
    L, T = 8, 5
    dims = (L,) * 3
    itab = O.interaction_table(dims, 1.0, [0.019894367886486918], 1.0, (2 * O.PI) ** 2)
    a = float(itab[0] * L ** 3)
    idx = _pw(L, 0.35)
    (b,) = O.run_batch([(L, T, 2, idx)], "RANLXS2", 1234, "ZTWO", a)
    ref = O.run_ensemble(O.Job(L=L, T=T, configs=2, seed=1234), O.plane_wave_sources(dims, idx))
    # the ensemble driver draws one extra field after each configuration's last
    # slice (the reference's Refresh at the end of every slice); the batch does
    # not -- configuration 0 agrees exactly
    assert _rel(b[0], ref[0]) < 1e-13


def test_oracle_batch_stream_order():
    """Job 0's determinants do not depend on the jobs after it; job 1's fields
    continue the stream where job 0's ended."""
    j0, j1 = (8, 4, 1, _pw(8, 0.35)), (8, 3, 1, _pw(8, 0.12))
    alone = O.run_batch([j0], "RANLXS2", 7, "GAUSS", 0.3)
    both = O.run_batch([j0, j1], "RANLXS2", 7, "GAUSS", 0.3)
    assert np.array_equal(alone[0], both[0])
    swapped = O.run_batch([j1, j0], "RANLXS2", 7, "GAUSS", 0.3)
    assert not np.allclose(swapped[1], both[0])


_JOBS = [(8, 6, 2, 0.35), (16, 4, 1, 0.1), (8, 3, 3, 0.12), (16, 7, 1, 0.13), (8, 5, 1, 0.35)]


@pytest.mark.gpu
@pytest.mark.parametrize("field", ["GAUSS", "ZTWO"])
def test_device_batch_fp64_matches_oracle(field):
    import nrcps_b200 as nb
    ctx = nb.default_context()
    jobs = [nb.BatchJob(L=L, T=T, n_conf=c, fermi_energy=ef) for L, T, c, ef in _JOBS]
    b = nb.Batch(jobs, seed=99, field=field, a=0.3, precision="f64", ctx=ctx)
    got = [d.cpu().numpy() for d in b.run()]
    refs = O.run_batch([(L, T, c, _pw(L, ef)) for L, T, c, ef in _JOBS], "RANLXS2", 99, field, 0.3)
    for g, r in zip(got, refs):
        assert g.shape == r.shape
        assert _rel(g, r) < FP64_REL
    # the second run continues the stream: it equals the jobs run after a copy of themselves
    got2 = [d.cpu().numpy() for d in b.run()]
    refs2 = O.run_batch([(L, T, c, _pw(L, ef)) for L, T, c, ef in _JOBS] * 2, "RANLXS2", 99, field, 0.3)
    for g, r in zip(got2, refs2[len(_JOBS):]):
        assert _rel(g, r) < FP64_REL
    b.close()


@pytest.mark.gpu
def test_device_batch_uneven_shapes_fp32_vs_fp64():
    """Uneven shapes (L in 16, 24, 32; N in 7, 19, 33; T in 8, 16): FP32
    orbitals against the FP64 batch on the same stream, 1e-5 relative."""
    import nrcps_b200 as nb
    ctx = nb.default_context()
    shell = {7: 1.5, 19: 2.5, 33: 4.5}  # E_F between closed shells, units of (2 pi / L)^2 / 2
    spec = [(16, 8, 7), (24, 16, 19), (32, 8, 33), (16, 16, 19), (32, 16, 7)]
    jobs = [nb.BatchJob(L=L, T=T, n_conf=2, fermi_energy=0.5 * (2 * np.pi / L) ** 2 * shell[N]) for L, T, N in spec]
    out = {}
    for prec in ("f32", "f64"):
        b = nb.Batch(jobs, seed=99, field="GAUSS", a=0.3, precision=prec, qr_period=8 if prec == "f32" else 0,
                     ctx=ctx)
        out[prec] = [(np.abs(d.cpu().numpy()) ** 2).mean(0) for d in b.run()]
        b.close()
    for a, r in zip(out["f32"], out["f64"]):
        assert _rel(a, r) < 1e-5


@pytest.mark.gpu
def test_device_batch_fp32_vs_fp64_at_the_largest_uneven_shapes():
    """FP32 orbitals at the uneven workload's largest shapes -- L=48, N=33,
    T=128 and L=24, N=19, T=64, 8 configurations each, Gaussian fields
    a=0.3 -- against the FP64 batch on the same stream, both re-orthonormalised
    every 8 slices (the FP64 QR keeps every determinant exact and the long
    T=128 runs well conditioned): <|det S_m(tau)|^2> per minor and slice."""
    import nrcps_b200 as nb
    ctx = nb.default_context()
    shell = {19: 2.5, 33: 4.5}
    spec = [(48, 128, 33), (24, 64, 19)]
    jobs = [nb.BatchJob(L=L, T=T, n_conf=8, fermi_energy=0.5 * (2 * np.pi / L) ** 2 * shell[N]) for L, T, N in spec]
    out = {}
    for prec in ("f32", "f64"):
        b = nb.Batch(jobs, seed=99, field="GAUSS", a=0.3, precision=prec, qr_period=8, ctx=ctx)
        assert b.n_orb == [N for _, _, N in spec]
        out[prec] = [(np.abs(d.cpu().numpy()) ** 2).mean(0) for d in b.run()]
        b.close()
    for (L, T, N), a, r in zip(spec, out["f32"], out["f64"]):
        err = np.max(np.abs(a - r) / np.abs(r), axis=tuple(range(1, a.ndim)))
        print(f"L={L} N={N} T={T}: FP32 vs FP64 max rel err of <|det|^2> per tau: " +
              " ".join(f"{v:.1e}" for v in err))
        assert err.max() < 1e-4, (L, err.max())


@pytest.mark.gpu
def test_device_batch_fp64_at_the_largest_uneven_shapes(golden):
    """The uneven workload's largest shapes -- one L=48, N=33, T=128 job, one
    L=24, N=19, T=64 job and two L=16, N=7, T=32 configurations, Gaussian
    fields a=0.3 from RANLXS2 seed 99 -- as one device batch in FP64 against
    the oracle's batch runner (tests/golden/batch_large.npz), 1e-12."""
    import json
    import nrcps_b200 as nb
    ctx = nb.default_context()
    g = golden("batch_large.npz")
    args = json.loads(str(g["args"]))
    jobs = [nb.BatchJob(L=int(L), T=int(T), n_conf=int(c), fermi_energy=float(ef))
            for (L, T, c, _), ef in zip(g["jobs"], g["fermi_energies"])]
    b = nb.Batch(jobs, seed=int(args["seed"]), field=args["field"], a=float(args["a"]), precision="f64", ctx=ctx)
    assert b.n_orb == [int(n) for n in g["jobs"][:, 3]]
    got = [d.cpu().numpy() for d in b.run()]
    b.close()
    for i, d in enumerate(got):
        ref = g[f"dets{i}"]
        assert d.shape == ref.shape
        assert _rel(d, ref) < FP64_REL, (i, _rel(d, ref))


@pytest.mark.gpu
def test_device_batch_fp32_real_weight_table():
    """FP32 batches with a real Gaussian field step on one FP32 weight per
    site ("batch.real_weights" 1, the default), staged into shared memory by
    the st.async fused step (kind 11): the same determinants, bit for bit, as
    the kind-7 step reading the same table per site (L = 32, 48, the sizes
    with a kind-7 variant), and within 1e-5 of the step that forms
    (1 + a phi)/V per site from phi (option 0)."""
    import nrcps_b200 as nb
    ctx = nb.default_context()
    shell = {7: 1.5, 19: 2.5}
    spec = [(48, 6, 7), (32, 8, 19), (24, 5, 7), (16, 8, 19)]
    jobs = [nb.BatchJob(L=L, T=T, n_conf=2, fermi_energy=0.5 * (2 * np.pi / L) ** 2 * shell[N]) for L, T, N in spec]

    def run(kind, table):
        ctx.set_option("fused.kind", kind)
        ctx.set_option("batch.real_weights", table)
        try:
            b = nb.Batch(jobs, seed=99, field="GAUSS", a=0.3, precision="f32", ctx=ctx)
            out = [d.cpu().numpy() for d in b.run()]
            b.close()
        finally:
            ctx.set_option("fused.kind", -1)
            ctx.set_option("batch.real_weights", 1)
        return out

    staged, per_site, from_phi = run(11, 1), run(7, 1), run(11, 0)
    for (L, T, N), s, p, g in zip(spec, staged, per_site, from_phi):
        if L >= 32:
            assert np.array_equal(s, p), (L, N)
        assert _rel(s, g) < 1e-5, (L, N, _rel(s, g))


@pytest.mark.gpu
def test_device_batch_field_prefetch_is_the_same_stream():
    """"batch.prefetch_fields" 1 (the default) draws the next run's fields on a
    side stream during a run, into a second weight buffer: three consecutive
    runs give bit for bit the determinants of three runs that draw their own
    fields first (option 0)."""
    import nrcps_b200 as nb
    ctx = nb.default_context()
    shell = {7: 1.5, 19: 2.5}
    spec = [(32, 6, 19), (16, 9, 7), (24, 4, 7)]
    jobs = [nb.BatchJob(L=L, T=T, n_conf=2, fermi_energy=0.5 * (2 * np.pi / L) ** 2 * shell[N]) for L, T, N in spec]

    def runs(prefetch):
        ctx.set_option("batch.prefetch_fields", prefetch)
        try:
            b = nb.Batch(jobs, seed=31, field="GAUSS", a=0.3, precision="f32", ctx=ctx)
            out = [[d.cpu().numpy() for d in b.run()] for _ in range(3)]
            b.close()
        finally:
            ctx.set_option("batch.prefetch_fields", 1)
        return out

    with_prefetch, without = runs(1), runs(0)
    for r in range(3):
        for a, b in zip(with_prefetch[r], without[r]):
            assert np.array_equal(a, b), r
    assert not np.array_equal(with_prefetch[0][0], with_prefetch[1][0])


@pytest.mark.gpu
def test_device_batch_field_prefetch_with_other_draws_in_between():
    """While a prefetching batch's next fields are drawn on its side stream,
    the context draws another Gaussian field with another seed (the shared
    scratch and generator arguments): both the batch's next run and that
    draw are what they are without the overlap."""
    import torch
    import nrcps_b200 as nb
    ctx = nb.default_context()
    jobs = [nb.BatchJob(L=32, T=5, n_conf=3, fermi_energy=0.5 * (2 * np.pi / 32) ** 2 * 2.5),
            nb.BatchJob(L=16, T=7, n_conf=2, fermi_energy=0.5 * (2 * np.pi / 16) ** 2 * 1.5)]
    b = nb.Batch(jobs, seed=31, field="GAUSS", a=0.3, precision="f32", ctx=ctx)
    first = [d.cpu().numpy() for d in b.run()]
    other, _ = nb.draw_fields("RANLXS2", 77, "GAUSS", 32 ** 3, 40, 0, ctx)  # during the side draw
    second = [d.cpu().numpy() for d in b.run()]
    other = other.cpu()
    b.close()
    ctx.set_option("batch.prefetch_fields", 0)
    try:
        ref = nb.Batch(jobs, seed=31, field="GAUSS", a=0.3, precision="f32", ctx=ctx)
        want = [[d.cpu().numpy() for d in ref.run()] for _ in range(2)]
        ref.close()
    finally:
        ctx.set_option("batch.prefetch_fields", 1)
    for got, w in zip((first, second), want):
        for a, c in zip(got, w):
            assert np.array_equal(a, c)
    again, _ = nb.draw_fields("RANLXS2", 77, "GAUSS", 32 ** 3, 40, 0, ctx)
    assert torch.equal(other, again.cpu())

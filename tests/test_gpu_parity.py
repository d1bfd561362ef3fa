"""GPU parity: every hot-path operation of libnrcps_b200 against the oracle
(the CPU restatement pinned to the reference) on identical inputs.

Tolerances: RNG and field integers bit-exact; FP64 propagation, overlaps and
determinants within 1e-12 relative; FP32 propagation within 1e-5 relative on
the correlators (the accuracy target of the fast mode).
"""
import ctypes
import json
import os

import numpy as np
import pytest
import torch

from oracle import oracle as O

from conftest import GOLDEN

pytestmark = pytest.mark.gpu

nb = pytest.importorskip("nrcps_b200")
from nrcps_b200 import _capi as C  # noqa: E402

FP64_REL = 1e-12
FP32_REL = 1e-5


def rel_err(got, ref):
    got, ref = np.asarray(got), np.asarray(ref)
    return np.max(np.abs(got - ref) / np.maximum(np.abs(ref), 1e-300))


def max_norm_err(got, ref):
    got, ref = np.asarray(got), np.asarray(ref)
    return np.max(np.abs(got - ref)) / np.max(np.abs(ref))


@pytest.fixture(scope="module")
def ctx():
    return nb.default_context()


# ------------------------------------------------------------------ RNG
@pytest.mark.parametrize("kind", ["RANLXS0", "RANLXS1", "RANLXS2", "RANLXD1", "RANLXD2", "RAN2"])
def test_uniforms_bit_exact_vs_reference(golden, ctx, kind):
    g = golden("rng_streams.npz")
    assert np.array_equal(nb.uniforms(kind, 1234, 600, 0, ctx).cpu().numpy(), g[f"{kind}_seed1234_skip0"])
    assert np.array_equal(nb.uniforms(kind, 1234, 200, 200_000, ctx).cpu().numpy(),
                          g[f"{kind}_seed1234_skip200000"])


@pytest.mark.parametrize("kind", ["RANLXS2", "RANLXD1"])
def test_uniforms_bit_exact_long_windows(ctx, kind):
    rs = np.random.default_rng(3)
    for off in [0, 95, 96, 1, 4095, 77777, 1_000_003]:
        n = int(rs.integers(1, 50_000))
        got = nb.uniforms(kind, 4321, n, off, ctx).cpu().numpy()
        assert np.array_equal(got, O.uniforms(kind, 4321, n, skip=off)), off


def test_known_answer_on_device(golden, ctx):
    k = golden("ranlx_kat.npz")
    u = nb.uniforms("RANLXS0", 32767, 96, int(k["ranlxs0_seed32767_first_index"]), ctx).cpu().numpy()
    assert np.array_equal(u * 2.0 ** 24, k["ranlxs0_seed32767_times_2p24"])
    u = nb.uniforms("RANLXD1", 32767, 48, int(k["ranlxd1_seed32767_first_index"]), ctx).cpu().numpy()
    assert np.array_equal(u * 2.0 ** 48, k["ranlxd1_seed32767_times_2p48"])


def test_fields_bit_exact_vs_reference(golden, ctx):
    g = golden("fields.npz")
    for key in g.files:
        field, kind, seed, L = key.split("_")
        ref = g[key]
        got, off = nb.draw_fields(kind, int(seed[4:]), field, int(L[1:]) ** 3, ref.shape[0], 0, ctx)
        assert np.array_equal(got.cpu().numpy(), ref), key


@pytest.mark.parametrize("field", ["GAUSS", "COMPLEXGAUSS"])
def test_gauss_fields_stream_exact(ctx, field):
    """Uniform consumption is bit-exact; values agree to a few ulp (log on the device)."""
    vol, slices = 4096, 5
    got, off = nb.draw_fields("RANLXS2", 99, field, vol, slices, 0, ctx)
    r = O.Rng("RANLXS2", 99)
    ref = r.fields(field, vol, slices)
    assert np.max(np.abs(got.cpu().numpy() - ref)) <= 4e-15 * np.max(np.abs(ref))
    # the next slice continues from the same stream position
    nxt, _ = nb.draw_fields("RANLXS2", 99, field, vol, 1, off, ctx)
    assert np.max(np.abs(nxt.cpu().numpy()[0] - r.fields(field, vol, 1)[0])) < 1e-13


def test_gauss_fields_large_draw_is_one_stream(ctx):
    """A draw larger than one round of the Gaussian sampler (128 M candidate
    pairs, so this one takes two rounds and a host read of the consumed
    stream length between them) equals the same stream drawn slice by slice,
    and ends at the same stream position."""
    vol, slices = 48 ** 3, 1000  # 110.6 M values
    big, off = nb.draw_fields("RANLXS2", 5, "GAUSS", vol, slices, 0, ctx)
    pos = 0
    for t0 in range(0, slices, 250):
        part, pos = nb.draw_fields("RANLXS2", 5, "GAUSS", vol, 250, pos, ctx)
        assert torch.equal(part, big[t0:t0 + 250])
        del part
    assert pos == off
    del big


def test_z2_bits(ctx):
    first, count = 96 * 7 + 5, 100_000
    bits = nb.draw_z2_bits("RANLXS2", 11, first, count, ctx).cpu().numpy().view(np.uint32)
    u = O.uniforms("RANLXS2", 11, count, skip=first)
    want = (np.floor(2 * u) >= 1)
    got = ((bits[np.arange(count) >> 5] >> (np.arange(count) & 31)) & 1).astype(bool)
    assert np.array_equal(got, want)


# ------------------------------------------------------------------ FFT
@pytest.mark.parametrize("dims", [(4, 4, 4), (8, 6, 12), (16, 16, 16), (24, 24, 24), (32, 32, 32), (48, 16, 2)])
@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_fft3d_matches_numpy(ctx, dims, precision):
    rs = np.random.default_rng(5)
    a = rs.standard_normal((3,) + dims) + 1j * rs.standard_normal((3,) + dims)
    f = nb.Fourier(3, dims, precision, ctx)
    f.b.copy_(torch.from_numpy(a))
    f.forward()
    tol = 1e-13 if precision == "f64" else 2e-6
    assert max_norm_err(f.b.cpu().numpy(), np.fft.fftn(a, axes=(1, 2, 3))) < tol
    f.b.copy_(torch.from_numpy(a))
    f.backward()
    assert max_norm_err(f.b.cpu().numpy(), np.fft.ifftn(a, axes=(1, 2, 3)) * np.prod(dims)) < tol


# ---------------------------------------------------------- propagation
def _steps_reference(golden_name, golden):
    g = golden(golden_name)
    args = json.loads(str(g["args"]))
    return g, args


def test_class_api_steps_match_reference_props(golden, ctx):
    """Propagator::Run([K, I, K]) through the class API against the reference's
    own per-step orbitals (multi-coupling interaction, ranlxd fields drawn on
    the device)."""
    g, args = _steps_reference("ensemble_multicoupling.npz", golden)
    dims = (8, 8, 8)
    couplings = [float(c) for c in args["couplings"].split(",")]
    rng = nb.Random(args["rng"], int(args["seed"]))
    lat = nb.Lattice(dims, rng, "ZTWO", ctx)
    inter = nb.Interaction(lat, 1.0, couplings, 1.0, float(args["cutoff"]))
    kin = nb.Kinetic(dims, "PERFECT", 1.0, 0.5, float(args["cutoff"]), ctx)
    N = g["sources"].shape[0]
    prop = nb.Propagator(N, dims, "f64", ctx)
    for n in range(N):
        prop.set(g["sources"][n], n)
    for t in range(g["props"].shape[0]):
        got = prop.get().b.reshape(N, -1).cpu().numpy()
        assert max_norm_err(got, g["props"][t]) < FP64_REL, t
        for h in (kin, inter, kin):
            h.initialize()
        prop.run([kin, inter, kin])
        lat.refresh()


def test_potential_steps_match_oracle(ctx):
    dims = (8, 8, 8)
    pot = nb.Potential(dims, 0.005, 0.5, "EXP", ctx)
    kin = nb.Kinetic(dims, "PERFECT", 1.0, 0.5, 0.99999, ctx)
    rng = nb.Random("RANLXS2", 31)
    lat = nb.Lattice(dims, rng, "ZTWO", ctx)
    inter = nb.Interaction(lat, 1.0, [0.019894367886486918], 1.0, 0.99999)
    rs = np.random.default_rng(9)
    psi0 = rs.standard_normal((3, 512)) + 1j * rs.standard_normal((3, 512))
    prop = nb.Propagator(3, dims, "f64", ctx)
    for n in range(3):
        prop.set(psi0[n], n)
    ref = psi0.copy()
    xi = O.kinetic_xi(dims, "PERFECT", 1.0, 0.5, (0.99999 * O.PI) ** 2)
    potv = O.potential_table(dims, 0.005, 0.5, "EXP")
    itab = O.interaction_table(dims, 1.0, [0.019894367886486918], 1.0, (0.99999 * O.PI) ** 2)
    fields = O.field_slices("RANLXS2", 31, "ZTWO", 512, 4)
    for t in range(4):
        inter.initialize()
        prop.run([kin, pot, inter, pot, kin])
        lat.refresh()
        fld = O.interaction_initialize(dims, fields[t], itab)
        ref = O.kinetic_evolve(ref, xi)
        ref = O.potential_evolve(dims, ref, potv)
        ref = O.interaction_evolve(dims, ref, fld)
        ref = O.potential_evolve(dims, ref, potv)
        ref = O.kinetic_evolve(ref, xi)
        assert max_norm_err(prop.get().b.reshape(3, -1).cpu().numpy(), ref) < FP64_REL, t


# ---------------------------------------------------------- measurement
def test_overlap_pair_and_dets_match_oracle(golden, ctx):
    g = golden("ensemble_trapped.npz")
    src = g["sources"]
    N, vol = src.shape
    psi = g["props"][2]  # reference orbitals after two steps
    S = nb.overlap(torch.from_numpy(src).to(ctx.device), torch.from_numpy(psi).to(ctx.device).reshape(1, N, vol), ctx)
    S_ref = O.project(src, psi)
    assert rel_err(S.cpu().numpy()[0], S_ref) < FP64_REL
    w, opp = O.two_body_tables((8, 8, 8), "TGND", "STANDARD", 1.0, 0.176776695, (0.99999 * O.PI) ** 2)
    tb = nb.TwoBody((8, 8, 8), "TGND", "STANDARD", 1.0, 0.176776695, 0.99999, ctx)
    p = torch.from_numpy(psi).to(ctx.device).reshape(1, N, vol)
    phi = tb.run_matrix(p, p).cpu().numpy()[0]
    phi_ref = O.pair_matrix(psi, psi, w, opp)
    assert max_norm_err(phi, phi_ref) < FP64_REL
    dets = nb.slater_dets(torch.from_numpy(phi_ref).to(ctx.device).reshape(1, N, N),
                          torch.from_numpy(S_ref).to(ctx.device).reshape(1, N, N), mode=1, ctx=ctx).cpu().numpy()[0]
    for n in range(N):
        assert rel_err(dets[2 * n + 1], O.minor_det(phi_ref, n + 1)) < FP64_REL
        assert rel_err(dets[2 * n], O.minor_det(phi_ref, n + 1, t0=n, psi1=S_ref)) < FP64_REL


# (n, dims, configurations): one orbital, odd n, n = 32 (one 2 x 2 block per
# thread, no groups), n = 33 (the per-pair kernel), a volume that is not a
# whole number of tiles (6^3 = 216 sites) and more configurations than SMs
@pytest.mark.parametrize("n,dims,nconf", [(1, (8, 8, 8), 3), (7, (6, 6, 6), 5), (10, (12, 12, 12), 300),
                                          (19, (8, 8, 8), 2), (32, (8, 8, 8), 3), (33, (8, 8, 8), 2)])
def test_pair_matrix_tiles_match_oracle(ctx, n, dims, nconf):
    """TwoBody::Run (src/two_body/noarch/two_body_run.C:45-75) on random
    orbitals: the tiled cluster kernel (n <= 32) and the per-pair kernel
    against the oracle, FP64 within 1e-12 and FP32 orbitals within 1e-6 of
    the FP64 sums of the same (rounded) orbitals."""
    rs = np.random.default_rng(n + nconf)
    vol = int(np.prod(dims))
    psi1 = rs.standard_normal((nconf, n, vol)) + 1j * rs.standard_normal((nconf, n, vol))
    psi2 = rs.standard_normal((nconf, n, vol)) + 1j * rs.standard_normal((nconf, n, vol))
    tb = nb.TwoBody(dims, "TGND", "STANDARD", 1.0, 0.176776695, 0.99999, ctx)
    for c in sorted({0, nconf - 1}):
        ref = O.pair_matrix(psi1[c], psi2[c], tb.w_host, tb.opp_host)
        for tile in (1, 0):
            ctx.set_option("pair.tile", tile)
            try:
                for dt, tol in ((torch.complex128, FP64_REL), (torch.complex64, 1e-6)):
                    p1 = torch.from_numpy(psi1).to(ctx.device).to(dt)
                    p2 = torch.from_numpy(psi2).to(ctx.device).to(dt)
                    r = ref if dt == torch.complex128 else O.pair_matrix(
                        p1[c].cpu().numpy().astype(np.complex128), p2[c].cpu().numpy().astype(np.complex128),
                        tb.w_host, tb.opp_host)
                    phi = tb.run_matrix(p1, p2).cpu().numpy()[c]
                    assert max_norm_err(phi, r) < tol, (tile, dt)
            finally:
                ctx.set_option("pair.tile", 1)


@pytest.mark.parametrize("n,dims,nconf,even", [(1, (8, 8, 8), 3, True), (10, (12, 12, 12), 300, True),
                                               (19, (8, 8, 8), 2, True), (32, (8, 8, 8), 3, True),
                                               (10, (8, 8, 8), 3, False)])
def test_pair_matrix_of_one_set_of_orbitals(ctx, n, dims, nconf, even):
    """psi1 = psi2 (the ensemble's pair sink) with TwoBody's weights, even
    under the pairing: the tiled kernel sums only the blocks on and above the
    diagonal and mirrors them; with weights that are not even (random) the
    device check turns that off.  Against the oracle: FP64 within 1e-12, FP32
    orbitals within 1e-6."""
    rs = np.random.default_rng(n + nconf + 7)
    vol = int(np.prod(dims))
    psi = rs.standard_normal((nconf, n, vol)) + 1j * rs.standard_normal((nconf, n, vol))
    tb = nb.TwoBody(dims, "TGND", "STANDARD", 1.0, 0.176776695, 0.99999, ctx)
    w = tb.w_host if even else rs.uniform(0.0, 1.0, vol)
    assert np.array_equal(w[tb.opp_host], w) == even
    wd = torch.from_numpy(np.ascontiguousarray(w)).to(ctx.device)
    od = torch.from_numpy(np.ascontiguousarray(tb.opp_host.astype(np.int32))).to(ctx.device)
    for dt, tol, prec in ((torch.complex128, FP64_REL, C.F64), (torch.complex64, 1e-6, C.F32)):
        p = torch.from_numpy(psi).to(ctx.device).to(dt)
        out = torch.empty((nconf, n, n), dtype=torch.complex128, device=ctx.device)
        ctx.check(nb.lib().nrcps_pair_matrix(ctx.handle, ctypes.c_void_p(p.data_ptr()), ctypes.c_void_p(p.data_ptr()),
                                             n, nconf, vol, ctypes.c_void_p(wd.data_ptr()),
                                             ctypes.c_void_p(od.data_ptr()), prec, ctypes.c_void_p(out.data_ptr())),
                  "pair_matrix")
        got = out.cpu().numpy()
        for c in sorted({0, nconf - 1}):
            pc = p[c].cpu().numpy().astype(np.complex128)
            r = O.pair_matrix(pc, pc, w, tb.opp_host)
            assert max_norm_err(got[c], r) < tol, (dt, c)
            if even:
                assert np.array_equal(got[c], got[c].T)


@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_pair_matrix_with_a_table_that_is_no_involution(ctx, precision):
    """The tiled kernel pairs each site with its opposite (opp(opp(i)) = i,
    as TwoBody's parity mirror); nrcps_pair_matrix checks that on the device
    and, for any other table (here a random permutation), sums every site's
    term through the plain gather: the same pair matrices as the oracle."""
    rs = np.random.default_rng(21)
    dims, n, nconf = (8, 8, 8), 10, 3
    vol = int(np.prod(dims))
    psi1 = rs.standard_normal((nconf, n, vol)) + 1j * rs.standard_normal((nconf, n, vol))
    psi2 = rs.standard_normal((nconf, n, vol)) + 1j * rs.standard_normal((nconf, n, vol))
    w = rs.uniform(0.0, 1.0, vol)
    opp = rs.permutation(vol).astype(np.int32)
    assert np.any(opp[opp] != np.arange(vol))
    dt, tol = (torch.complex128, FP64_REL) if precision == "f64" else (torch.complex64, 1e-6)
    p1 = torch.from_numpy(psi1).to(ctx.device).to(dt)
    p2 = torch.from_numpy(psi2).to(ctx.device).to(dt)
    out = torch.empty((nconf, n, n), dtype=torch.complex128, device=ctx.device)
    wd = torch.from_numpy(w).to(ctx.device)
    od = torch.from_numpy(opp).to(ctx.device)
    ctx.check(nb.lib().nrcps_pair_matrix(ctx.handle, ctypes.c_void_p(p1.data_ptr()), ctypes.c_void_p(p2.data_ptr()),
                                         n, nconf, vol, ctypes.c_void_p(wd.data_ptr()), ctypes.c_void_p(od.data_ptr()),
                                         C.F64 if precision == "f64" else C.F32, ctypes.c_void_p(out.data_ptr())),
              "pair_matrix")
    got = out.cpu().numpy()
    for c in range(nconf):
        r = O.pair_matrix(p1[c].cpu().numpy().astype(np.complex128), p2[c].cpu().numpy().astype(np.complex128),
                          w, opp)
        assert max_norm_err(got[c], r) < tol


@pytest.mark.parametrize("tile", [1, 0])
def test_pair_matrix_skips_partners_outside_the_lattice(ctx, tile):
    """nrcps_pair_matrix with an opposite-site table holding indices outside
    [0, vol) (-1 and vol): those sites contribute nothing, in the tiled and
    the per-pair kernels, and nothing is read out of bounds."""
    rs = np.random.default_rng(5)
    dims, n, nconf = (8, 8, 8), 6, 2
    vol = int(np.prod(dims))
    psi1 = rs.standard_normal((nconf, n, vol)) + 1j * rs.standard_normal((nconf, n, vol))
    psi2 = rs.standard_normal((nconf, n, vol)) + 1j * rs.standard_normal((nconf, n, vol))
    w = rs.uniform(0.0, 1.0, vol)
    opp = rs.permutation(vol).astype(np.int32)
    bad = rs.choice(vol, 20, replace=False)
    opp[bad[:10]] = -1
    opp[bad[10:]] = vol
    p1 = torch.from_numpy(psi1).to(ctx.device)
    p2 = torch.from_numpy(psi2).to(ctx.device)
    out = torch.empty((nconf, n, n), dtype=torch.complex128, device=ctx.device)
    wd = torch.from_numpy(w).to(ctx.device)
    od = torch.from_numpy(opp).to(ctx.device)
    ctx.set_option("pair.tile", tile)
    try:
        ctx.check(nb.lib().nrcps_pair_matrix(ctx.handle, ctypes.c_void_p(p1.data_ptr()),
                                             ctypes.c_void_p(p2.data_ptr()), n, nconf, vol,
                                             ctypes.c_void_p(wd.data_ptr()), ctypes.c_void_p(od.data_ptr()), C.F64,
                                             ctypes.c_void_p(out.data_ptr())),
                  "pair_matrix")
        ctx.synchronize()
    finally:
        ctx.set_option("pair.tile", 1)
    keep = (opp >= 0) & (opp < vol)
    w0 = np.where(keep, w, 0.0)
    opp0 = np.where(keep, opp, 0)
    got = out.cpu().numpy()
    for c in range(nconf):
        assert max_norm_err(got[c], O.pair_matrix(psi1[c], psi2[c], w0, opp0)) < FP64_REL


def test_lu_cases_match_reference(golden, ctx):
    """Determinants against ludcmp: 1e-12 relative, or 1e-13 of the Hadamard
    bound (product of row norms) for the deliberately near-singular cases,
    whose determinant is pure cancellation."""
    g = golden("lu_cases.npz")
    for i, ref in enumerate(g["dets"]):
        m = g[f"m{i}"]
        n = m.shape[0]
        d = nb.slater_dets(torch.from_numpy(m).to(ctx.device).reshape(1, n, n), ctx=ctx).cpu().numpy()[0, n - 1]
        hadamard = np.prod(np.linalg.norm(m, axis=1))
        assert abs(d - ref) <= max(1e-12 * abs(ref), 1e-13 * hadamard), i


def test_log_det(ctx):
    rs = np.random.default_rng(2)
    m = rs.standard_normal((6, 6)) + 1j * rs.standard_normal((6, 6))
    d = nb.slater_dets(torch.from_numpy(m).to(ctx.device).reshape(1, 6, 6), log=True, ctx=ctx).cpu().numpy()[0]
    for n in range(1, 7):
        ref = O.minor_det(m, n, log=True)
        assert abs(np.exp(d[n - 1]) - np.exp(ref)) < 1e-12 * abs(np.exp(ref))


# ------------------------------------------------------------- ensemble
def _job_from_golden(args, precision):
    j = nb.EnsembleJob(L=int(args["L"]), T=int(args["T"]), n_conf=int(args["configs"]), rng=args.get("rng", "RANLXS2"),
                       seed=int(args["seed"]), field=args.get("field", "ZTWO"), precision=precision,
                       cutoff=float(args["cutoff"]), couplings=[float(c) for c in str(args["couplings"]).split(",")])
    if args.get("potential"):
        j.potential, j.kappa, j.pot_type = True, float(args["kappa"]), args["ptype"]
    if args.get("mode") == "slater2":
        j.mode, j.wavefunc = "slater2", args["wavefunc"]
        j.wf_disp, j.wf_lambda = args["tb_disp"], float(args["tb_lambda"])
    return j


def _golden_sources(g, args, dims):
    """The fixture's dense sources; fixtures too large to hold them store every
    k-th entry, and the sources are rebuilt by the library's OneBody::Set
    (nrcps_sho_source) and checked against that sample."""
    if "sources" in g.files:
        return g["sources"]
    sho = json.load(open(os.path.join(GOLDEN, "sho_coefficients.json")))
    lam = (float(args["lambda1"]), float(args["lambda2"]), float(args["lambda3"]))
    src = np.stack([nb.sho_source(dims, lam, sho[str(n)]) for n in range(int(args["N"]))])
    assert np.array_equal(src[:, ::int(g["sources_stride"])], g["sources_sample"])
    return src


def _ensemble_from_golden(g, args, job, ctx):
    if "momenta" in g.files and args.get("sources", "mom") == "mom":
        idx, _, _ = nb.momenta(job.dims, "PERFECT", 1.0, float(args["ef"]), job.cutoff)
        return nb.Ensemble(job, plane_wave_index=idx, ctx=ctx)
    return nb.Ensemble(job, sources=_golden_sources(g, args, job.dims), ctx=ctx)


def per_tau_rel_err(got, ref, symmetric=False):
    """max over configurations and minors of |got - ref| / |ref| (or, when
    `symmetric`, / max(|got|, |ref|)), per slice."""
    got, ref = np.asarray(got), np.asarray(ref)
    den = np.maximum(np.abs(got), np.abs(ref)) if symmetric else np.abs(ref)
    e = np.abs(got - ref) / np.maximum(den, 1e-300)
    return e.reshape(-1, e.shape[-2], e.shape[-1]).max(axis=(0, 2))


# config 1 (L=16, N=7, T=32), small lattices with several couplings, Gaussian
# fields and the trapped form, and the reference's own run at the batched
# workload's shape (L=32, N=19, T=64, 2 configurations)
@pytest.mark.parametrize("name", ["ensemble_config1.npz", "ensemble_multicoupling.npz", "ensemble_gauss.npz",
                                  "ensemble_trapped.npz", "ensemble_config2.npz"])
def test_ensemble_fp64_matches_reference(golden, ctx, name):
    g = golden(name)
    args = json.loads(str(g["args"]))
    job = _job_from_golden(args, "f64")
    ens = _ensemble_from_golden(g, args, job, ctx)
    dets = ens.run(0).cpu().numpy()
    ens.close()
    ref = g["dets"]
    assert dets.shape == ref.shape
    err = per_tau_rel_err(dets, ref)
    print(f"{name}: FP64 vs reference, max rel err per tau: " + " ".join(f"{v:.1e}" for v in err))
    assert err.max() < FP64_REL, err.max()


def test_trapped_shape_fp64_matches_reference_to_its_conditioning(golden, ctx):
    """The reference's own run at the trapped workload's shape (L=48, T=128,
    SHO N=10, [K,V,I,V,K], pair sink; 2 configurations).  Unstabilised, the
    10 orbitals align as tau grows and the pair-matrix minors become
    ill-conditioned: any FP64 evaluation of them, the reference's included,
    carries rounding amplified by the condition number.  So each slice is held
    to 1e-12 or to the problem's own sensitivity, whichever is larger: the
    change of this library's FP64 result when every source entry moves by one
    ulp, times 1e4 (the rounding of tau steps of four 3-D FFTs against a
    single perturbation of the input).  The early slices, where the
    sensitivity is below 1e-16, are held to 1e-12 outright.  Differences are
    taken relative to the larger of the two values: by the last slices some
    minors pass through zero by cancellation, and a relative difference
    against the smaller value there measures only how close to zero the
    reference's rounding happened to land.  From about tau = 115 the bound
    exceeds 1: the reference's own FP64 values carry no significant digit
    there, and only re-orthonormalised runs (the next test) say anything
    about those slices."""
    g = golden("ensemble_trapped48.npz")
    args = json.loads(str(g["args"]))
    job = _job_from_golden(args, "f64")
    src = _golden_sources(g, args, job.dims)
    ens = nb.Ensemble(job, sources=src, ctx=ctx)
    dets = ens.run(0).cpu().numpy()
    ens.close()
    rs = np.random.default_rng(48)
    ulp = np.spacing(np.abs(src.real)) * rs.choice([-1.0, 1.0], src.shape) + \
        1j * np.spacing(np.abs(src.imag)) * rs.choice([-1.0, 1.0], src.shape)
    ens = nb.Ensemble(job, sources=src + ulp, ctx=ctx)
    moved = ens.run(0).cpu().numpy()
    ens.close()
    ref = g["dets"]
    assert dets.shape == ref.shape
    err = per_tau_rel_err(dets, ref, symmetric=True)
    sens = per_tau_rel_err(moved, dets, symmetric=True)
    print("trapped48 FP64 vs reference, max rel err per tau: " + " ".join(f"{v:.1e}" for v in err))
    print("  sensitivity to one ulp of the sources:          " + " ".join(f"{v:.1e}" for v in sens))
    bound = np.maximum(FP64_REL, 1e4 * sens)
    assert np.all(err < bound), np.flatnonzero(err >= bound)
    assert np.all(err[:16] < FP64_REL)


def test_trapped_workload_fp32_vs_fp64_full_shape(golden, ctx):
    """The trapped workload at its own shape and size: L=48, T=128, SHO N=10,
    [K,V,I,V,K] with kappa = 0.005, pair sink, Z2 a=0.5, RANLXS2 seed 31,
    1024 configurations.  FP32 propagation (dense FP32 overlap on the tensor
    cores) against the FP64 mode on the same fields, both re-orthonormalised
    every 8 slices (the determinants are rescaled to the unstabilised ones):
    the correlators C_m(tau) = <det S2_m(tau)>
    (production/slater_det2_trapped/main-no_cum.C:205-207) within 1e-5
    relative at every tau."""
    g = golden("ensemble_trapped48.npz")
    args = json.loads(str(g["args"]))
    out = {}
    for prec in ("f32", "f64"):
        job = _job_from_golden(args, prec)
        job.n_conf = 1024
        job.qr_period = 8
        ens = _ensemble_from_golden(g, args, job, ctx)
        d = ens.run(0)
        out[prec] = d.mean(0).cpu().numpy()  # [T, 2N]
        scale = d.abs().mean(0).cpu().numpy()
        ens.close()
        del d
    c32, c64 = out["f32"], out["f64"]
    err = np.max(np.abs(c32 - c64) / np.abs(c64), axis=1)
    err_scale = np.max(np.abs(c32 - c64) / scale, axis=1)
    print("trapped L=48 T=128 1024 conf: FP32 vs FP64, max rel err of C(tau) per tau: " +
          " ".join(f"{v:.1e}" for v in err))
    print("  relative to <|det|>: " + " ".join(f"{v:.1e}" for v in err_scale))
    assert err.max() < FP32_REL, err.max()


def test_full_size_batch_matches_a_two_configuration_run(ctx):
    """The batched workload's size: 4096 configurations x 19 orbitals of 32^3
    sites (2.55 G complex FP32 values, 20.4 GB; offsets past 2^31 in every
    kernel of the step and the measurement).  The last two configurations'
    determinants equal, bit for bit, a separate run of just those two
    configurations (same fields: configuration c reads its own stream
    window), for 8 slices with a re-orthonormalisation after 4."""
    idx, _, _ = nb.momenta((32, 32, 32), "PERFECT", 1.0, 0.045, 2.0)
    assert len(idx) == 19
    job = nb.EnsembleJob(L=32, T=8, n_conf=4096, seed=7, precision="f32", fermi_energy=0.045, qr_period=4)
    ens = nb.Ensemble(job, plane_wave_index=idx, ctx=ctx)
    big = ens.run(0)[-2:].clone()
    ens.close()
    torch.cuda.empty_cache()
    job.n_conf = 2
    ens = nb.Ensemble(job, plane_wave_index=idx, ctx=ctx)
    small = ens.run(4094).clone()
    ens.close()
    assert torch.equal(big, small)


def test_ensemble_fp32_config1(golden, ctx):
    """FP32 propagation: every per-configuration determinant within 5e-5 of
    the reference (FP32 rounding random-walks through 32 steps of six FFT
    passes), and the ensemble-averaged correlator C_n(tau) = <|det S_n|^2>
    within 1e-5 of the FP64 result over 128 configurations."""
    g = golden("ensemble_config1.npz")
    args = json.loads(str(g["args"]))
    job = _job_from_golden(args, "f32")
    idx, _, _ = nb.momenta(job.dims, "PERFECT", 1.0, 0.1, job.cutoff)
    dets = nb.Ensemble(job, plane_wave_index=idx, ctx=ctx).run(0).cpu().numpy()
    assert rel_err(dets, g["dets"]) < 5e-5
    job32 = _job_from_golden(args, "f32")
    job64 = _job_from_golden(args, "f64")
    job32.n_conf = job64.n_conf = 128
    d32 = nb.Ensemble(job32, plane_wave_index=idx, ctx=ctx).run(0).cpu().numpy()
    d64 = nb.Ensemble(job64, plane_wave_index=idx, ctx=ctx).run(0).cpu().numpy()
    c32 = (np.abs(d32) ** 2).mean(0)
    c64 = (np.abs(d64) ** 2).mean(0)
    assert rel_err(c32, c64) < FP32_REL


def test_ensemble_later_configurations_use_later_fields(ctx):
    """Configurations 3..4 of a run from the stream start equal a run that starts at 3."""
    job = nb.EnsembleJob(L=8, T=6, n_conf=5, fermi_energy=0.35, precision="f64")
    idx, _, _ = nb.momenta(job.dims, "PERFECT", 1.0, 0.35, job.cutoff)
    full = nb.Ensemble(job, plane_wave_index=idx, ctx=ctx).run(0).cpu().numpy()
    job2 = nb.EnsembleJob(L=8, T=6, n_conf=2, fermi_energy=0.35, precision="f64")
    part = nb.Ensemble(job2, plane_wave_index=idx, ctx=ctx).run(3).cpu().numpy()
    assert np.array_equal(full[3:5], part)


def test_free_gas_analytic_on_device(ctx):
    """Kinetic only: det S_n(tau) = prod_{i<=n} xi(p_i)^(-tau) (tests/free_gas)."""
    dims = (16, 16, 16)
    idx, _, _ = nb.momenta(dims, "PERFECT", 1.0, 0.1, 2.0)
    xi = nb.kinetic_table(dims, "PERFECT", 1.0, 0.5, 2.0)
    kin = nb.Kinetic(dims, "PERFECT", 1.0, 0.5, 2.0, ctx)
    prop = nb.Propagator(len(idx), dims, "f64", ctx)
    for n, j in enumerate(idx):
        v = np.zeros(4096, complex)
        v[j] = 1
        prop.set(v, n)
    src = torch.zeros((len(idx), 4096), dtype=torch.complex128, device=ctx.device)
    src[torch.arange(len(idx)), torch.as_tensor(idx, dtype=torch.long)] = 1
    for tau in range(1, 5):
        prop.run([kin, kin])
        S = nb.overlap(src, prop.get().b.reshape(1, len(idx), -1), ctx)
        d = nb.slater_dets(S, ctx=ctx).cpu().numpy()[0]
        for n in range(1, len(idx) + 1):
            expect = np.prod(xi[idx[:n]] ** (-2.0 * tau))
            assert abs(d[n - 1] / expect - 1) < 1e-13


# ------------------------------------------------ fused single-pass kernel
def _random_step_inputs(ctx, L, nconf, batch, precision, seed=0):
    rs = np.random.default_rng(seed)
    vol = L ** 3
    psi = rs.standard_normal((nconf * batch, L, L, L)) + 1j * rs.standard_normal((nconf * batch, L, L, L))
    dt = torch.complex128 if precision == "f64" else torch.complex64
    kinv = torch.from_numpy(1.0 / nb.kinetic_table((L, L, L), "PERFECT", 1.0, 0.5, 2.0)).to(ctx.device)
    bits = nb.draw_z2_bits("RANLXS2", 5 + seed, 0, nconf * vol, ctx)
    return torch.from_numpy(psi).to(dt).to(ctx.device), kinv, bits


@pytest.mark.parametrize("L,precision", [(16, "f32"), (24, "f32"), (32, "f32"), (48, "f32"), (12, "f32"),
                                         (16, "f64")])
def test_real_weight_table_field(ctx, L, precision):
    """Field mode 3: the Gaussian field as one FP32 weight (1 + a phi)/V per
    site, against mode 2 forming it from phi per site: within 2e-6 of the
    orbitals' norm after one step (the weight rounded to FP32 once), in the
    fused step (FP32; staged in shared memory by kind 11, or read per site
    from a table that is not 16-byte aligned) and in the pencil passes
    (L = 12, and FP64)."""
    nconf, batch = 3, 2
    psi, kinv, _ = _random_step_inputs(ctx, L, nconf, batch, precision, seed=3)
    phi, _ = nb.draw_fields("RANLXS2", 11, "GAUSS", L ** 3, nconf, 0, ctx)
    wt = ((1.0 + 0.3 * phi[..., 0]) / L ** 3).to(torch.float32).contiguous()
    a, b = psi.clone(), psi.clone()
    nb.propagate(a, batch, kinv, phi, 0.3, field_mode=2, ctx=ctx)
    nb.propagate(b, batch, kinv, wt, 0.0, field_mode=3, ctx=ctx)
    assert max_norm_err(b.cpu().numpy(), a.cpu().numpy()) < 2e-6
    # a table that starts 4 bytes past a 16-byte boundary: the weights are
    # read per site instead of staged, the same products
    buf = torch.zeros(wt.numel() + 1, dtype=torch.float32, device=ctx.device)
    buf[1:] = wt.reshape(-1)
    c = psi.clone()
    nb.propagate(c, batch, kinv, buf[1:], 0.0, field_mode=3, ctx=ctx)
    assert buf[1:].data_ptr() % 16 == 4
    assert torch.equal(c, b)


@pytest.mark.parametrize("L", [8, 16, 32])
def test_orbitals_off_a_16_byte_boundary_take_the_pencil_passes(ctx, L):
    """FP32 orbitals whose array starts 8 bytes past a 16-byte boundary (a
    view at an odd element): the fused kinds that move slabs by bulk copy
    need 16-byte starts, so such a call takes the pencil passes -- the same
    values as the pencil passes on an aligned copy."""
    psi, kinv, bits = _random_step_inputs(ctx, L, 2, 3, "f32", seed=4)
    buf = torch.zeros(psi.numel() + 1, dtype=psi.dtype, device=ctx.device)
    buf[1:] = psi.reshape(-1)
    view = buf[1:].view(psi.shape)
    assert view.data_ptr() % 16 == 8
    nb.propagate(view, 3, kinv, bits, 0.5, ctx=ctx)
    ref = psi.clone()
    ctx.set_option("propagate.fused", 0)
    try:
        nb.propagate(ref, 3, kinv, bits, 0.5, ctx=ctx)
    finally:
        ctx.set_option("propagate.fused", 1)
    assert torch.equal(view, ref)


@pytest.mark.parametrize("L,precision", [(8, "f32"), (16, "f32"), (24, "f32"), (32, "f32"), (48, "f32"),
                                         (8, "f64"), (16, "f64"), (24, "f64"), (32, "f64")])
def test_fused_step_matches_pencil_passes(ctx, L, precision):
    psi, kinv, bits = _random_step_inputs(ctx, L, 3, 2, precision)
    a = psi.clone()
    b = psi.clone()
    ctx.set_option("propagate.fused", 1)
    nb.propagate(a, 2, kinv, bits, 0.5, ctx=ctx)
    ctx.set_option("propagate.fused", 0)
    nb.propagate(b, 2, kinv, bits, 0.5, ctx=ctx)
    ctx.set_option("propagate.fused", 1)
    tol = 1e-13 if precision == "f64" else 3e-6
    assert max_norm_err(a.cpu().numpy(), b.cpu().numpy()) < tol


@pytest.mark.parametrize("L,precision,clusters", [(32, "f32", [8, 16]), (24, "f32", [3, 4]), (16, "f32", [1, 2]),
                                                  (32, "f64", [8, 16])])
def test_fused_every_cluster_size_agrees(ctx, L, precision, clusters):
    psi, kinv, bits = _random_step_inputs(ctx, L, 2, 3, precision, seed=1)
    outs = []
    for c in clusters:
        ctx.set_option("fused.cluster", c)
        p = psi.clone()
        nb.propagate(p, 3, kinv, bits, 0.5, ctx=ctx)
        outs.append(p.cpu().numpy())
    ctx.set_option("fused.cluster", 0)
    tol = 1e-14 if precision == "f64" else 1e-6
    for o in outs[1:]:
        assert max_norm_err(o, outs[0]) < tol


def test_fused_step_vs_oracle_fp64(ctx):
    """One fused step against the oracle's K, I, K sequence on identical input."""
    L = 16
    dims = (L, L, L)
    rs = np.random.default_rng(4)
    psi0 = rs.standard_normal((2, L ** 3)) + 1j * rs.standard_normal((2, L ** 3))
    xi = O.kinetic_xi(dims, "PERFECT", 1.0, 0.5, (2 * O.PI) ** 2)
    itab = O.interaction_table(dims, 1.0, [0.019894367886486918], 1.0, (2 * O.PI) ** 2)
    field = O.field_slices("RANLXS2", 77, "ZTWO", L ** 3, 1)[0]
    ref = O.kinetic_evolve(O.interaction_evolve(dims, O.kinetic_evolve(psi0, xi),
                                                O.interaction_initialize(dims, field, itab)), xi)
    psi = torch.from_numpy(psi0.reshape(2, L, L, L)).to(ctx.device)
    bits = nb.draw_z2_bits("RANLXS2", 77, 0, L ** 3, ctx)
    kinv = torch.from_numpy(1.0 / xi).to(ctx.device)
    nb.propagate(psi, 2, kinv, bits, float(itab[0] * L ** 3), conf_stride=0, ctx=ctx)
    assert max_norm_err(psi.reshape(2, -1).cpu().numpy(), ref) < FP64_REL


def test_autotune_returns_a_variant(ctx):
    assert abs(ctx.autotune("f32", 32)) in (8, 16)


@pytest.mark.parametrize("L,precision", [(16, "f32"), (24, "f32"), (32, "f32"), (48, "f32"), (16, "f64"),
                                         (32, "f64")])
def test_lane_split_variant_agrees(ctx, L, precision):
    psi, kinv, bits = _random_step_inputs(ctx, L, 2, 3, precision, seed=2)
    outs = []
    for sp in (0, 1):
        ctx.set_option("fused.split", sp)
        q = psi.clone()
        nb.propagate(q, 3, kinv, bits, 0.5, ctx=ctx)
        outs.append(q.cpu().numpy())
    ctx.set_option("fused.split", -1)
    tol = 1e-14 if precision == "f64" else 2e-6
    assert max_norm_err(outs[1], outs[0]) < tol


_EXCHANGE_VARIANTS = [(2, "f32", 16, 2), (2, "f32", 24, 3), (2, "f32", 24, 4), (2, "f32", 32, 8), (2, "f64", 16, 2),
                      (2, "f64", 24, 4), (2, "f64", 32, 16), (3, "f32", 32, 8), (3, "f32", 32, 16),
                      (3, "f32", 48, 16), (3, "f64", 32, 16)]


@pytest.mark.parametrize("kind,precision,L,cluster", _EXCHANGE_VARIANTS)
def test_exchange_variants_are_bit_identical(ctx, kind, precision, L, cluster):
    """The bulk-copy exchanges (kinds 2 and 3) move the same values through
    the same arithmetic as the peer-access kernel (kind 0): results agree
    bit for bit."""
    psi, kinv, bits = _random_step_inputs(ctx, L, 3, 5, precision, seed=3)
    try:
        ctx.set_option("fused.kind", 0)
        ref = psi.clone()
        nb.propagate(ref, 5, kinv, bits, 0.5, ctx=ctx)
        ctx.set_option("fused.kind", kind)
        ctx.set_option("fused.cluster", cluster)
        q = psi.clone()
        nb.propagate(q, 5, kinv, bits, 0.5, ctx=ctx)
        ctx.synchronize()
        assert torch.equal(q, ref)
    finally:
        ctx.set_option("fused.cluster", 0)
        ctx.set_option("fused.kind", -1)


_PACKED_VARIANTS = [(4, 8, 1), (4, 16, 1), (4, 24, 4), (5, 24, 3), (4, 32, 8), (5, 32, 8), (6, 32, 8), (4, 48, 16)]


@pytest.mark.parametrize("kind,L,cluster", _PACKED_VARIANTS)
def test_packed_variants_agree(ctx, kind, L, cluster):
    """Kinds 4-6 compute the transforms two half-length DFTs per packed
    FP32x2 instruction: a different (equally accurate) operation order, so
    they agree with the scalar kernel to FP32 rounding, not bit for bit."""
    psi, kinv, bits = _random_step_inputs(ctx, L, 3, 5, "f32", seed=5)
    try:
        ctx.set_option("fused.kind", 0)
        ctx.set_option("fused.cluster", cluster)
        ref = psi.clone()
        nb.propagate(ref, 5, kinv, bits, 0.5, ctx=ctx)
        ctx.set_option("fused.kind", kind)
        q = psi.clone()
        nb.propagate(q, 5, kinv, bits, 0.5, ctx=ctx)
        ctx.synchronize()
        assert max_norm_err(q.cpu().numpy(), ref.cpu().numpy()) < 2e-6
    finally:
        ctx.set_option("fused.cluster", 0)
        ctx.set_option("fused.kind", -1)


@pytest.mark.parametrize("kind,ref_kind,precision,cluster,L", [
    (5, 4, "f32", 8, 32), (6, 4, "f32", 8, 32), (8, 4, "f32", 8, 32), (7, 0, "f32", 8, 32), (7, 0, "f64", 16, 32),
    (9, 4, "f32", 8, 32), (10, 0, "f32", 8, 32), (11, 0, "f32", 8, 32), (12, 4, "f32", 8, 32),
    (11, 3, "f32", 16, 32), (11, 0, "f64", 16, 32), (11, 0, "f32", 2, 16), (11, 0, "f32", 4, 24),
    (11, 0, "f64", 4, 24), (11, 3, "f32", 12, 48),
    (7, 3, "f32", 12, 48)])
def test_same_arithmetic_variants_are_bit_identical(ctx, kind, ref_kind, precision, cluster, L):
    """Variants that differ only in how the slab reaches shared memory or how
    the exchange moves it (peer loads and stores, bulk copies, or peer loads
    with st.async write-backs completing on the owner's mbarrier) run the same
    arithmetic: results agree bit for bit."""
    psi, kinv, bits = _random_step_inputs(ctx, L, 3, 5, precision, seed=6)
    try:
        ctx.set_option("fused.cluster", cluster)
        ctx.set_option("fused.kind", ref_kind)
        ref = psi.clone()
        nb.propagate(ref, 5, kinv, bits, 0.5, ctx=ctx)
        ctx.set_option("fused.kind", kind)
        q = psi.clone()
        nb.propagate(q, 5, kinv, bits, 0.5, ctx=ctx)
        ctx.synchronize()
        assert torch.equal(q, ref)
    finally:
        ctx.set_option("fused.cluster", 0)
        ctx.set_option("fused.kind", -1)


@pytest.mark.parametrize("kind,precision,L,cluster", [(0, "f32", 32, 8), (4, "f32", 48, 16), (3, "f32", 48, 16),
                                                      (1, "f32", 48, 16), (11, "f32", 32, 8), (7, "f32", 32, 8),
                                                      (2, "f32", 24, 4), (0, "f64", 32, 16), (11, "f64", 24, 4),
                                                      (0, "f32", 16, 1), (11, "f32", 48, 12)])
def test_z2_position_weights_table_is_bit_identical(ctx, kind, precision, L, cluster):
    """A Z2 field with a position factor P ([K,V,I,V,K]): the fused step reads
    the weights (1 +- a) P(x)/V of every site from a table made ahead of the
    step ("fused.zpos" 1) or forms them per site from P ("fused.zpos" 0).
    The table holds the same products split the same way, so the two agree
    bit for bit; against the pencil passes they agree to rounding."""
    psi, kinv, bits = _random_step_inputs(ctx, L, 3, 5, precision, seed=8)
    rs = np.random.default_rng(L)
    pos = torch.from_numpy(np.exp(-rs.uniform(0.0, 2.0, L ** 3))).to(ctx.device)
    outs = []
    try:
        ctx.set_option("fused.cluster", cluster)
        ctx.set_option("fused.kind", kind)
        for zpos in (0, 1):
            ctx.set_option("fused.zpos", zpos)
            q = psi.clone()
            nb.propagate(q, 5, kinv, bits, 0.5, pos=pos, ctx=ctx)
            outs.append(q)
        choice = ctx.fused_choice(precision, L)
        ctx.set_option("fused.kind", -1)
        ctx.set_option("fused.cluster", 0)
        ctx.set_option("propagate.fused", 0)
        ref = psi.clone()
        nb.propagate(ref, 5, kinv, bits, 0.5, pos=pos, ctx=ctx)
        ctx.synchronize()
    finally:
        ctx.set_option("propagate.fused", 1)
        ctx.set_option("fused.zpos", 1)
        ctx.set_option("fused.cluster", 0)
        ctx.set_option("fused.kind", -1)
    assert choice == (kind, cluster)
    assert torch.equal(outs[0], outs[1])
    tol = 1e-13 if precision == "f64" else 3e-6
    assert max_norm_err(outs[1].cpu().numpy(), ref.cpu().numpy()) < tol


@pytest.mark.parametrize("cluster", [2, 4])
def test_st_async_kernel_cluster_sizes_are_bit_identical(ctx, cluster):
    """Kind 11 with 2 or 4 CTAs per cluster (16 or 8 x-planes per CTA) runs
    every pencil through the same arithmetic as with 8: bit for bit."""
    psi, kinv, bits = _random_step_inputs(ctx, 32, 3, 5, "f32", seed=10)
    out = []
    try:
        ctx.set_option("fused.kind", 11)
        for c in (8, cluster):
            ctx.set_option("fused.cluster", c)
            q = psi.clone()
            nb.propagate(q, 5, kinv, bits, 0.5, ctx=ctx)
            out.append(q)
            assert ctx.fused_choice("f32", 32) == (11, c)
        ctx.synchronize()
    finally:
        ctx.set_option("fused.cluster", 0)
        ctx.set_option("fused.kind", -1)
    assert torch.equal(out[0], out[1])


@pytest.mark.parametrize("off0", [0, 7, 32 * 5 + 3])
@pytest.mark.parametrize("L,cluster", [(32, 8), (48, 12)])
def test_st_async_kernel_field_words_at_any_bit_offset(ctx, off0, L, cluster):
    """Kind 11 reads the Z2 field words of its rows from shared memory when
    the configuration's field starts on a 32-bit word, and from L2 otherwise
    (a field window at an odd bit offset, as the branching driver's
    sub-streams have): both bit-identical to the peer-access kernel (kind 0,
    or kind 3 where kind 0 has no cluster of that size)."""
    psi, kinv, _ = _random_step_inputs(ctx, L, 3, 5, "f32", seed=9)
    # configuration c reads bits off0 + c (V - 1) .. + V - 1: mixed word alignment
    bits = nb.draw_z2_bits("RANLXS2", 11, 0, 3 * L ** 3 + 1024, ctx)
    ref_kind = 0 if cluster == 8 else 3
    out = []
    try:
        ctx.set_option("fused.cluster", cluster)
        for kind in (ref_kind, 11):
            ctx.set_option("fused.kind", kind)
            q = psi.clone()
            nb.propagate(q, 5, kinv, bits, 0.5, off0=off0, conf_stride=L ** 3 - 1, ctx=ctx)
            out.append(q)
        ctx.synchronize()
    finally:
        ctx.set_option("fused.cluster", 0)
        ctx.set_option("fused.kind", -1)
    assert torch.equal(out[0], out[1])


@pytest.mark.parametrize("kind,ref_kind,L,cluster", [(10, 0, 16, 2), (10, 0, 24, 4), (9, 4, 24, 4), (9, 5, 32, 8)])
def test_resident_kinetic_slab_variants(ctx, kind, ref_kind, L, cluster):
    """Kinds 9 and 10 read k(p) from the CTA's resident slab in shared
    memory instead of L2: the same values and arithmetic as kinds 6 and 3,
    so they agree bit for bit with the kernels of the same transform order."""
    psi, kinv, bits = _random_step_inputs(ctx, L, 3, 5, "f32", seed=7)
    try:
        ctx.set_option("fused.cluster", cluster)
        ctx.set_option("fused.kind", ref_kind)
        ref = psi.clone()
        nb.propagate(ref, 5, kinv, bits, 0.5, ctx=ctx)
        ctx.set_option("fused.kind", kind)
        q = psi.clone()
        nb.propagate(q, 5, kinv, bits, 0.5, ctx=ctx)
        ctx.synchronize()
        assert torch.equal(q, ref)
    finally:
        ctx.set_option("fused.cluster", 0)
        ctx.set_option("fused.kind", -1)


def test_synchronize_reports_no_timeout(ctx):
    psi, kinv, bits = _random_step_inputs(ctx, 32, 2, 2, "f32")
    nb.propagate(psi, 2, kinv, bits, 0.5, ctx=ctx)
    ctx.synchronize()  # raises NrcpsError(TIMEOUT) if a bounded wait gave up


# every fused kernel with mbarrier waits: peer access with a staged slab (0,
# also as a one-CTA cluster), lane split (1), bulk exchange staged (2) and via
# L2 (3), st.async write-backs (11)
_WAITING_VARIANTS = [(0, "f32", 32, 8, "z2"), (0, "f32", 16, 1, "z2"), (1, "f32", 32, 8, "z2"),
                     (2, "f32", 32, 8, "z2"), (3, "f32", 32, 8, "z2"), (3, "f64", 32, 16, "z2"),
                     (11, "f32", 32, 8, "z2"), (11, "f64", 32, 16, "z2"), (11, "f32", 48, 12, "z2"),
                     (11, "f32", 32, 8, "gauss"), (12, "f32", 32, 8, "gauss")]


@pytest.mark.parametrize("kind,precision,L,cluster,field", _WAITING_VARIANTS)
def test_fused_wait_time_out_is_reported_and_context_survives(ctx, kind, precision, L, cluster, field):
    """A wait that runs out: the first wait of CTA 0 of cluster 0 is made on
    an mbarrier nothing arrives on (a stand-in for a copy that never lands),
    with a 2 ms limit.  Its cluster leaves the orbital loop together, the
    launch ends in milliseconds, nrcps_synchronize reports TIMEOUT, and the
    next step on the same context is bit-identical to a clean run.  Kinds
    11/12 have one instance per field class: a Gaussian field runs the
    other one."""
    import time
    psi, kinv, bits = _random_step_inputs(ctx, L, 3, 5, precision, seed=8)
    if field == "gauss":
        phi, _ = nb.draw_fields("RANLXS2", 3, "GAUSS", L ** 3, 3, 0, ctx)
        fld = {"field": phi, "a": 0.3, "field_mode": 2}
    else:
        fld = {"field": bits, "a": 0.5}

    def step(q):
        nb.propagate(q, 5, kinv, fld["field"], fld["a"], field_mode=fld.get("field_mode", 1), ctx=ctx)

    try:
        ctx.set_option("fused.kind", kind)
        ctx.set_option("fused.cluster", cluster)
        ref = psi.clone()
        step(ref)
        ctx.synchronize()
        ctx.set_option("fused.wait_ns", 2_000_000)
        ctx.set_option("fused.stall_test", 1)
        bad = psi.clone()
        t0 = time.perf_counter()
        step(bad)
        with pytest.raises(nb.NrcpsError) as err:
            ctx.synchronize()
        assert err.value.status == 7  # NRCPS_ERR_TIMEOUT
        assert time.perf_counter() - t0 < 5.0
        ctx.set_option("fused.stall_test", 0)
        ctx.set_option("fused.wait_ns", 2_000_000_000)
        again = psi.clone()
        step(again)
        ctx.synchronize()
        assert torch.equal(again, ref)
    finally:
        ctx.set_option("fused.stall_test", 0)
        ctx.set_option("fused.wait_ns", 2_000_000_000)
        ctx.set_option("fused.cluster", 0)
        ctx.set_option("fused.kind", -1)


# ------------------------------------------------ re-orthonormalisation
@pytest.mark.parametrize("period", [1, 2, 5])
def test_qr_reorthonormalisation_preserves_determinants_fp64(ctx, period):
    """det S_n(Psi) = det S_n(Q) prod R_ii: re-orthonormalised runs reproduce
    the unstabilised determinants (the reference's semantics)."""
    base = dict(L=8, T=12, n_conf=6, fermi_energy=0.35, precision="f64", seed=4321)
    idx, _, _ = nb.momenta((8, 8, 8), "PERFECT", 1.0, 0.35, 2.0)
    plain = nb.Ensemble(nb.EnsembleJob(**base), plane_wave_index=idx, ctx=ctx).run(0).cpu().numpy()
    qr = nb.Ensemble(nb.EnsembleJob(qr_period=period, **base), plane_wave_index=idx, ctx=ctx).run(0).cpu().numpy()
    assert rel_err(qr, plain) < 1e-11


def test_qr_pair_sink_fp64(golden, ctx):
    """Re-orthonormalisation under the pair sink (SlaterDet2 on TwoBody, the
    replaced-column minors too): with Phi(Psi) = R^T Phi(Q) R the rescaled
    determinants reproduce the unstabilised ones."""
    g = golden("ensemble_trapped.npz")
    args = json.loads(str(g["args"]))
    job0 = _job_from_golden(args, "f64")
    job0.T, job0.n_conf = 9, 3
    jobq = _job_from_golden(args, "f64")
    jobq.T, jobq.n_conf, jobq.qr_period = 9, 3, 2
    plain = nb.Ensemble(job0, sources=g["sources"], ctx=ctx).run(0).cpu().numpy()
    qr = nb.Ensemble(jobq, sources=g["sources"], ctx=ctx).run(0).cpu().numpy()
    assert rel_err(qr, plain) < 1e-11


def test_qr_dense_sources_fp64(golden, ctx):
    g = golden("ensemble_trapped.npz")
    src = g["sources"]
    job = dict(L=8, T=6, n_conf=2, seed=31, precision="f64", cutoff=0.99999, potential=True, kappa=0.005)
    plain = nb.Ensemble(nb.EnsembleJob(**job), sources=src, ctx=ctx).run(0).cpu().numpy()
    qr = nb.Ensemble(nb.EnsembleJob(qr_period=2, **job), sources=src, ctx=ctx).run(0).cpu().numpy()
    assert rel_err(qr, plain) < 1e-11


def test_qr_fp32_against_fp64(golden, ctx):
    g = golden("ensemble_config1.npz")
    idx, _, _ = nb.momenta((16, 16, 16), "PERFECT", 1.0, 0.1, 2.0)
    base = dict(L=16, T=32, n_conf=64, seed=1234)
    d64 = nb.Ensemble(nb.EnsembleJob(precision="f64", **base), plane_wave_index=idx, ctx=ctx).run(0).cpu().numpy()
    d32 = nb.Ensemble(nb.EnsembleJob(precision="f32", qr_period=8, **base), plane_wave_index=idx,
                      ctx=ctx).run(0).cpu().numpy()
    assert rel_err(d32, d64) < 5e-5
    assert rel_err((np.abs(d32) ** 2).mean(0), (np.abs(d64) ** 2).mean(0)) < FP32_REL
    assert rel_err(d64[:2], g["dets"]) < FP64_REL


@pytest.mark.parametrize("L,T,ef,n_conf", [(24, 64, 0.08, 16), (48, 32, 0.02, 4)])
def test_fp32_correlators_other_extents(ctx, L, T, ef, n_conf):
    """The same FP32-vs-FP64 bound at the extents whose register DFTs use
    radix-3 stages (24 = 8 x 3, 48 = 16 x 3), N = 19, QR every 8 slices."""
    idx, _, _ = nb.momenta((L, L, L), "PERFECT", 1.0, ef, 2.0)
    assert len(idx) == 19
    out = {}
    for prec, qr in (("f32", 8), ("f64", 0)):
        job = nb.EnsembleJob(L=L, T=T, n_conf=n_conf, seed=11, precision=prec, fermi_energy=ef, qr_period=qr)
        ens = nb.Ensemble(job, plane_wave_index=idx, ctx=ctx)
        out[prec] = (np.abs(ens.run(0).cpu().numpy()) ** 2).mean(0)
        ens.close()
    assert rel_err(out["f32"], out["f64"]) < FP32_REL


def test_fp32_correlators_at_the_batched_config_shape(ctx):
    """L=32, T=64, N=19 plane waves, Z2 a=0.5, seed 7: FP32 propagation with
    re-orthonormalisation every 8 slices against the FP64 mode (itself held to
    1e-12 of the oracle by the tests above) -- C_n(tau) = <|det S_n(tau)|^2>
    over 32 configurations within 1e-5 relative for every n and tau."""
    idx, _, _ = nb.momenta((32, 32, 32), "PERFECT", 1.0, 0.045, 2.0)
    assert len(idx) == 19
    out = {}
    for prec, qr in (("f32", 8), ("f64", 0)):
        job = nb.EnsembleJob(L=32, T=64, n_conf=32, seed=7, precision=prec, fermi_energy=0.045, qr_period=qr)
        ens = nb.Ensemble(job, plane_wave_index=idx, ctx=ctx)
        out[prec] = (np.abs(ens.run(0).cpu().numpy()) ** 2).mean(0)
        ens.close()
    assert rel_err(out["f32"], out["f64"]) < FP32_REL

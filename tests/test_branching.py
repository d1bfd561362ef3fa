"""The multilevel branching driver (production/two_body-branched/main.C:23-80)
breadth first on the device against the reference's own recursion over its
current classes (tests/golden/branching.npz, written by the reference build)
and the oracle's depth-first restatement.

Tolerances: FP64 1e-12 of each slice's value; FP32 1e-5 against FP64.
"""
import numpy as np
import pytest

from oracle import oracle as O


def _sources(L):
    dims = (L,) * 3
    idx, _, _ = O.momenta(dims, "PERFECT", 1.0, 0.35 * (8 / L) ** 2, (2 * O.PI) ** 2)
    src = np.zeros((2, L ** 3), dtype=np.complex128)
    src[0, idx[0]] = 1.0
    src[1, idx[0]] = 1.0
    return src


def test_oracle_branching_levels_one_is_a_plain_run():
    """levels = 1, one branch: the tree is one plain evolution of the pair."""
    L = 4
    src = _sources(L)
    wf, opp = O.two_body_tables((L,) * 3, "TGND", "STANDARD", 1.0, 0.176776695, (2.0 * O.PI) ** 2)
    a = O.run_branching(L, 1, 1, 5, 1, "RANLXS2", 3, "ZTWO", 0.5, src, wf, opp)
    b = O.run_branching(L, 1, 1, 5, 1, "RANLXS2", 3, "ZTWO", 0.5, src, wf, opp)
    assert np.array_equal(a, b)
    assert a[0] == pytest.approx(O.pair_matrix(src[:1], src[1:], wf, opp)[0, 0], rel=1e-14)


@pytest.mark.gpu
@pytest.mark.parametrize("L,levels,branches,steps,field", [(8, 3, 2, 2, "ZTWO"), (8, 2, 3, 3, "GAUSS"),
                                                           (4, 4, 2, 1, "ZTWO")])
def test_device_branching_fp64_matches_oracle(L, levels, branches, steps, field):
    import nrcps_b200 as nb
    ctx = nb.default_context()
    src = _sources(L)
    br = nb.Branching(L, levels, branches, steps, src, seed=11, field=field, a=0.5, precision="f64", ctx=ctx)
    wf, opp = O.two_body_tables((L,) * 3, "TGND", "STANDARD", 1.0, 0.176776695, (2.0 * O.PI) ** 2)
    got = br.run().cpu().numpy() + br.run().cpu().numpy()  # two trees
    ref = O.run_branching(L, levels, branches, steps, 2, "RANLXS2", 11, field, 0.5, src, wf, opp)
    assert np.max(np.abs(got - ref) / np.abs(ref)) < 1e-12
    br.close()


@pytest.mark.gpu
def test_device_branching_fp32_vs_fp64():
    import nrcps_b200 as nb
    ctx = nb.default_context()
    L = 16
    src = _sources(L)
    out = {}
    for prec in ("f32", "f64"):
        br = nb.Branching(L, 6, 2, 4, src, seed=5, field="ZTWO", a=0.5, precision=prec, ctx=ctx)
        out[prec] = br.run().cpu().numpy()
        br.close()
    assert np.max(np.abs(out["f32"] - out["f64"]) / np.abs(out["f64"])) < 1e-5


def _golden_case(g, k):
    L, levels, branches, steps, trees, seed = (int(v) for v in g[f"c{k}_params"])
    return L, levels, branches, steps, trees, seed, str(g[f"c{k}_field"])


def _local_a(L, couplings):
    """The one-coupling Interaction's (1 + a phi)/V: a = c(p) V."""
    return float(O.interaction_table((L,) * 3, 1.0, list(couplings), 1.0, (2 * O.PI) ** 2)[0] * L ** 3)


def test_oracle_branching_matches_reference_trees(golden):
    """The oracle's restatement against the reference's recursion (plane
    waves at p = 0, TGND sink), every slice to 1e-13."""
    g = golden("branching.npz")
    for k in range(int(g["cases"])):
        L, levels, branches, steps, trees, seed, field = _golden_case(g, k)
        if levels > 4:
            continue  # the deep tree runs on the device only
        src = _sources(L)
        wf, opp = O.two_body_tables((L,) * 3, "TGND", "STANDARD", 1.0, 0.176776695, (2.0 * O.PI) ** 2)
        got = O.run_branching(L, levels, branches, steps, trees, "RANLXS2", seed, field,
                              _local_a(L, g["couplings"]), src, wf, opp)
        ref = g[f"c{k}_corr"]
        assert np.max(np.abs(got - ref) / np.abs(ref)) < 1e-13, k


@pytest.mark.gpu
def test_device_branching_fp64_matches_reference_trees(golden):
    """The device tree walk in FP64 against the reference's recursion,
    including a 10-level binary tree (1024 leaves), to 1e-12 per slice."""
    import nrcps_b200 as nb
    ctx = nb.default_context()
    g = golden("branching.npz")
    for k in range(int(g["cases"])):
        L, levels, branches, steps, trees, seed, field = _golden_case(g, k)
        br = nb.Branching(L, levels, branches, steps, _sources(L), seed=seed, field=field,
                          a=_local_a(L, g["couplings"]), precision="f64", ctx=ctx)
        got = sum(br.run().cpu().numpy() for _ in range(trees))
        br.close()
        ref = g[f"c{k}_corr"]
        assert np.max(np.abs(got - ref) / np.abs(ref)) < 1e-12, k

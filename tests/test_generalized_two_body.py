"""GeneralizedTwoBody::Run (the Oh-projected pair contraction,
src/two_body/noarch/two_body_run.C:45-75) against the reference itself.

Golden fixture tests/golden/ohpair.npz (tests/golden/make_golden.py,
oracle/ref_build/ohpair_dump.cc): the reference class's tables for four
(L, distinct vector, wave function) cases -- 1, 6, 24 and 48 subshell vectors
-- random propagators and Run for all ten OctahedralReps.
CPU: the oracle's restatement of the loop; GPU: nrcps_shifted_pair_matrix
in FP64, 1e-12 of the largest |Run| of the case.
"""
import numpy as np
import pytest

from oracle import oracle as O


def _cases(golden):
    g = golden("ohpair.npz")
    for k in range(int(g["cases"])):
        yield k, {n: g[f"c{k}_{n}"] for n in ("shift", "hsw", "opp", "weights", "props", "run")}


def test_oracle_matches_reference_run(golden):
    for k, c in _cases(golden):
        if c["shift"].shape[0] > 24:  # the 48-vector case runs on the GPU only (Python loops)
            continue
        scale = np.max(np.abs(c["run"]))
        for r in (0, 3, 5, 9):
            got = O.generalized_pair(c["props"][0], c["props"][1], c["shift"], c["hsw"], c["opp"],
                                     c["weights"][:, r])
            assert abs(got - c["run"][r]) <= 1e-13 * scale, (k, r)


@pytest.mark.gpu
def test_device_matches_reference_run(golden):
    import torch
    import nrcps_b200 as nb
    ctx = nb.default_context()
    for k, c in _cases(golden):
        gtb = nb.GeneralizedTwoBody(c["shift"], c["hsw"], c["opp"], c["weights"], ctx=ctx)
        p = torch.from_numpy(c["props"]).to(ctx.device)
        scale = np.max(np.abs(c["run"]))
        for r in range(10):
            got = gtb.run(p[0], p[1], r)
            assert abs(got - c["run"][r]) <= 1e-12 * scale, (k, r)


@pytest.mark.gpu
def test_device_batched_matrix_equals_single_runs(golden):
    """[nconf, n, V] batches: every (c, s, t) element equals the single Run."""
    import torch
    import nrcps_b200 as nb
    ctx = nb.default_context()
    _, c = next(iter(_cases(golden)))
    gtb = nb.GeneralizedTwoBody(c["shift"], c["hsw"], c["opp"], c["weights"], ctx=ctx)
    rs = np.random.default_rng(2)
    V = c["opp"].size
    props = rs.standard_normal((3, 2, V)) + 1j * rs.standard_normal((3, 2, V))
    P = torch.from_numpy(props).to(ctx.device)
    phi = gtb.run_matrix(P, P, 3).cpu().numpy()
    for ci in range(3):
        for s in range(2):
            for t in range(2):
                ref = gtb.run(P[ci, s], P[ci, t], 3)
                assert abs(phi[ci, s, t] - ref) <= 1e-13 * abs(ref) + 1e-300

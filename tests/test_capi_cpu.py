"""CPU-side checks of the C ABI: the library loads, exports every symbol the
header declares, and its host-side parts (tables, seeding, skip-ahead) agree
bit-for-bit with the oracle.  No GPU compute here."""
import json
import os
import re

import numpy as np
import pytest

import nrcps_b200 as nb
from nrcps_b200 import _capi
from oracle import oracle as O

from conftest import GOLDEN, REPO

HEADER = os.path.join(REPO, "include", "nrcps_b200.h")


def test_library_exports_every_declared_symbol():
    decl = set(re.findall(r"\b(nrcps_[a-z0-9_]+)\s*\(", open(HEADER).read()))
    L = nb.lib()
    missing = [s for s in sorted(decl) if not hasattr(L, s)]
    assert not missing, missing
    # and the Python bindings cover all of them
    assert decl == set(_capi.SIGNATURES), decl ^ set(_capi.SIGNATURES)


def test_version_string():
    assert nb.lib().nrcps_version().decode().startswith("nrcps_b200")


@pytest.mark.parametrize("dims", [(16, 16, 16), (8, 8, 8), (8, 6, 4), (24, 24, 24)])
def test_tables_bit_exact(dims):
    cs2, cs1 = (2.0 * O.PI) ** 2, (0.99999 * O.PI) ** 2
    for disp in ["STANDARD", "QUADRATIC", "PERFECT"]:
        assert np.array_equal(nb.dispersion_table(dims, disp, 1.3, True, 0.99999),
                              O.dispersion(dims, disp, 1.3, True, cs1))
        assert np.array_equal(nb.kinetic_table(dims, disp, 1.0, 0.5, 2.0), O.kinetic_xi(dims, disp, 1.0, 0.5, cs2))
    for c in ([0.0198], [0.02, 0.004, 0.001]):
        for it in ["ONEMINUSXIINVSQ", "XISQMINUSONE"]:
            assert np.array_equal(nb.interaction_table(dims, 1.0, c, 1.0, 0.99999, it),
                                  O.interaction_table(dims, 1.0, c, 1.0, cs1, it))
    for pt in ["EXP", "LIN"]:
        assert np.array_equal(nb.potential_table(dims, 0.005, 0.5, pt), O.potential_table(dims, 0.005, 0.5, pt))
    for wf in ["UNIFORM", "GND", "TGND", "PAIR1", "PAIR2"]:
        w1, o1 = nb.two_body_tables(dims, wf, "STANDARD", 1.0, 0.3, 0.99999)
        w2, o2 = O.two_body_tables(dims, wf, "STANDARD", 1.0, 0.3, cs1)
        assert np.array_equal(w1, w2) and np.array_equal(o1, o2), wf


def test_momenta_and_sources_bit_exact(golden):
    g = golden("ensemble_config1.npz")
    idx, en, par = nb.momenta((16, 16, 16), "PERFECT", 1.0, 0.1, 2.0)
    mom = g["momenta"]
    assert np.array_equal(idx, mom[:, 2] + 16 * (mom[:, 1] + 16 * mom[:, 0]))
    assert np.array_equal(par, mom[:, 3])
    t = golden("ensemble_trapped.npz")
    sho = json.load(open(os.path.join(GOLDEN, "sho_coefficients.json")))
    for n in range(t["sources"].shape[0]):
        assert np.array_equal(nb.sho_source((8, 8, 8), (2.0, 2.0, 2.0), sho[str(n)]), t["sources"][n])


def test_headline_and_trapped_shape_tables_bit_exact(golden):
    """The batched workload's 19 plane waves at L=32 (E_F = 0.045) and the
    trapped workload's 10 SHO sources at L=48 (lambda = 4) against the
    reference's own (the momenta list and every 61st source entry)."""
    g = golden("ensemble_config2.npz")
    idx, _, par = nb.momenta((32, 32, 32), "PERFECT", 1.0, 0.045, 2.0)
    mom = g["momenta"]
    assert len(idx) == 19
    assert np.array_equal(idx, mom[:, 2] + 32 * (mom[:, 1] + 32 * mom[:, 0]))
    assert np.array_equal(par, mom[:, 3])
    t = golden("ensemble_trapped48.npz")
    sho = json.load(open(os.path.join(GOLDEN, "sho_coefficients.json")))
    stride = int(t["sources_stride"])
    for n in range(t["sources_sample"].shape[0]):
        got = nb.sho_source((48, 48, 48), (4.0, 4.0, 4.0), sho[str(n)])
        assert np.array_equal(got[::stride], t["sources_sample"][n]), n


@pytest.mark.parametrize("dims,wavefunc,cutoff", [((48, 48, 48), "TGND", 0.99999), ((32, 32, 32), "TGND", 2.0),
                                                   ((8, 6, 4), "TGND", 0.99999), ((16, 16, 16), "PAIR1", 0.99999)])
def test_two_body_tables_are_paired_and_even(dims, wavefunc, cutoff):
    """The pair kernels' preconditions on TwoBody's tables (host-built, as the
    ensemble and the branching driver check them): the opposite-site index is
    an involution of the lattice, so sites pair up and each orbital element is
    read once, and the weight is even under it, w(opp(i)) = w(i), so one set
    of orbitals gives a symmetric pair matrix (the upper triangle suffices)."""
    w, opp = nb.two_body_tables(dims, wavefunc, "STANDARD", 1.0, 0.176776695, cutoff)
    vol = int(np.prod(dims))
    assert opp.min() >= 0 and opp.max() < vol
    assert np.array_equal(opp[opp], np.arange(vol))
    assert np.array_equal(w[opp], w)


def test_momenta_errors():
    with pytest.raises(nb.NrcpsError):
        nb.momenta((16, 16, 16), "PERFECT", 1.0, -1.0, 2.0)  # nothing below the Fermi level
    with pytest.raises(nb.NrcpsError):
        nb.kinetic_table((15, 16, 16))  # odd extent (global_job_parameter.C:40-42)


@pytest.mark.parametrize("kind", ["RANLXS0", "RANLXS1", "RANLXS2", "RANLXD1", "RANLXD2"])
def test_seed_state_and_skip_ahead_bit_exact(kind):
    st = nb.rng_seed_state(kind, 1234)
    r = O.Rng(kind, 1234)
    assert np.array_equal(st, r.get_state())
    for n in [1, 47, 48, 49, 95, 96, 97, 1000, 54321, 300_000]:
        st = nb.rng_skip(kind, st, n)
        for _ in range(n):
            r.uniform()
        assert np.array_equal(st, r.get_state()), n


def test_skip_ahead_matches_known_answer(golden):
    """Jump straight to Luscher's published ranlxs block (no serial draws)."""
    k = golden("ranlx_kat.npz")
    first = int(k["ranlxs0_seed32767_first_index"])
    st = nb.rng_skip("RANLXS0", nb.rng_seed_state("RANLXS0", 32767), first)
    r = O.Rng("RANLXS0", 1)
    r.set_state(st)
    got = np.array([r.uniform() for _ in range(96)]) * 2.0 ** 24
    assert np.array_equal(got, k["ranlxs0_seed32767_times_2p24"])


def test_ran2_seed_state_matches_oracle():
    st = nb.rng_seed_state("RAN2", 77)
    assert st.size == 36 and st[0] == 36


def test_bad_seed_rejected():
    with pytest.raises(nb.NrcpsError):
        nb.rng_seed_state("RANLXS2", 0)

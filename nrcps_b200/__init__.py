"""nrcps_b200 -- B200 (sm_100a) implementation of nrCPS's auxiliary-field
transfer-matrix hot path behind the reference's class API.

    import nrcps_b200 as nb
    ens = nb.Ensemble(nb.EnsembleJob(L=32, T=64, n_conf=4096, precision="f32"), plane_wave_index=idx)
    dets = ens.run()            # [n_conf, T, N] raw Slater determinants

The numerical work lives in libnrcps_b200.so (C ABI: include/nrcps_b200.h);
this package only binds it.  Build with ``python -m nrcps_b200.build``.
"""
from ._capi import NrcpsError, lib  # noqa: F401
from .api import (  # noqa: F401
    Batch, BatchJob, Branching, Context, GeneralizedTwoBody, Ensemble, EnsembleJob, accumulate, jackknife, reorthonormalise, Fourier, Interaction, Kinetic, Lattice, OneBody, Potential, Propagator,
    Random, SlaterDet, TwoBody, cutoff_sq, default_context, dispersion_table, draw_fields, draw_z2_bits,
    interaction_table, kinetic_table, momenta, overlap, propagate, overlap_planewave, potential_table, rng_seed_state,
    rng_skip, sho_source, slater_dets, two_body_tables, uniforms,
)

__version__ = "0.1.0"

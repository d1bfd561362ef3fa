"""ctypes front end of the oracle restatement (oracle/oracle.c).

TEST INFRASTRUCTURE ONLY.  This module is the checker for the B200 library:
tests/, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` leg of bench.py
may import it, and only to compare the library's results against it.  The
product package (``nrcps_b200``) never imports it.

Each wrapper names the reference function it restates (mgendres/nrCPS v2_7_6,
file:line); the C file carries the detailed citations.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass, field as dc_field

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_SO = os.path.join(_HERE, "_build", "liboracle.so")

RNG_KINDS = {
    "RAN0": 0, "RAN1": 1, "RAN2": 2, "RAN3": 3,
    "RANLXS0": 4, "RANLXS1": 5, "RANLXS2": 6, "RANLXD1": 7, "RANLXD2": 8,
}
FIELD_TYPES = {"GAUSS": 0, "COMPLEXGAUSS": 1, "ZTWO": 2, "ZTHREE": 3}
DISP_TYPES = {"STANDARD": 0, "QUADRATIC": 1, "PERFECT": 2}
WAVEFUNC_TYPES = {"NONE": 0, "UNIFORM": 1, "GND": 2, "TGND": 3, "PAIR1": 4, "PAIR2": 5}
PI = 3.1415926535897932  # include/constants.h:12


def build() -> str:
    """Compiles liboracle.so if it is missing (gcc only)."""
    if not os.path.exists(_SO):
        subprocess.check_call(["make", "-s", "-C", _HERE])
    return _SO


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(_SO)
        dp = ctypes.POINTER(ctypes.c_double)
        ip = ctypes.POINTER(ctypes.c_int)
        L.o_uniforms.argtypes = [ctypes.c_int, ctypes.c_long, ctypes.c_long, ctypes.c_long, dp]
        L.o_gaussians.argtypes = [ctypes.c_int, ctypes.c_long, ctypes.c_long, ctypes.c_long, dp]
        L.o_rng_init.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_long]
        L.o_rng_uniform.argtypes = [ctypes.c_void_p]
        L.o_rng_uniform.restype = ctypes.c_double
        L.o_rng_get_state.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_long)]
        L.o_rng_set_state.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_long)]
        L.o_field_slices.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_long, ctypes.c_long, dp]
        L.o_dispersion.argtypes = [ip, ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.c_double, dp]
        L.o_kinetic_xi.argtypes = [ip, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double, dp]
        L.o_interaction_table.argtypes = [ip, ctypes.c_double, ctypes.c_int, dp, ctypes.c_int,
                                          ctypes.c_double, ctypes.c_double, dp]
        L.o_potential_table.argtypes = [ip, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                        ctypes.c_double, ctypes.c_double, dp]
        L.o_momenta.argtypes = [ip, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                ip, dp, ip, ctypes.c_int]
        L.o_sho_source.argtypes = [ip, ctypes.c_double, ctypes.c_double, ctypes.c_double, dp, dp]
        L.o_dawson.argtypes = [ctypes.c_double]
        L.o_dawson.restype = ctypes.c_double
        L.o_two_body_tables.argtypes = [ip, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                        ctypes.c_double, ctypes.c_double, ctypes.c_double, dp, ip]
        L.o_interaction_initialize.argtypes = [ip, dp, dp, dp]
        L.o_kinetic_evolve.argtypes = [ctypes.c_long, ctypes.c_int, dp, dp]
        L.o_potential_evolve.argtypes = [ip, ctypes.c_int, dp, dp]
        L.o_interaction_evolve.argtypes = [ip, ctypes.c_int, dp, dp]
        L.o_project.argtypes = [ctypes.c_long, ctypes.c_int, dp, ctypes.c_int, dp, dp]
        L.o_pair_matrix.argtypes = [ctypes.c_long, ctypes.c_int, dp, dp, dp, ip, dp]
        L.o_ludcmp.argtypes = [dp, ctypes.c_int, ip, dp]
        L.o_minor_det.argtypes = [dp, ctypes.c_int, ctypes.c_int, ctypes.c_int, dp, ctypes.c_int, dp]
        L.o_fft3d.argtypes = [dp, ip, ctypes.c_int, ctypes.c_int]
        L.o_run_ensemble.argtypes = [ctypes.c_void_p, dp, dp]
        L.o_run_branching.argtypes = [ip, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                      ctypes.c_long, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                      ctypes.c_double, dp, dp, ip, dp]
        pp = ctypes.POINTER(ctypes.POINTER(ctypes.c_int))
        L.o_run_batch.argtypes = [ctypes.c_int, ip, ip, ip, ip, pp, ctypes.c_int, ctypes.c_long, ctypes.c_int,
                                  ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                  ctypes.POINTER(ctypes.POINTER(ctypes.c_double))]
        L.o_run_ensemble.restype = ctypes.c_int
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _ip(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


def _dims(dims):
    return np.ascontiguousarray(np.asarray(dims, dtype=np.int32))


# ---------------------------------------------------------------- RNG
class Rng:
    """Random + UniformDeviate (src/random/random.C:12-132)."""

    _SIZE = 4096  # >= sizeof(o_rng)

    def __init__(self, kind: str, seed: int):
        self._buf = ctypes.create_string_buffer(self._SIZE)
        lib().o_rng_init(self._buf, RNG_KINDS[kind], seed)

    def uniform(self) -> float:
        return lib().o_rng_uniform(self._buf)

    def get_state(self) -> np.ndarray:
        st = np.zeros(105, dtype=np.int64)
        lib().o_rng_get_state(self._buf, st.ctypes.data_as(ctypes.POINTER(ctypes.c_long)))
        return st

    def set_state(self, st) -> None:
        st = np.ascontiguousarray(st, dtype=np.int64)
        lib().o_rng_set_state(self._buf, st.ctypes.data_as(ctypes.POINTER(ctypes.c_long)))

    def fields(self, field_type: str, vol: int, slices: int) -> np.ndarray:
        out = np.zeros(slices * 2 * vol)
        lib().o_field_slices(self._buf, FIELD_TYPES[field_type], vol, slices, _dp(out))
        return out.reshape(slices, vol, 2)


def uniforms(kind: str, seed: int, count: int, skip: int = 0) -> np.ndarray:
    out = np.zeros(count)
    lib().o_uniforms(RNG_KINDS[kind], seed, skip, count, _dp(out))
    return out


def gaussians(kind: str, seed: int, count: int, skip: int = 0) -> np.ndarray:
    out = np.zeros(count)
    lib().o_gaussians(RNG_KINDS[kind], seed, skip, count, _dp(out))
    return out


def field_slices(kind: str, seed: int, field_type: str, vol: int, slices: int) -> np.ndarray:
    """Lattice constructor draw + (slices-1) Refresh calls: [slices, vol, 2]."""
    return Rng(kind, seed).fields(field_type, vol, slices)


# ---------------------------------------------------------------- tables
def dispersion(dims, dtype: str, mass: float, hard_cutoff: bool, cutoff_sq: float) -> np.ndarray:
    out = np.zeros(int(np.prod(dims)))
    lib().o_dispersion(_ip(_dims(dims)), DISP_TYPES[dtype], mass, int(hard_cutoff), cutoff_sq, _dp(out))
    return out


def kinetic_xi(dims, dtype: str, mass: float, dt: float, cutoff_sq: float) -> np.ndarray:
    out = np.zeros(int(np.prod(dims)))
    lib().o_kinetic_xi(_ip(_dims(dims)), DISP_TYPES[dtype], mass, dt, cutoff_sq, _dp(out))
    return out


def interaction_table(dims, mass: float, couplings, dt: float, cutoff_sq: float,
                      itype: str = "ONEMINUSXIINVSQ") -> np.ndarray:
    c = np.ascontiguousarray(np.asarray(couplings, dtype=np.float64))
    out = np.zeros(int(np.prod(dims)))
    t = 1 if itype == "XISQMINUSONE" else 2
    lib().o_interaction_table(_ip(_dims(dims)), mass, t, _dp(c), len(c), dt, cutoff_sq, _dp(out))
    return out


def potential_table(dims, kappa, dt: float, ptype: str = "EXP") -> np.ndarray:
    k = list(kappa) if np.ndim(kappa) else [kappa] * 3
    out = np.zeros(int(np.prod(dims)))
    lib().o_potential_table(_ip(_dims(dims)), 1 if ptype == "EXP" else 0, k[0], k[1], k[2], dt, _dp(out))
    return out


def momenta(dims, dtype: str, mass: float, fermi_energy: float, cutoff_sq: float):
    cap = int(np.prod(dims))
    idx = np.zeros(cap, dtype=np.int32)
    en = np.zeros(cap)
    par = np.zeros(cap, dtype=np.int32)
    n = lib().o_momenta(_ip(_dims(dims)), DISP_TYPES[dtype], mass, fermi_energy, cutoff_sq,
                        _ip(idx), _dp(en), _ip(par), cap)
    return idx[:n].copy(), en[:n].copy(), par[:n].copy()


def plane_wave_sources(dims, idx) -> np.ndarray:
    """OneBody::Set(n1,n2,n3) (src/one_body/one_body.C:215-228): unit delta in momentum space."""
    vol = int(np.prod(dims))
    src = np.zeros((len(idx), vol), dtype=np.complex128)
    for n, j in enumerate(idx):
        src[n, j] = 1.0
    return src


def sho_source(dims, lambdas, coeff_lines) -> np.ndarray:
    """OneBody::Set(string) + SHO branch; coeff_lines = [(n1, n2, n3, re, im), ...]."""
    vol = int(np.prod(dims))
    X, Y, Z = dims
    co = np.zeros(2 * vol)
    for n1, n2, n3, re, im in coeff_lines:
        j = (n3 % Z) + Z * ((n2 % Y) + Y * (n1 % X))
        co[2 * j] = re
        co[2 * j + 1] = im
    out = np.zeros(2 * vol)
    lib().o_sho_source(_ip(_dims(dims)), lambdas[0], lambdas[1], lambdas[2], _dp(co), _dp(out))
    return out.view(np.complex128)


def dawson(x: float) -> float:
    return lib().o_dawson(x)


def two_body_tables(dims, wf_type: str, disp: str, mass: float, lam: float, cutoff_sq: float):
    vol = int(np.prod(dims))
    wf = np.zeros(vol)
    opp = np.zeros(vol, dtype=np.int32)
    lib().o_two_body_tables(_ip(_dims(dims)), WAVEFUNC_TYPES[wf_type], DISP_TYPES[disp], DISP_TYPES[disp],
                            mass, mass, lam, cutoff_sq, _dp(wf), _ip(opp))
    return wf, opp


# ---------------------------------------------------------------- propagation
def fft3d(data: np.ndarray, sign: int) -> np.ndarray:
    """Unnormalised FFTW-convention transform of [batch, X, Y, Z] complex data."""
    a = np.ascontiguousarray(data, dtype=np.complex128).copy()
    dims = _dims(a.shape[-3:])
    batch = int(np.prod(a.shape[:-3])) if a.ndim > 3 else 1
    lib().o_fft3d(_dp(a.view(np.float64)), _ip(dims), batch, sign)
    return a


def interaction_initialize(dims, lat: np.ndarray, itab: np.ndarray) -> np.ndarray:
    lat = np.ascontiguousarray(lat, dtype=np.float64).reshape(-1)
    itab = np.ascontiguousarray(itab, dtype=np.float64)
    fld = np.zeros(lat.size)
    lib().o_interaction_initialize(_ip(_dims(dims)), _dp(lat), _dp(itab), _dp(fld))
    return fld.view(np.complex128)


def kinetic_evolve(psi: np.ndarray, xi: np.ndarray) -> np.ndarray:
    a = np.ascontiguousarray(psi, dtype=np.complex128).copy()
    vol = xi.size
    lib().o_kinetic_evolve(vol, a.size // vol, _dp(a.view(np.float64)), _dp(np.ascontiguousarray(xi)))
    return a


def potential_evolve(dims, psi: np.ndarray, pot: np.ndarray) -> np.ndarray:
    a = np.ascontiguousarray(psi, dtype=np.complex128).copy()
    vol = pot.size
    lib().o_potential_evolve(_ip(_dims(dims)), a.size // vol, _dp(a.view(np.float64)),
                             _dp(np.ascontiguousarray(pot)))
    return a


def interaction_evolve(dims, psi: np.ndarray, fld: np.ndarray) -> np.ndarray:
    a = np.ascontiguousarray(psi, dtype=np.complex128).copy()
    f = np.ascontiguousarray(fld, dtype=np.complex128)
    vol = f.size
    lib().o_interaction_evolve(_ip(_dims(dims)), a.size // vol, _dp(a.view(np.float64)),
                               _dp(f.view(np.float64)))
    return a


# ---------------------------------------------------------------- measurement
def project(src: np.ndarray, psi: np.ndarray) -> np.ndarray:
    src = np.ascontiguousarray(src, dtype=np.complex128)
    psi = np.ascontiguousarray(psi, dtype=np.complex128)
    ns, nt, vol = src.shape[0], psi.shape[0], src.shape[-1]
    S = np.zeros((ns, nt), dtype=np.complex128)
    lib().o_project(vol, ns, _dp(src.view(np.float64)), nt, _dp(psi.view(np.float64)),
                    _dp(S.view(np.float64)))
    return S


def pair_matrix(psi1, psi2, wf, opp) -> np.ndarray:
    psi1 = np.ascontiguousarray(psi1, dtype=np.complex128)
    psi2 = np.ascontiguousarray(psi2, dtype=np.complex128)
    n, vol = psi1.shape[0], psi1.shape[-1]
    phi = np.zeros((n, n), dtype=np.complex128)
    lib().o_pair_matrix(vol, n, _dp(psi1.view(np.float64)), _dp(psi2.view(np.float64)),
                        _dp(np.ascontiguousarray(wf)), _ip(np.ascontiguousarray(opp, dtype=np.int32)),
                        _dp(phi.view(np.float64)))
    return phi


def ludcmp(a: np.ndarray):
    """ludcmp (src/utils/ludcmp.C:9-65): returns (LU, indx, d, singular)."""
    m = np.ascontiguousarray(a, dtype=np.complex128).copy()
    n = m.shape[0]
    indx = np.zeros(n, dtype=np.int32)
    d = np.zeros(1)
    bad = lib().o_ludcmp(_dp(m.view(np.float64)), n, _ip(indx), _dp(d))
    return m, indx, float(d[0]), bool(bad)


def minor_det(S: np.ndarray, n: int, t0: int = -1, psi1=None, log: bool = False) -> complex:
    S = np.ascontiguousarray(S, dtype=np.complex128)
    N = S.shape[0]
    p1 = np.ascontiguousarray(psi1 if psi1 is not None else np.zeros((N, N)), dtype=np.complex128)
    out = np.zeros(2)
    lib().o_minor_det(_dp(S.view(np.float64)), N, n, t0, _dp(p1.view(np.float64)), int(log), _dp(out))
    return complex(out[0], out[1])


# ----------------------------------------------------- generalized pair
def generalized_pair(p1: np.ndarray, p2: np.ndarray, shift: np.ndarray, hsw: np.ndarray, opp: np.ndarray,
                     weights_R: np.ndarray) -> complex:
    """GeneralizedTwoBody::Run(prop1, prop2, R) (src/two_body/noarch/two_body_run.C:45-75):
    sum over subshell vectors l (outer) and sites i (inner) of
    weight(R, l) * prop1[shift[l][i]] * prop2[opp[i]] * hsw[l][i], accumulated
    in that order (pure Python loops: small lattices only)."""
    re = im = 0.0
    a, b = np.asarray(p1, dtype=np.complex128), np.asarray(p2, dtype=np.complex128)
    for l in range(shift.shape[0]):
        w = float(weights_R[l])
        for i in range(shift.shape[1]):
            x, y, h = a[shift[l, i]], b[opp[i]], float(hsw[l, i])
            re += w * (x.real * y.real - x.imag * y.imag) * h
            im += w * (x.real * y.imag + x.imag * y.real) * h
    return complex(re, im)


# ------------------------------------------------------------- branching
def run_branching(L: int, levels: int, branches: int, steps: int, trees: int, rng: str, seed: int, field: str,
                  a: float, sources2: np.ndarray, wf: np.ndarray, opp: np.ndarray, kin_dt: float = 0.5,
                  cutoff: float = 2.0) -> np.ndarray:
    """MultiLevel trees (o_run_branching): corr [levels * steps] complex, summed over trees."""
    dims = np.array([L, L, L], dtype=np.int32)
    src = np.ascontiguousarray(sources2, dtype=np.complex128).reshape(2, -1)
    corr = np.zeros(levels * steps, dtype=np.complex128)
    c = cutoff * PI
    lib().o_run_branching(dims.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), levels, branches, steps, trees,
                          RNG_KINDS[rng], seed, FIELD_TYPES[field], a, kin_dt, c * c, _dp(src.view(np.float64)),
                          _dp(np.ascontiguousarray(wf, dtype=np.float64)),
                          np.ascontiguousarray(opp, dtype=np.int32).ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                          _dp(corr.view(np.float64)))
    return corr


# ----------------------------------------------------------------- batch
def run_batch(jobs, rng: str, seed: int, field: str, a: float, kin_dt: float = 0.5, cutoff: float = 2.0):
    """Jobs one after another with one generator (o_run_batch): jobs = list of
    (L, T, n_conf, plane-wave index list); returns one [n_conf, T, N] complex
    array per job."""
    n = len(jobs)
    Ls = (ctypes.c_int * n)(*[j[0] for j in jobs])
    Ts = (ctypes.c_int * n)(*[j[1] for j in jobs])
    Cs = (ctypes.c_int * n)(*[j[2] for j in jobs])
    Ns = (ctypes.c_int * n)(*[len(j[3]) for j in jobs])
    idx = [np.ascontiguousarray(np.asarray(j[3], dtype=np.int32)) for j in jobs]
    idx_p = (ctypes.POINTER(ctypes.c_int) * n)(*[i.ctypes.data_as(ctypes.POINTER(ctypes.c_int)) for i in idx])
    outs = [np.zeros((j[2], j[1], len(j[3])), dtype=np.complex128) for j in jobs]
    out_p = (ctypes.POINTER(ctypes.c_double) * n)(*[_dp(o.view(np.float64)) for o in outs])
    c = cutoff * PI
    lib().o_run_batch(n, Ls, Ts, Cs, Ns, idx_p, RNG_KINDS[rng], seed, FIELD_TYPES[field], ctypes.c_double(a),
                      ctypes.c_double(kin_dt), ctypes.c_double(c * c), out_p)
    return outs


# ------------------------------------------------------------ estimators
def block_sums(dets: np.ndarray, mode: str = "slater", n_cumulants: int = 0):
    """The production drivers' per-block accumulation, configuration by
    configuration in index order (pure Python loops; small inputs only):
    corr[m][t] += tmp * conj(tmp)            production/slater_det/main.C:208-211 (mode 'slater')
    corr[m][t] += slat                       production/slater_det2_trapped/main-no_cum.C:205-207
    cum[0] = log(abs(slat)); cum[k] = cum[0] * cum[k-1]; z[k][m][t] += cum[k]
                                             production/slater_det2_trapped/main-cum.C:219-233
    dets [n_conf, T, nmeas] complex -> corr [nmeas, T] complex, z [Nc, nmeas, T] real."""
    d = np.asarray(dets, dtype=np.complex128)
    n_conf, T, nmeas = d.shape
    corr = np.zeros((nmeas, T), dtype=np.complex128)
    z = np.zeros((n_cumulants, nmeas, T))
    for c in range(n_conf):
        for t in range(T):
            for m in range(nmeas):
                v = d[c, t, m]
                corr[m, t] += (v * np.conj(v)).real if mode == "slater" else v
                if n_cumulants:
                    cum = np.log(abs(v))
                    p = cum
                    for k in range(n_cumulants):
                        z[k, m, t] += p
                        p = cum * p
    return corr, z


# ---------------------------------------------------------------- ensemble
class _OJob(ctypes.Structure):
    _fields_ = [
        ("dims", ctypes.c_int * 3), ("T", ctypes.c_int), ("n_orb", ctypes.c_int),
        ("configs", ctypes.c_int), ("rng_kind", ctypes.c_int), ("seed", ctypes.c_long),
        ("field_type", ctypes.c_int), ("kin_mass", ctypes.c_double), ("kin_dt", ctypes.c_double),
        ("kin_disp", ctypes.c_int), ("cutoff_sq", ctypes.c_double), ("int_mass", ctypes.c_double),
        ("int_dt", ctypes.c_double), ("int_type", ctypes.c_int), ("n_coup", ctypes.c_int),
        ("coup", ctypes.c_double * 8), ("use_potential", ctypes.c_int), ("pot_type", ctypes.c_int),
        ("pot_k", ctypes.c_double * 3), ("pot_dt", ctypes.c_double), ("mode", ctypes.c_int),
        ("wf_type", ctypes.c_int), ("wf_disp", ctypes.c_int), ("wf_mass", ctypes.c_double),
        ("wf_lambda", ctypes.c_double),
    ]


@dataclass
class Job:
    """One ensemble run, with the reference's argument meanings (include/arg.h)."""
    L: int = 16
    T: int = 32
    configs: int = 1
    rng: str = "RANLXS2"
    seed: int = 1234
    field: str = "ZTWO"
    kin_disp: str = "PERFECT"
    kin_mass: float = 1.0
    kin_dt: float = 0.5
    cutoff: float = 2.0  # units of pi (DoArg.cutoff)
    int_mass: float = 1.0
    int_dt: float = 1.0
    int_type: str = "ONEMINUSXIINVSQ"
    couplings: list = dc_field(default_factory=lambda: [0.019894367886486918])
    potential: bool = False
    pot_type: str = "EXP"
    kappa: float = 0.005
    pot_dt: float = 0.5
    mode: str = "slater"  # or "slater2"
    wavefunc: str = "TGND"
    wf_disp: str = "STANDARD"
    wf_mass: float = 1.0
    wf_lambda: float = 0.176776695

    @property
    def dims(self):
        return (self.L, self.L, self.L)

    @property
    def cutoff_sq(self) -> float:
        c = self.cutoff * PI
        return c * c


def run_ensemble(job: Job, sources: np.ndarray) -> np.ndarray:
    """production/slater_det/main.C loop; returns dets[config, t, m] (complex)."""
    src = np.ascontiguousarray(sources, dtype=np.complex128)
    N = src.shape[0]
    o = _OJob()
    o.dims[:] = job.dims
    o.T, o.n_orb, o.configs = job.T, N, job.configs
    o.rng_kind, o.seed, o.field_type = RNG_KINDS[job.rng], job.seed, FIELD_TYPES[job.field]
    o.kin_mass, o.kin_dt, o.kin_disp = job.kin_mass, job.kin_dt, DISP_TYPES[job.kin_disp]
    o.cutoff_sq = job.cutoff_sq
    o.int_mass, o.int_dt = job.int_mass, job.int_dt
    o.int_type = 1 if job.int_type == "XISQMINUSONE" else 2
    o.n_coup = len(job.couplings)
    for i, c in enumerate(job.couplings):
        o.coup[i] = c
    o.use_potential, o.pot_type = int(job.potential), 1 if job.pot_type == "EXP" else 0
    o.pot_k[:] = (job.kappa,) * 3
    o.pot_dt = job.pot_dt
    o.mode = 1 if job.mode == "slater2" else 0
    o.wf_type, o.wf_disp = WAVEFUNC_TYPES[job.wavefunc], DISP_TYPES[job.wf_disp]
    o.wf_mass, o.wf_lambda = job.wf_mass, job.wf_lambda
    nmeas = 2 * N if o.mode else N
    dets = np.zeros((job.configs, job.T, nmeas), dtype=np.complex128)
    lib().o_run_ensemble(ctypes.byref(o), _dp(src.view(np.float64)), _dp(dets.view(np.float64)))
    return dets

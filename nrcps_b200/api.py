"""Python host API over the C ABI, mirroring the reference's class API.

The reference (mgendres/nrCPS v2_7_6) exposes its hot path as C++ classes
(include/fourier.h, hamiltonian.h, propagator.h, lattice.h, random.h,
one_body.h, two_body.h, slater_det.h).  The classes below keep those names,
argument meanings and call order so that scripts and tests read like the
reference's drivers; every numerical operation is a call into
libnrcps_b200.so.  Device memory is held in torch tensors (complex128 /
complex64 are interleaved (re, im), the layout the library expects).
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field as dc_field
from typing import Optional, Sequence

import numpy as np
import torch

from . import _capi as C
from ._capi import check, lib

PI = 3.1415926535897932  # include/constants.h:12


def _ip(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


def _dp(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _dims(dims) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(dims, dtype=np.int32).reshape(3))


def _ptr(t: Optional[torch.Tensor]):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


def cutoff_sq(cutoff: float) -> float:
    """GJP.CutoffSq() for DoArg.cutoff in units of pi (global_job_parameter.C:48,112)."""
    c = cutoff * PI
    return c * c


# --------------------------------------------------------------------- context
class Context:
    """One device, one stream (torch's current stream by default)."""

    def __init__(self, device: int = 0):
        if not torch.cuda.is_available():
            raise RuntimeError("nrcps_b200 needs a CUDA device")
        self.device = torch.device("cuda", device)
        h = ctypes.c_void_p()
        check(lib().nrcps_create(device, ctypes.byref(h)), None, "nrcps_create")
        self.handle = h
        self.use_current_stream()

    def use_current_stream(self) -> None:
        s = torch.cuda.current_stream(self.device).cuda_stream
        check(lib().nrcps_set_stream(self.handle, ctypes.c_void_p(s)), self.handle, "nrcps_set_stream")

    def check(self, status: int, what: str = "") -> None:
        check(status, self.handle, what)

    def synchronize(self) -> None:
        self.check(lib().nrcps_synchronize(self.handle), "synchronize")

    def set_option(self, name: str, value: int) -> None:
        """nrcps_set_option: "propagate.fused" (1/0), "fused.cluster" (0 = autotuned),
        "fused.split" (-1 = autotuned, 0, 1), "fused.kind" (-1 = autotuned, 0..12)."""
        self.check(lib().nrcps_set_option(self.handle, name.encode(), int(value)), "set_option")

    def autotune(self, precision: str, L: int) -> int:
        """Times the fused kernel's cluster sizes for (precision, L); returns the chosen one."""
        c = ctypes.c_int()
        self.check(lib().nrcps_autotune(self.handle, _prec(precision), L, ctypes.byref(c)), "autotune")
        return c.value

    def fused_choice(self, precision: str, L: int):
        """(kind, cluster) of the fused kernel nrcps_propagate runs for (precision, L^3); (-1, -1) if none."""
        k, c = ctypes.c_int(), ctypes.c_int()
        self.check(lib().nrcps_fused_choice(self.handle, _prec(precision), L, ctypes.byref(k), ctypes.byref(c)),
                   "fused_choice")
        return k.value, c.value

    def close(self) -> None:
        if self.handle:
            lib().nrcps_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_default_ctx: Optional[Context] = None


def default_context() -> Context:
    global _default_ctx
    if _default_ctx is None:
        _default_ctx = Context(torch.cuda.current_device())
    return _default_ctx


# ---------------------------------------------------------------- host tables
def dispersion_table(dims, dtype: str = "PERFECT", mass: float = 1.0, hard_cutoff: bool = True,
                     cutoff: float = 2.0) -> np.ndarray:
    """Dispersion (src/alg/dispersion.C:11-75)."""
    d = _dims(dims)
    out = np.zeros(int(np.prod(d)))
    check(lib().nrcps_dispersion_table(_ip(d), C.DISP_TYPES[dtype], mass, int(hard_cutoff), cutoff_sq(cutoff),
                                       _dp(out)), None, "dispersion_table")
    return out


def kinetic_table(dims, dtype: str = "PERFECT", mass: float = 1.0, dt: float = 0.5, cutoff: float = 2.0) -> np.ndarray:
    """Kinetic's xi(p) = 1 + disp(m/dt) (src/hamiltonian/hamiltonian.C:260-281)."""
    d = _dims(dims)
    out = np.zeros(int(np.prod(d)))
    check(lib().nrcps_kinetic_table(_ip(d), C.DISP_TYPES[dtype], mass, dt, cutoff_sq(cutoff), _dp(out)), None,
          "kinetic_table")
    return out


def interaction_table(dims, mass: float = 1.0, couplings: Sequence[float] = (0.019894367886486918,),
                      dt: float = 1.0, cutoff: float = 2.0, itype: str = "ONEMINUSXIINVSQ") -> np.ndarray:
    """Interaction's momentum factor c(p) (src/hamiltonian/hamiltonian.C:77-147)."""
    d = _dims(dims)
    c = np.ascontiguousarray(np.asarray(couplings, dtype=np.float64))
    out = np.zeros(int(np.prod(d)))
    check(lib().nrcps_interaction_table(_ip(d), mass, C.INTERACTION_TYPES[itype], _dp(c), len(c), dt,
                                        cutoff_sq(cutoff), _dp(out)), None, "interaction_table")
    return out


def potential_table(dims, kappa=0.005, dt: float = 0.5, ptype: str = "EXP") -> np.ndarray:
    """Harmonic Potential incl. 1/V (src/hamiltonian/hamiltonian.C:165-244)."""
    d = _dims(dims)
    k = list(kappa) if np.ndim(kappa) else [kappa] * 3
    out = np.zeros(int(np.prod(d)))
    check(lib().nrcps_potential_table(_ip(d), C.POTENTIAL_TYPES[ptype], k[0], k[1], k[2], dt, _dp(out)), None,
          "potential_table")
    return out


def momenta(dims, dtype: str = "PERFECT", mass: float = 1.0, fermi_energy: float = 0.1, cutoff: float = 2.0):
    """Momenta below the Fermi energy, energy-sorted (src/alg/momenta.C:12-139)."""
    d = _dims(dims)
    cap = int(np.prod(d))
    idx = np.zeros(cap, dtype=np.int32)
    en = np.zeros(cap)
    par = np.zeros(cap, dtype=np.int32)
    n = ctypes.c_int()
    check(lib().nrcps_momenta(_ip(d), C.DISP_TYPES[dtype], mass, fermi_energy, cutoff_sq(cutoff), cap, _ip(idx),
                              _dp(en), _ip(par), ctypes.byref(n)), None, "momenta")
    k = n.value
    return idx[:k].copy(), en[:k].copy(), par[:k].copy()


def sho_source(dims, lambdas, coeff_lines) -> np.ndarray:
    """OneBody::Set(file) for SHO sources (src/one_body/one_body.C:53-213)."""
    d = _dims(dims)
    X, Y, Z = (int(v) for v in d)
    vol = X * Y * Z
    co = np.zeros(2 * vol)
    for n1, n2, n3, re, im in coeff_lines:
        j = (int(n3) % Z) + Z * ((int(n2) % Y) + Y * (int(n1) % X))
        co[2 * j], co[2 * j + 1] = re, im
    out = np.zeros(2 * vol)
    check(lib().nrcps_sho_source(_ip(d), lambdas[0], lambdas[1], lambdas[2], _dp(co), _dp(out)), None, "sho_source")
    return out.view(np.complex128)


def two_body_tables(dims, wavefunc: str = "TGND", disp: str = "STANDARD", mass: float = 1.0,
                    lam: float = 0.176776695, cutoff: float = 0.99999):
    """TwoBody's pair wave function and opposite-parity index (src/two_body/two_body.C:21-141)."""
    d = _dims(dims)
    vol = int(np.prod(d))
    w = np.zeros(vol)
    opp = np.zeros(vol, dtype=np.int32)
    check(lib().nrcps_two_body_tables(_ip(d), C.WAVEFUNC_TYPES[wavefunc], C.DISP_TYPES[disp], C.DISP_TYPES[disp],
                                      mass, mass, lam, cutoff_sq(cutoff), _dp(w), _ip(opp)), None, "two_body_tables")
    return w, opp


# ------------------------------------------------------------------------ RNG
def rng_seed_state(kind: str, seed: int) -> np.ndarray:
    st = np.zeros(105, dtype=np.int64)
    n = ctypes.c_int()
    check(lib().nrcps_rng_seed_state(C.RNG_KINDS[kind], seed, st.ctypes.data_as(ctypes.POINTER(ctypes.c_long)),
                                     ctypes.byref(n)), None, "rng_seed_state")
    return st[: n.value].copy()


def rng_skip(kind: str, state: np.ndarray, n: int) -> np.ndarray:
    st = np.ascontiguousarray(state, dtype=np.int64).copy()
    check(lib().nrcps_rng_skip(C.RNG_KINDS[kind], st.ctypes.data_as(ctypes.POINTER(ctypes.c_long)), n), None,
          "rng_skip")
    return st


def uniforms(kind: str, seed: int, count: int, offset: int = 0, ctx: Optional[Context] = None) -> torch.Tensor:
    ctx = ctx or default_context()
    out = torch.empty(count, dtype=torch.float64, device=ctx.device)
    ctx.check(lib().nrcps_rng_uniforms(ctx.handle, C.RNG_KINDS[kind], seed, offset, count, _ptr(out)), "uniforms")
    return out


def draw_fields(kind: str, seed: int, field: str, vol: int, slices: int, offset: int = 0,
                ctx: Optional[Context] = None):
    """Lattice::Refresh slices on the GPU: ([slices, vol, 2] float64, next stream offset)."""
    ctx = ctx or default_context()
    out = torch.empty((slices, vol, 2), dtype=torch.float64, device=ctx.device)
    off = ctypes.c_uint64(offset)
    ctx.check(lib().nrcps_draw_fields(ctx.handle, C.RNG_KINDS[kind], seed, C.FIELD_KINDS[field], vol, slices,
                                      ctypes.byref(off), _ptr(out)), "draw_fields")
    return out, off.value


def draw_z2_bits(kind: str, seed: int, first: int, count: int, ctx: Optional[Context] = None) -> torch.Tensor:
    ctx = ctx or default_context()
    out = torch.empty((count + 31) // 32, dtype=torch.int32, device=ctx.device)
    ctx.check(lib().nrcps_draw_z2_bits(ctx.handle, C.RNG_KINDS[kind], seed, first, count, _ptr(out)), "draw_z2_bits")
    return out


# ------------------------------------------------------------- class mirrors
def _cdtype(precision: str):
    return torch.complex128 if precision == "f64" else torch.complex64


def _prec(precision: str) -> int:
    return C.F64 if precision == "f64" else C.F32


class Random:
    """Random (src/random/random.C:12-93): generator kind, seed (+491*rank) and stream position."""

    def __init__(self, kind: str = "RANLXS2", seed: int = 1234, rank: int = 0):
        self.kind = kind
        self.seed = seed + 491 * rank
        self.offset = 0


class Lattice:
    """Lattice (src/alg/lattice.C): one field slice, drawn on the GPU from the Random stream."""

    def __init__(self, dims, rng: Random, field: str = "ZTWO", ctx: Optional[Context] = None):
        self.ctx = ctx or default_context()
        self.dims = tuple(int(v) for v in dims)
        self.vol = int(np.prod(self.dims))
        self.rng = rng
        self.field_type = field
        self.field = None
        self.refresh()  # the constructor draws the first slice (lattice.C:15-31)

    def refresh(self) -> None:
        f, self.rng.offset = draw_fields(self.rng.kind, self.rng.seed, self.field_type, self.vol, 1,
                                         self.rng.offset, self.ctx)
        self.field = f[0]

    def get(self) -> torch.Tensor:
        return self.field


class Fourier:
    """Fourier (src/fourier/cuda/fourier.cu): a batch of orbitals with in-place 3-D DFTs."""

    def __init__(self, batch: int, dims, precision: str = "f64", ctx: Optional[Context] = None):
        self.ctx = ctx or default_context()
        self.dims = tuple(int(v) for v in dims)
        self.precision = precision
        self.b = torch.zeros((batch,) + self.dims, dtype=_cdtype(precision), device=self.ctx.device)

    def batch_size(self) -> int:
        return self.b.shape[0]

    def forward(self) -> None:  # FFTW_FORWARD: momentum -> position
        self.ctx.check(lib().nrcps_fft3d(self.ctx.handle, _ptr(self.b), self.batch_size(), _ip(_dims(self.dims)),
                                         _prec(self.precision), -1), "Fourier::Forward")

    def backward(self) -> None:  # FFTW_BACKWARD: position -> momentum
        self.ctx.check(lib().nrcps_fft3d(self.ctx.handle, _ptr(self.b), self.batch_size(), _ip(_dims(self.dims)),
                                         _prec(self.precision), +1), "Fourier::Backward")

    def get(self, n: int) -> torch.Tensor:
        if n < 0 or n >= self.batch_size():
            raise ValueError("Fourier::Get: argument out of range")  # fourier_common.C:14-15
        return self.b[n]


class Kinetic:
    """Kinetic (src/hamiltonian/hamiltonian.C:260-281): psi(p) /= xi(p)."""

    def __init__(self, dims, dispersion: str = "PERFECT", mass: float = 1.0, dt: float = 0.5, cutoff: float = 2.0,
                 ctx: Optional[Context] = None):
        self.ctx = ctx or default_context()
        self.xi_host = kinetic_table(dims, dispersion, mass, dt, cutoff)
        self.xi = torch.from_numpy(self.xi_host).to(self.ctx.device)

    def initialize(self) -> None:
        pass

    def evolve(self, b: Fourier) -> None:
        self.ctx.check(lib().nrcps_kinetic_evolve(self.ctx.handle, _ptr(b.b), b.batch_size(), self.xi.numel(),
                                                  _ptr(self.xi), _prec(b.precision)), "Kinetic::Evolve")


class Potential:
    """Potential (src/hamiltonian/hamiltonian.C:165-244): FFT, psi(x) *= v(x), IFFT."""

    def __init__(self, dims, kappa=0.005, dt: float = 0.5, ptype: str = "EXP", ctx: Optional[Context] = None):
        self.ctx = ctx or default_context()
        self.dims = tuple(int(v) for v in dims)
        self.pot_host = potential_table(dims, kappa, dt, ptype)
        self.pot = torch.from_numpy(self.pot_host).to(self.ctx.device)

    def initialize(self) -> None:
        pass

    def evolve(self, b: Fourier) -> None:
        self.ctx.check(lib().nrcps_potential_evolve(self.ctx.handle, _ptr(b.b), b.batch_size(), _ip(_dims(self.dims)),
                                                    _ptr(self.pot), _prec(b.precision)), "Potential::Evolve")


class Interaction:
    """Interaction (src/hamiltonian/hamiltonian.C:77-147): smeared aux-field factor."""

    def __init__(self, lattice: Lattice, mass: float = 1.0, couplings=(0.019894367886486918,), dt: float = 1.0,
                 cutoff: float = 2.0, itype: str = "ONEMINUSXIINVSQ"):
        self.ctx = lattice.ctx
        self.lattice = lattice
        self.dims = lattice.dims
        self.itab_host = interaction_table(self.dims, mass, couplings, dt, cutoff, itype)
        self.itab = torch.from_numpy(self.itab_host).to(self.ctx.device)
        self.fld = torch.zeros((lattice.vol, 2), dtype=torch.float64, device=self.ctx.device)

    def initialize(self) -> None:
        self.ctx.check(lib().nrcps_interaction_initialize(self.ctx.handle, _ptr(self.lattice.get()), _ptr(self.itab),
                                                          _ip(_dims(self.dims)), _ptr(self.fld)),
                       "Interaction::Initialize")

    def evolve(self, b: Fourier) -> None:
        self.ctx.check(lib().nrcps_interaction_evolve(self.ctx.handle, _ptr(b.b), b.batch_size(),
                                                      _ip(_dims(self.dims)), _ptr(self.fld), _prec(b.precision)),
                       "Interaction::Evolve")


class Propagator:
    """Propagator (src/alg/propagator.C): N orbitals advanced by a Hamiltonian list."""

    def __init__(self, n_fermions: int, dims, precision: str = "f64", ctx: Optional[Context] = None):
        self.b = Fourier(n_fermions, dims, precision, ctx)
        self.ctx = self.b.ctx

    def run(self, hamiltonians) -> None:
        for h in hamiltonians:
            h.evolve(self.b)

    def set(self, psi, n: int) -> None:
        src = psi if isinstance(psi, torch.Tensor) else torch.from_numpy(np.asarray(psi))
        self.b.get(n).copy_(src.reshape(self.b.dims).to(self.b.b.dtype).to(self.ctx.device))

    def get(self, n: Optional[int] = None):
        return self.b if n is None else self.b.get(n)


class OneBody:
    """OneBody (src/one_body/one_body.C): a source vector in momentum space."""

    def __init__(self, dims, ctx: Optional[Context] = None):
        self.ctx = ctx or default_context()
        self.dims = tuple(int(v) for v in dims)
        self.vol = int(np.prod(self.dims))
        self.psi = torch.zeros(self.vol, dtype=torch.complex128, device=self.ctx.device)

    def set_momentum(self, n1: int, n2: int, n3: int) -> None:  # OneBody::Set(int,int,int)
        X, Y, Z = self.dims
        self.psi.zero_()
        self.psi[(n3 % Z) + Z * ((n2 % Y) + Y * (n1 % X))] = 1.0

    def set_vector(self, v) -> None:  # OneBody::Set(Float*)
        self.psi.copy_(torch.as_tensor(np.asarray(v), dtype=torch.complex128).reshape(-1))

    def get(self) -> torch.Tensor:
        return self.psi

    def project(self, phi: torch.Tensor) -> complex:  # OneBody::Project
        S = overlap(self.psi.reshape(1, -1), phi.reshape(1, -1), self.ctx)
        return complex(S[0, 0, 0].item())


class TwoBody:
    """TwoBody (src/two_body/two_body.C): pair sink sum_p w(p) psi1(p) psi2(-p)."""

    def __init__(self, dims, wavefunc: str = "TGND", disp: str = "STANDARD", mass: float = 1.0,
                 lam: float = 0.176776695, cutoff: float = 0.99999, ctx: Optional[Context] = None):
        self.ctx = ctx or default_context()
        self.w_host, self.opp_host = two_body_tables(dims, wavefunc, disp, mass, lam, cutoff)
        self.w = torch.from_numpy(self.w_host).to(self.ctx.device)
        self.opp = torch.from_numpy(self.opp_host).to(self.ctx.device)

    def run_matrix(self, props1: torch.Tensor, props2: torch.Tensor) -> torch.Tensor:
        """TwoBody::Run(Float**, Float**, complex*, int): [nconf, n, n] pair matrices."""
        p1 = props1.reshape(-1, props1.shape[-2] if props1.dim() > 2 else props1.shape[0], self.w.numel())
        p2 = props2.reshape(p1.shape)
        nconf, n, vol = p1.shape
        out = torch.empty((nconf, n, n), dtype=torch.complex128, device=self.ctx.device)
        prec = C.F64 if p1.dtype == torch.complex128 else C.F32
        self.ctx.check(lib().nrcps_pair_matrix(self.ctx.handle, _ptr(p1), _ptr(p2), n, nconf, vol, _ptr(self.w),
                                               _ptr(self.opp), prec, _ptr(out)), "TwoBody::Run")
        return out

    def run(self, prop1: torch.Tensor, prop2: torch.Tensor) -> complex:
        """TwoBody::Run(Float*, Float*)."""
        return complex(self.run_matrix(prop1.reshape(1, 1, -1), prop2.reshape(1, 1, -1))[0, 0, 0].item())


def propagate(psi: torch.Tensor, batch: int, kinv: torch.Tensor, field: torch.Tensor, a: float,
              field_mode: int = 1, off0: int = 0, conf_stride: Optional[int] = None,
              pos: Optional[torch.Tensor] = None, ctx: Optional[Context] = None) -> None:
    """One fused Propagator::Run step on psi [nconf*batch, X, Y, Z] (in place):
    psi <- k . B[w . F[k . psi]], k = kinv (FP64, V), w from `field`
    (field_mode 1: Z2 bits, 2: interleaved complex phi, 0: complex fld)."""
    ctx = ctx or default_context()
    dims = tuple(psi.shape[-3:])
    vol = int(np.prod(dims))
    nconf = psi.shape[0] // batch
    pf = C.PositionFactor()
    pf.field_mode, pf.dev_field, pf.bit0 = field_mode, field.data_ptr(), off0
    pf.conf_stride = vol if conf_stride is None else conf_stride
    pf.a, pf.dev_pos = a, (pos.data_ptr() if pos is not None else None)
    prec = C.F64 if psi.dtype == torch.complex128 else C.F32
    ctx.check(lib().nrcps_propagate(ctx.handle, _ptr(psi), batch, nconf, _ip(_dims(dims)), _ptr(kinv),
                                    ctypes.byref(pf), prec), "propagate")


def overlap(src: torch.Tensor, psi: torch.Tensor, ctx: Optional[Context] = None) -> torch.Tensor:
    """S[c][s][t] = <src_s | psi_{c,t}>; src [ns, V] complex128, psi [nconf, nt, V] or [nt, V]."""
    ctx = ctx or default_context()
    src = src.reshape(src.shape[0], -1).contiguous()
    vol = src.shape[1]
    p = psi.reshape(-1, psi.shape[-2] if psi.dim() >= 3 else psi.shape[0], vol).contiguous()
    nconf, nt, _ = p.shape
    S = torch.empty((nconf, src.shape[0], nt), dtype=torch.complex128, device=ctx.device)
    prec = C.F64 if p.dtype == torch.complex128 else C.F32
    ctx.check(lib().nrcps_overlap(ctx.handle, _ptr(src), src.shape[0], _ptr(p), nt, nconf, vol, prec, _ptr(S)),
              "overlap")
    return S


def overlap_planewave(index, psi: torch.Tensor, ctx: Optional[Context] = None) -> torch.Tensor:
    ctx = ctx or default_context()
    idx = torch.as_tensor(np.asarray(index, dtype=np.int32), device=ctx.device)
    p = psi.contiguous()
    nconf, nt, vol = p.shape
    S = torch.empty((nconf, idx.numel(), nt), dtype=torch.complex128, device=ctx.device)
    prec = C.F64 if p.dtype == torch.complex128 else C.F32
    ctx.check(lib().nrcps_overlap_planewave(ctx.handle, _ptr(idx), idx.numel(), _ptr(p), nt, nconf, vol, prec,
                                            _ptr(S)), "overlap_planewave")
    return S


def slater_dets(S: torch.Tensor, psi1: Optional[torch.Tensor] = None, mode: int = 0, log: bool = False,
                ctx: Optional[Context] = None) -> torch.Tensor:
    """All leading-minor determinants of [nconf, N, N] Slater matrices (SlaterDet::Run / SlaterDet2::Run)."""
    ctx = ctx or default_context()
    S = S.contiguous()
    nconf, N, _ = S.shape
    nmeas = 2 * N if mode else N
    out = torch.empty((nconf, nmeas), dtype=torch.complex128, device=ctx.device)
    p1 = psi1.contiguous() if psi1 is not None else None
    ctx.check(lib().nrcps_slater_dets(ctx.handle, _ptr(S), _ptr(p1), N, nconf, mode, int(log), _ptr(out)),
              "slater_dets")
    return out


def reorthonormalise(psi: torch.Tensor, logR: Optional[torch.Tensor] = None,
                     ctx: Optional[Context] = None) -> torch.Tensor:
    """CholeskyQR in place of psi [nconf, N, V] (complex64 or complex128):
    psi <- psi R^-1; returns logR [nconf, N] (FP64) with log R_ii added."""
    ctx = ctx or default_context()
    nconf, N = psi.shape[0], psi.shape[1]
    vol = psi[0, 0].numel()
    if not psi.is_contiguous():
        raise ValueError("reorthonormalise works in place on a contiguous tensor")
    if logR is None:
        logR = torch.zeros((nconf, N), dtype=torch.float64, device=ctx.device)
    work = torch.empty((nconf, N, N, 2), dtype=torch.float64, device=ctx.device)
    prec = C.F64 if psi.dtype == torch.complex128 else C.F32
    ctx.check(lib().nrcps_reorthonormalise(ctx.handle, _ptr(psi), N, vol, nconf, prec, _ptr(work), _ptr(logR)),
              "reorthonormalise")
    return logR


def accumulate(dets: torch.Tensor, mode: str = "slater", n_cumulants: int = 0, ctx: Optional[Context] = None):
    """Block sums of the production drivers on the device (FP64):
    corr [nmeas, T] complex = sum_c |det|^2 (mode 'slater', main.C:208-211) or
    sum_c det (mode 'slater2', main-no_cum.C:205-207), and for n_cumulants = Nc > 0
    z [Nc, nmeas, T] = sum_c (log|det|)^(k+1) (main-cum.C:219-233).
    dets: [n_conf, T, nmeas] complex128 on the device."""
    ctx = ctx or default_context()
    d = dets.to(torch.complex128).contiguous()
    n_conf, T, nmeas = d.shape
    corr = torch.empty((nmeas, T), dtype=torch.complex128, device=ctx.device)
    z = torch.empty((max(n_cumulants, 0), nmeas, T), dtype=torch.float64, device=ctx.device)
    ctx.check(lib().nrcps_accumulate(ctx.handle, _ptr(d), n_conf, T, nmeas, 0 if mode == "slater" else 1,
                                     n_cumulants, _ptr(corr), _ptr(z) if n_cumulants > 0 else None), "accumulate")
    return corr, z


def jackknife(x: torch.Tensor, n_bins: int, effective_energy: bool = False, ctx: Optional[Context] = None):
    """Binned jackknife on the device: x [n_samples, n_obs] FP64 -> (mean, err),
    plus (E_eff, E_eff err) of log(C(t)/C(t+1)) when effective_energy."""
    ctx = ctx or default_context()
    x = x.to(torch.float64).contiguous()
    n, n_obs = x.shape
    mean = torch.empty(n_obs, dtype=torch.float64, device=ctx.device)
    err = torch.empty_like(mean)
    em = torch.empty(max(n_obs - 1, 1), dtype=torch.float64, device=ctx.device) if effective_energy else None
    ee = torch.empty_like(em) if effective_energy else None
    ctx.check(lib().nrcps_jackknife(ctx.handle, _ptr(x), n, n_obs, n_bins, _ptr(mean), _ptr(err), _ptr(em),
                                    _ptr(ee)), "jackknife")
    if effective_energy:
        return mean, err, em[: n_obs - 1], ee[: n_obs - 1]
    return mean, err


class SlaterDet:
    """SlaterDet (src/slater_det/slater_det.C): S[s][t] = <src_s|prop_t>, det of leading minors."""

    def __init__(self, props: torch.Tensor, one_bodies: Sequence[OneBody]):
        self.ctx = one_bodies[0].ctx
        src = torch.stack([ob.get() for ob in one_bodies])
        self.mat = overlap(src, props.reshape(1, len(one_bodies), -1), self.ctx)
        self._dets = None
        self.log = False

    def set_det_type(self, log: bool) -> None:
        self.log = log
        self._dets = None

    def slater_mat(self, s: int, t: int) -> complex:
        return complex(self.mat[0, s, t].item())

    def run(self, n: int) -> complex:
        if n > self.mat.shape[1]:
            raise ValueError("Submatrix exceeds size of matrix.")  # slater_det.C:66-68
        if n < 1:
            return 1.0
        if self._dets is None:
            self._dets = slater_dets(self.mat, log=self.log, ctx=self.ctx).cpu()
        return complex(self._dets[0, n - 1])


# ------------------------------------------------------------------ ensemble
@dataclass
class EnsembleJob:
    """One batched run of the production loop (production/slater_det/main.C)."""
    L: int = 16
    T: int = 32
    n_conf: int = 200
    rng: str = "RANLXS2"
    seed: int = 1234
    rank: int = 0
    field: str = "ZTWO"
    precision: str = "f64"
    kin_disp: str = "PERFECT"
    kin_mass: float = 1.0
    kin_dt: float = 0.5
    cutoff: float = 2.0
    int_mass: float = 1.0
    int_dt: float = 1.0
    int_type: str = "ONEMINUSXIINVSQ"
    couplings: list = dc_field(default_factory=lambda: [0.019894367886486918])
    potential: bool = False
    pot_type: str = "EXP"
    kappa: float = 0.005
    pot_dt: float = 0.5
    mode: str = "slater"  # "slater" (N minors) or "slater2" (2N, pair sink)
    wavefunc: str = "TGND"
    wf_disp: str = "STANDARD"
    wf_mass: float = 1.0
    wf_lambda: float = 0.176776695
    fermi_energy: float = 0.1
    qr_period: int = 0  # re-orthonormalise every k steps (0: never)

    @property
    def dims(self):
        return (self.L, self.L, self.L)


class GeneralizedTwoBody:
    """GeneralizedTwoBody::Run (src/two_body/noarch/two_body_run.C:45-75) on the
    device.  The tables are the reference class's own (built on the host by
    its OhGroup, src/two_body/two_body.C:209-288): shift [nterms, V],
    half_site_wavefunc [nterms, V], opposite [V], weights [nterms, 10]
    (OhGroup::GetWeight(R, l))."""

    def __init__(self, shift, half_site_wavefunc, opposite, weights, ctx: Optional[Context] = None):
        self.ctx = ctx or default_context()
        dev = self.ctx.device
        self.shift = torch.as_tensor(np.ascontiguousarray(shift, dtype=np.int32), device=dev)
        self.hsw = torch.as_tensor(np.ascontiguousarray(half_site_wavefunc, dtype=np.float64), device=dev)
        self.opp = torch.as_tensor(np.ascontiguousarray(opposite, dtype=np.int32), device=dev)
        self.weights = np.asarray(weights, dtype=np.float64)
        self._wl = {}

    def _folded(self, rep: int) -> torch.Tensor:
        if rep not in self._wl:
            w = torch.as_tensor(self.weights[:, rep], device=self.ctx.device)
            self._wl[rep] = (self.hsw * w[:, None]).contiguous()
        return self._wl[rep]

    def run_matrix(self, props1: torch.Tensor, props2: torch.Tensor, rep: int) -> torch.Tensor:
        """phi[c][s][t] for props [nconf, n, V] (or [n, V]) in representation rep (0 = A1g)."""
        p1 = props1.reshape(-1, props1.shape[-2] if props1.dim() >= 2 else 1, props1.shape[-1]).contiguous()
        p2 = props2.reshape(p1.shape).contiguous()
        nconf, n, vol = p1.shape
        phi = torch.empty((nconf, n, n), dtype=torch.complex128, device=self.ctx.device)
        prec = C.F64 if p1.dtype == torch.complex128 else C.F32
        self.ctx.check(lib().nrcps_shifted_pair_matrix(self.ctx.handle, _ptr(p1), _ptr(p2), n, nconf, vol,
                                                       self.shift.shape[0], _ptr(self.shift), _ptr(self._folded(rep)),
                                                       _ptr(self.opp), prec, _ptr(phi)), "shifted_pair_matrix")
        return phi

    def run(self, prop1: torch.Tensor, prop2: torch.Tensor, rep: int) -> complex:
        return complex(self.run_matrix(prop1.reshape(1, 1, -1), prop2.reshape(1, 1, -1), rep).cpu().item())


class Branching:
    """The multilevel branching driver (production/two_body-branched/main.C:23-80)
    on the device: run() walks one tree and returns its corr[t] contributions."""

    def __init__(self, L: int, levels: int, branches: int, steps: int, sources2: np.ndarray, rng: str = "RANLXS2",
                 seed: int = 1234, field: str = "ZTWO", a: float = 0.5, precision: str = "f64",
                 wavefunc: str = "TGND", wf_disp: str = "STANDARD", wf_mass: float = 1.0,
                 wf_lambda: float = 0.176776695, kin_dt: float = 0.5, cutoff: float = 2.0,
                 potential: Optional[np.ndarray] = None, ctx: Optional[Context] = None):
        self.ctx = ctx or default_context()
        dims = (L, L, L)
        self.T = levels * steps
        p = C.BranchParams()
        p.dims[:] = dims
        p.levels, p.branches, p.steps = levels, branches, steps
        p.rng_kind, p.seed, p.field_kind = C.RNG_KINDS[rng], seed, C.FIELD_KINDS[field]
        p.precision, p.a = _prec(precision), a
        xi = np.ascontiguousarray(kinetic_table(dims, "PERFECT", 1.0, kin_dt, cutoff))
        w, opp = two_body_tables(dims, wavefunc, wf_disp, wf_mass, wf_lambda, cutoff)
        src = np.ascontiguousarray(np.asarray(sources2, dtype=np.complex128).reshape(2, -1))
        pot = None if potential is None else np.ascontiguousarray(potential, dtype=np.float64)
        h = ctypes.c_void_p()
        self.ctx.check(lib().nrcps_branch_create(
            self.ctx.handle, ctypes.byref(p), xi.ctypes.data_as(ctypes.c_void_p),
            pot.ctypes.data_as(ctypes.c_void_p) if pot is not None else None,
            src.view(np.float64).ctypes.data_as(ctypes.c_void_p),
            np.ascontiguousarray(w, dtype=np.float64).ctypes.data_as(ctypes.c_void_p),
            np.ascontiguousarray(opp, dtype=np.int32).ctypes.data_as(ctypes.c_void_p), ctypes.byref(h)),
            "branch_create")
        self.handle = h

    def run(self) -> torch.Tensor:
        corr = torch.zeros(self.T, dtype=torch.complex128, device=self.ctx.device)
        self.ctx.check(lib().nrcps_branch_run(self.handle, _ptr(corr)), "branch_run")
        return corr

    def close(self) -> None:
        if getattr(self, "handle", None):
            lib().nrcps_branch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


@dataclass
class BatchJob:
    """One job of a Batch: an L^3 lattice, T slices, n_conf configurations,
    plane-wave sources (the Fermi sea of `fermi_energy`, or an explicit
    lattice-index list)."""
    L: int
    T: int
    n_conf: int = 1
    fermi_energy: float = 0.1
    pw_index: Optional[list] = None


class Batch:
    """nrcps_batch: jobs of different L, N and T, all time loops in one graph
    launch; fields from one generator stream in job order."""

    def __init__(self, jobs: Sequence[BatchJob], rng: str = "RANLXS2", seed: int = 99, field: str = "GAUSS",
                 a: float = 0.3, precision: str = "f32", qr_period: int = 0, kin_dt: float = 0.5,
                 cutoff: float = 2.0, ctx: Optional[Context] = None):
        self.ctx = ctx or default_context()
        self.jobs = list(jobs)
        n = len(self.jobs)
        self._keep = []
        arr = (C.BatchJob * n)()
        self.n_orb = []
        for i, jb in enumerate(self.jobs):
            dims = (jb.L,) * 3
            idx = jb.pw_index if jb.pw_index is not None else momenta(dims, "PERFECT", 1.0, jb.fermi_energy, cutoff)[0]
            idx = np.ascontiguousarray(np.asarray(idx, dtype=np.int32))
            xi = np.ascontiguousarray(kinetic_table(dims, "PERFECT", 1.0, kin_dt, cutoff))
            self._keep += [idx, xi]
            self.n_orb.append(int(idx.size))
            arr[i].L, arr[i].n_orb, arr[i].T, arr[i].n_conf = jb.L, idx.size, jb.T, jb.n_conf
            arr[i].pw_index = idx.ctypes.data_as(ctypes.POINTER(ctypes.c_int))
            arr[i].kin_xi = xi.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        p = C.BatchParams()
        p.rng_kind, p.seed, p.field_kind = C.RNG_KINDS[rng], seed, C.FIELD_KINDS[field]
        p.precision, p.a, p.qr_period = _prec(precision), a, qr_period
        h = ctypes.c_void_p()
        self.ctx.check(lib().nrcps_batch_create(self.ctx.handle, ctypes.byref(p), arr, n, ctypes.byref(h)),
                       "batch_create")
        self.handle = h
        size = ctypes.c_long()
        self.ctx.check(lib().nrcps_batch_output_size(h, ctypes.byref(size), None), "batch_output_size")
        self.out = torch.empty(size.value // 2, dtype=torch.complex128, device=self.ctx.device)
        self.layout = []
        for i in range(n):
            off, sz = ctypes.c_long(), ctypes.c_long()
            self.ctx.check(lib().nrcps_batch_layout(h, i, ctypes.byref(off), ctypes.byref(sz)), "batch_layout")
            self.layout.append((off.value // 2, sz.value // 2))

    def run(self):
        """One run (the next window of the stream); returns one [n_conf, T, N]
        complex128 device view per job."""
        self.ctx.check(lib().nrcps_batch_run(self.handle, _ptr(self.out)), "batch_run")
        return [self.out[o:o + s].view(jb.n_conf, jb.T, n) for (o, s), jb, n in zip(self.layout, self.jobs, self.n_orb)]

    def launches(self) -> int:
        v = ctypes.c_long()
        self.ctx.check(lib().nrcps_batch_output_size(self.handle, None, ctypes.byref(v)), "batch_output_size")
        return v.value

    def close(self) -> None:
        if getattr(self, "handle", None):
            lib().nrcps_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Ensemble:
    """nrcps_ensemble: every configuration of a run advanced together, time loop in a CUDA graph."""

    def __init__(self, job: EnsembleJob, sources: Optional[np.ndarray] = None, plane_wave_index=None,
                 ctx: Optional[Context] = None):
        self.ctx = ctx or default_context()
        self.job = job
        dims = job.dims
        vol = int(np.prod(dims))
        xi = kinetic_table(dims, job.kin_disp, job.kin_mass, job.kin_dt, job.cutoff)
        itab = interaction_table(dims, job.int_mass, job.couplings, job.int_dt, job.cutoff, job.int_type)
        pot = potential_table(dims, job.kappa, job.pot_dt, job.pot_type) if job.potential else None
        local = len(job.couplings) == 1
        if plane_wave_index is not None:
            idx = np.ascontiguousarray(np.asarray(plane_wave_index, dtype=np.int32))
            n_orb = idx.size
            src = None
        else:
            src = np.ascontiguousarray(np.asarray(sources, dtype=np.complex128).reshape(-1, vol))
            n_orb = src.shape[0]
            idx = None
        self.n_orb = n_orb
        self.nmeas = 2 * n_orb if job.mode == "slater2" else n_orb
        w = opp = None
        if job.mode == "slater2":
            w, opp = two_body_tables(dims, job.wavefunc, job.wf_disp, job.wf_mass, job.wf_lambda, job.cutoff)
        j = C.Job()
        j.dims[:] = dims
        j.T, j.n_orb, j.n_conf = job.T, n_orb, job.n_conf
        j.rng_kind, j.seed = C.RNG_KINDS[job.rng], job.seed + 491 * job.rank
        j.field_kind = C.FIELD_KINDS[job.field]
        j.mode = 1 if job.mode == "slater2" else 0
        j.precision = _prec(job.precision)
        j.plane_wave = int(idx is not None)
        j.use_potential = int(pot is not None)
        j.qr_period = job.qr_period
        j.a = float(itab[0] * vol)  # c(p) * V: the local (1 + a phi) coupling
        j.local_interaction = int(local)
        self._keep = (xi, itab, pot, src, idx, w, opp)
        h = ctypes.c_void_p()
        dp = lambda a: None if a is None else _dp(a.view(np.float64) if a.dtype == np.complex128 else a)
        ipn = lambda a: None if a is None else _ip(a)
        self.ctx.check(lib().nrcps_ensemble_create(self.ctx.handle, ctypes.byref(j), dp(xi), dp(itab), dp(pot),
                                                   dp(src), ipn(idx), dp(w), ipn(opp), ctypes.byref(h)),
                       "ensemble_create")
        self.handle = h
        self.dets = torch.empty((job.n_conf, job.T, self.nmeas), dtype=torch.complex128, device=self.ctx.device)

    def set_sources(self, sources=None, plane_wave_index=None) -> None:
        """Sources of later runs from host memory (OneBody::Set + Propagator::Set):
        dense [N, V] complex128 or plane-wave indices [N] int32, the kind given at
        creation.  Pinned host tensors keep the copy asynchronous."""
        if plane_wave_index is not None:
            idx = plane_wave_index
            if isinstance(idx, torch.Tensor):
                p = ctypes.cast(idx.data_ptr(), ctypes.POINTER(ctypes.c_int))
            else:
                idx = np.ascontiguousarray(np.asarray(idx, dtype=np.int32))
                p = _ip(idx)
            self.ctx.check(lib().nrcps_ensemble_set_sources(self.handle, None, p), "ensemble_set_sources")
            self._src_keep = idx  # the copy may read it after this call returns
        else:
            src = sources
            if isinstance(src, torch.Tensor):
                p = ctypes.cast(src.data_ptr(), ctypes.POINTER(ctypes.c_double))
            else:
                src = np.ascontiguousarray(np.asarray(src, dtype=np.complex128))
                p = _dp(src.view(np.float64))
            self.ctx.check(lib().nrcps_ensemble_set_sources(self.handle, p, None), "ensemble_set_sources")
            self._src_keep = src

    def run(self, first_conf: int = 0) -> torch.Tensor:
        """Raw determinants [n_conf, T, nmeas] of configurations first_conf.. (device tensor)."""
        self.ctx.check(lib().nrcps_ensemble_run(self.handle, first_conf, _ptr(self.dets)), "ensemble_run")
        return self.dets

    def launches(self) -> int:
        n = ctypes.c_long()
        self.ctx.check(lib().nrcps_ensemble_launches(self.handle, ctypes.byref(n)), "ensemble_launches")
        return n.value

    def field_bits_ptr(self) -> Optional[int]:
        """Device address of the last run's Z2 field bits (configuration c,
        slice t at bit (c T + t) V), valid until the next run; None for other
        fields."""
        p = ctypes.c_void_p()
        self.ctx.check(lib().nrcps_ensemble_field_bits(self.handle, ctypes.byref(p)), "ensemble_field_bits")
        return p.value

    def close(self) -> None:
        if getattr(self, "handle", None):
            lib().nrcps_ensemble_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

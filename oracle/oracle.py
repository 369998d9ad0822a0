"""TEST INFRASTRUCTURE ONLY -- Python access to the CPU oracle.

`oracle/tbpm_oracle.cpp` restates the reference TBPLaS Fortran TBPM core
(tbplas/fortran/tbpm.f90, propagation.f90, csr.F90, math.F90, funcs.f90,
kpm.f90, fft.F90, random.f90).  This module loads it with ctypes and exposes

* numpy-level functions (`tbpm_dos`, `tbpm_accond`, `tbpm_dccond`,
  `tbpm_psi_t`, `cheb_timestep`, `fermi`, `fermi_cheb_coef`, `random_state`),
* `F2pyShim`, a module-like object with the f2py-visible signatures of the
  reference's `tbplas.fortran.f2py`, so the reference's own Solver can run on
  the oracle (used to generate the golden fixtures).

Parity status: the Fortran core cannot be compiled here (no Fortran compiler),
so the oracle is pinned by exact-diagonalisation known answers, by the
reference's Python layer (CSR builders, Bessel series, Analyzer) and by the
Philox4x32-10 known-answer vectors; the gfortran RANDOM_NUMBER stream of the
reference is not reproducible (random states are injected in parity tests).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it.
"""

import ctypes
import os
from typing import Optional

import numpy as np

from . import build_oracle

_lib = None

_i32p = ctypes.c_void_p
_vp = ctypes.c_void_p
_int = ctypes.c_int
_i64 = ctypes.c_int64
_dbl = ctypes.c_double


def lib(native: bool = False) -> ctypes.CDLL:
    """Load (building first if needed) the oracle shared library."""
    global _lib
    if _lib is None or native:
        path = build_oracle.build(native=native)
        L = ctypes.CDLL(path)
        L.orc_set_threads.argtypes = [_int]
        L.orc_max_threads.restype = _int
        L.orc_philox4x32_10.argtypes = [_vp, ctypes.c_uint32, ctypes.c_uint32]
        L.orc_random_state.argtypes = [_vp, _i64, _i64, _int]
        L.orc_fermi_cheb_coef.argtypes = [_vp, _int, _dbl, _dbl, _int, _dbl]
        L.orc_fermi_cheb_coef.restype = _int
        L.orc_cheb_timestep.argtypes = [_vp, _int, _vp, _vp, _vp, _i64, _vp, _vp, _int]
        L.orc_fermi.argtypes = [_vp, _int, _vp, _vp, _vp, _i64, _vp, _vp]
        L.orc_tbpm_dos.argtypes = [_vp, _int, _vp, _vp, _vp, _i64, _vp, _int, _int, _int, _int,
                                   _int, _dbl, _int, _vp]
        L.orc_tbpm_accond.argtypes = [_vp, _int, _dbl, _dbl, _vp, _vp, _vp, _i64, _i64, _dbl,
                                      _vp, _vp, _vp, _int, _int, _int, _int, _dbl, _int, _int,
                                      _dbl, _int, _vp]
        L.orc_tbpm_dccond.argtypes = [_vp, _int, _vp, _vp, _vp, _i64, _i64, _dbl, _vp, _vp,
                                      _vp, _int, _int, _int, _dbl, _vp, _int, _vp, _int, _int,
                                      _int, _dbl, _int, _vp, _vp]
        L.orc_tbpm_psi_t.argtypes = [_vp, _int, _vp, _vp, _vp, _i64, _vp, _vp, _int, _int, _int,
                                     _dbl, _vp]
        L.orc_tbpm_dyn_pol.argtypes = [_vp, _int, _dbl, _dbl, _vp, _vp, _vp, _i64, _vp, _vp, _vp,
                                       _vp, _int, _vp, _int, _int, _int, _int, _dbl, _int, _int,
                                       _dbl, _int, _vp]
        L.orc_tbpm_eigenstates.argtypes = [_vp, _int, _vp, _vp, _vp, _i64, _vp, _int, _int, _int,
                                           _dbl, _vp, _int, _int, _int, _dbl, _int, _vp]
        L.orc_tbpm_kbdc.argtypes = [_vp, _vp, _vp, _i64, _i64, _dbl, _vp, _vp, _vp, _int, _int,
                                    _int, _int, _int, _int, _vp]
        L.orc_cond_from_trace.argtypes = [_vp, _int, _vp, _int, _dbl, _dbl, _int, _vp]
        L.orc_haydock_coef.argtypes = [_vp, _int, _vp, _vp, _vp, _i64, _dbl, _vp, _int, _int,
                                       _int, _int, _vp, _vp]
        if native:
            return L
        _lib = L
    return _lib


class OracleError(RuntimeError):
    pass


def _check(rc: int, what: str) -> None:
    if rc == 2:
        raise OracleError(f"{what}: wave function norm broken (check_norm)")
    if rc != 0:
        raise OracleError(f"{what}: invalid arguments (status {rc})")


def _c(a, dt):
    return np.ascontiguousarray(np.asarray(a, dtype=dt))


def _p(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data


def _csr(indptr, indices, hop):
    ip = _c(indptr, np.int32)
    ix = _c(indices, np.int32)
    hv = _c(hop, np.complex128)
    return ip, ix, hv, ip.size - 1, hv.size


def set_threads(n: int) -> None:
    lib().orc_set_threads(int(n))


def max_threads() -> int:
    return int(lib().orc_max_threads())


def philox4x32_10(counter, key):
    ctr = np.array(counter, dtype=np.uint32)
    lib().orc_philox4x32_10(ctr.ctypes.data, int(key[0]), int(key[1]))
    return ctr


def random_state(n: int, iseed: int, kind: int = 0) -> np.ndarray:
    """random.f90:36-69 with the Philox uniform source; iseed as passed by the
    drivers (seed*(i_sample + rank*n_samples))."""
    wf = np.zeros(int(n), dtype=np.complex128)
    lib().orc_random_state(wf.ctypes.data, int(n), int(iseed), int(kind))
    return wf


def fermi_cheb_coef(nr_fermi: int, beta: float, mu: float, one_minus: bool,
                    eps: float) -> np.ndarray:
    coef = np.zeros(int(nr_fermi) + 1)
    n = lib().orc_fermi_cheb_coef(coef.ctypes.data, int(nr_fermi), float(beta), float(mu),
                                  1 if one_minus else 0, float(eps))
    if n < 0:
        raise OracleError("bad nr_fermi")
    return coef[:n].copy()


def cheb_timestep(bes, indptr, indices, hop, wf, forward: bool = True) -> np.ndarray:
    bes = _c(bes, np.float64)
    ip, ix, hv, n, _ = _csr(indptr, indices, hop)
    w = _c(wf, np.complex128)
    out = np.zeros_like(w)
    _check(lib().orc_cheb_timestep(_p(bes), bes.size, _p(ip), _p(ix), _p(hv), n, _p(w),
                                   _p(out), 1 if forward else 0), "cheb_timestep")
    return out


def fermi(coef, indptr, indices, hop, wf) -> np.ndarray:
    coef = _c(coef, np.float64)
    ip, ix, hv, n, _ = _csr(indptr, indices, hop)
    w = _c(wf, np.complex128)
    out = np.zeros_like(w)
    _check(lib().orc_fermi(_p(coef), coef.size, _p(ip), _p(ix), _p(hv), n, _p(w), _p(out)),
           "fermi")
    return out


def tbpm_dos(bes, indptr, indices, hop, n_timestep, wf0=None, seed=1337, n_samples=1,
             rank=0, chk_step=128, chk_thr=1e-9, state_kind=0) -> np.ndarray:
    bes = _c(bes, np.float64)
    ip, ix, hv, n, _ = _csr(indptr, indices, hop)
    if wf0 is not None:
        wf0 = _c(np.atleast_2d(wf0), np.complex128)
        n_samples = wf0.shape[0]
    corr = np.zeros(int(n_timestep) + 1, dtype=np.complex128)
    _check(lib().orc_tbpm_dos(_p(bes), bes.size, _p(ip), _p(ix), _p(hv), n, _p(wf0), int(seed),
                              int(n_timestep), int(n_samples), int(rank), int(chk_step),
                              float(chk_thr), int(state_kind), _p(corr)), "tbpm_dos")
    return corr


def tbpm_accond(bes, beta, mu, indptr, indices, hop, rescale, dx, dy, n_timestep, wf0=None,
                seed=1337, n_samples=1, nr_fermi=2**15, fermi_precision=1e-12, rank=0,
                chk_step=128, chk_thr=1e-9, state_kind=0) -> np.ndarray:
    bes = _c(bes, np.float64)
    ip, ix, hv, n, nnz = _csr(indptr, indices, hop)
    dx, dy = _c(dx, np.float64), _c(dy, np.float64)
    if wf0 is not None:
        wf0 = _c(np.atleast_2d(wf0), np.complex128)
        n_samples = wf0.shape[0]
    corr = np.zeros((4, int(n_timestep)), dtype=np.complex128, order="F")
    _check(lib().orc_tbpm_accond(_p(bes), bes.size, float(beta), float(mu), _p(ip), _p(ix),
                                 _p(hv), n, nnz, float(rescale), _p(dx), _p(dy), _p(wf0),
                                 int(seed), int(n_timestep), int(n_samples), int(nr_fermi),
                                 float(fermi_precision), int(rank), int(chk_step),
                                 float(chk_thr), int(state_kind), _p(corr)), "tbpm_accond")
    return corr


def tbpm_dccond(bes, indptr, indices, hop, rescale, dx, dy, n_timestep, t_step, energies,
                en_inds, wf0=None, seed=1337, n_samples=1, rank=0, chk_step=128,
                chk_thr=1e-9, state_kind=0):
    bes = _c(bes, np.float64)
    ip, ix, hv, n, nnz = _csr(indptr, indices, hop)
    dx, dy = _c(dx, np.float64), _c(dy, np.float64)
    en = _c(energies, np.float64)
    ei = _c(en_inds, np.int32)
    if wf0 is not None:
        wf0 = _c(np.atleast_2d(wf0), np.complex128)
        n_samples = wf0.shape[0]
    dos = np.zeros(int(n_timestep), dtype=np.complex128)
    dc = np.zeros((2, en.size, int(n_timestep)), dtype=np.complex128, order="F")
    _check(lib().orc_tbpm_dccond(_p(bes), bes.size, _p(ip), _p(ix), _p(hv), n, nnz,
                                 float(rescale), _p(dx), _p(dy), _p(wf0), int(seed),
                                 int(n_timestep), int(n_samples), float(t_step), _p(en),
                                 en.size, _p(ei), ei.size, int(rank), int(chk_step),
                                 float(chk_thr), int(state_kind), _p(dos), _p(dc)),
           "tbpm_dccond")
    return dos, dc


def tbpm_psi_t(bes, indptr, indices, hop, psi0, time_log, n_timestep, chk_step=128,
               chk_thr=1e-9) -> np.ndarray:
    bes = _c(bes, np.float64)
    ip, ix, hv, n, _ = _csr(indptr, indices, hop)
    p0 = _c(psi0, np.complex128)
    tl = _c(time_log, np.int32)
    out = np.zeros((n, tl.size), dtype=np.complex128, order="F")
    _check(lib().orc_tbpm_psi_t(_p(bes), bes.size, _p(ip), _p(ix), _p(hv), n, _p(p0), _p(tl),
                                tl.size, int(n_timestep), int(chk_step), float(chk_thr),
                                _p(out)), "tbpm_psi_t")
    return out


def tbpm_dyn_pol(bes, beta, mu, indptr, indices, hop, site_x, site_y, site_z, q_points,
                 n_timestep, wf0=None, seed=1337, n_samples=1, nr_fermi=2**15,
                 fermi_precision=1e-12, rank=0, chk_step=128, chk_thr=1e-9,
                 state_kind=0) -> np.ndarray:
    """tbpm.f90:355-493; returns (n_q, n_timestep) float64."""
    bes = _c(bes, np.float64)
    ip, ix, hv, n, _ = _csr(indptr, indices, hop)
    sx, sy, sz = _c(site_x, np.float64), _c(site_y, np.float64), _c(site_z, np.float64)
    q = _c(np.atleast_2d(q_points), np.float64)
    if wf0 is not None:
        wf0 = _c(np.atleast_2d(wf0), np.complex128)
        n_samples = wf0.shape[0]
    corr = np.zeros((q.shape[0], int(n_timestep)), order="F")
    _check(lib().orc_tbpm_dyn_pol(_p(bes), bes.size, float(beta), float(mu), _p(ip), _p(ix),
                                  _p(hv), n, _p(sx), _p(sy), _p(sz), _p(q), q.shape[0],
                                  _p(wf0), int(seed), int(n_timestep), int(n_samples),
                                  int(nr_fermi), float(fermi_precision), int(rank),
                                  int(chk_step), float(chk_thr), int(state_kind), _p(corr)),
           "tbpm_dyn_pol")
    return corr


def tbpm_eigenstates(bes, indptr, indices, hop, n_timestep, t_step, energies, wf0=None,
                     seed=1337, n_samples=1, rank=0, chk_step=128, chk_thr=1e-9,
                     state_kind=0) -> np.ndarray:
    """tbpm.f90:721-830; returns (n_energies, n_orb) float64."""
    bes = _c(bes, np.float64)
    ip, ix, hv, n, _ = _csr(indptr, indices, hop)
    en = _c(energies, np.float64)
    if wf0 is not None:
        wf0 = _c(np.atleast_2d(wf0), np.complex128)
        n_samples = wf0.shape[0]
    out = np.zeros((en.size, n), order="F")
    _check(lib().orc_tbpm_eigenstates(_p(bes), bes.size, _p(ip), _p(ix), _p(hv), n, _p(wf0),
                                      int(seed), int(n_timestep), int(n_samples), float(t_step),
                                      _p(en), en.size, int(rank), int(chk_step), float(chk_thr),
                                      int(state_kind), _p(out)), "tbpm_eigenstates")
    return out


def tbpm_kbdc(indptr, indices, hop, rescale, dx, dy, n_kernel, direction, wf0=None,
              seed=1337, n_samples=1, rank=0, state_kind=0) -> np.ndarray:
    """tbpm.f90:836-960; returns mu (n_kernel, n_kernel) complex128."""
    ip, ix, hv, n, nnz = _csr(indptr, indices, hop)
    dx, dy = _c(dx, np.float64), _c(dy, np.float64)
    if wf0 is not None:
        wf0 = _c(np.atleast_2d(wf0), np.complex128)
        n_samples = wf0.shape[0]
    mu = np.zeros((int(n_kernel), int(n_kernel)), dtype=np.complex128, order="F")
    _check(lib().orc_tbpm_kbdc(_p(ip), _p(ix), _p(hv), n, nnz, float(rescale), _p(dx), _p(dy),
                               _p(wf0), int(seed), int(n_samples), int(n_kernel),
                               int(direction), int(rank), int(state_kind), _p(mu)),
           "tbpm_kbdc")
    return mu


def haydock_coef(site_indices, indptr, indices, hop, rescale, n_depth, wf_sites=None,
                 seed=1337, n_samples=1, state_kind=0):
    """propagation.f90:85-155 averaged as in tbpm.f90:998-1018; returns
    (coefa complex[n_depth], coefb float[n_depth])."""
    ip, ix, hv, n, _ = _csr(indptr, indices, hop)
    si = _c(site_indices, np.int32)
    if wf_sites is not None:
        wf_sites = _c(np.atleast_2d(wf_sites), np.complex128)
        n_samples = wf_sites.shape[0]
    a = np.zeros(int(n_depth), dtype=np.complex128)
    b = np.zeros(int(n_depth))
    _check(lib().orc_haydock_coef(_p(si), si.size, _p(ip), _p(ix), _p(hv), n, float(rescale),
                                  _p(wf_sites), int(seed), int(n_depth), int(n_samples),
                                  int(state_kind), _p(a), _p(b)), "haydock_coef")
    return a, b


def cond_from_trace(mu_mn, mu, h_rescale, beta, ne_integral) -> np.ndarray:
    """analysis.f90:6-69; returns float64[len(mu)]."""
    m = np.asfortranarray(np.asarray(mu_mn, dtype=np.complex128))
    mus = _c(mu, np.float64).reshape(-1)
    cond = np.zeros(mus.size)
    _check(lib().orc_cond_from_trace(m.ctypes.data, m.shape[0], _p(mus), mus.size,
                                     float(h_rescale), float(beta), int(ne_integral),
                                     _p(cond)), "cond_from_trace")
    return cond


def green_function(energy: float, delta: float, coefa, coefb) -> complex:
    """funcs.f90:152-172: continued fraction from the deepest level up."""
    e = complex(energy, delta)
    g = 0j
    for i in range(len(coefa) - 1, -1, -1):
        g = 1.0 / (e - coefa[i] - coefb[i] ** 2 * g)
    return g


def ldos_haydock(site_indices, delta, e_range, indptr, indices, hop, rescale, seed, n_depth,
                 n_timestep, n_samples, wf_sites=None, state_kind=0):
    """tbpm.f90:963-1026; returns (energy, ldos) on 2*n_timestep+1 points."""
    a, b = haydock_coef(site_indices, indptr, indices, hop, rescale, n_depth,
                        wf_sites=wf_sites, seed=seed, n_samples=n_samples,
                        state_kind=state_kind)
    energy = np.array([0.5 * i * e_range / n_timestep for i in range(-n_timestep,
                                                                     n_timestep + 1)])
    ldos = np.array([-1.0 / np.pi * green_function(e, delta, a, b).imag for e in energy])
    return energy, ldos


class F2pyShim:
    """The reference's f2py TBPM signatures backed by the oracle.

    `states` (n_samples, n_orb), when set, replaces the random initial states
    so that runs are comparable with other implementations.
    """

    def __init__(self, states: Optional[np.ndarray] = None) -> None:
        self.states = states

    def tbpm_dos(self, bes, s_indptr, s_indices, s_hop, seed, n_timestep, n_ran_samples,
                 output_filename, rank, wfn_chk_step, wfn_chk_thr):
        return tbpm_dos(bes, s_indptr, s_indices, s_hop, n_timestep, wf0=self.states,
                        seed=seed, n_samples=n_ran_samples, rank=rank, chk_step=wfn_chk_step,
                        chk_thr=wfn_chk_thr)

    def tbpm_accond(self, bes, beta, mu, s_indptr, s_indices, s_hop, h_rescale, s_dx, s_dy,
                    seed, n_timestep, n_ran_samples, nr_fermi, fermi_precision,
                    output_filename, rank, wfn_chk_step, wfn_chk_thr):
        return tbpm_accond(bes, beta, mu, s_indptr, s_indices, s_hop, h_rescale, s_dx, s_dy,
                           n_timestep, wf0=self.states, seed=seed, n_samples=n_ran_samples,
                           nr_fermi=nr_fermi, fermi_precision=fermi_precision, rank=rank,
                           chk_step=wfn_chk_step, chk_thr=wfn_chk_thr)

    def tbpm_dccond(self, bes, beta, mu, s_indptr, s_indices, s_hop, h_rescale, s_dx, s_dy,
                    seed, n_timestep, n_ran_samples, t_step, energies, en_inds,
                    output_filename_dos, output_filename_dc, rank, wfn_chk_step, wfn_chk_thr):
        return tbpm_dccond(bes, s_indptr, s_indices, s_hop, h_rescale, s_dx, s_dy, n_timestep,
                           t_step, energies, en_inds, wf0=self.states, seed=seed,
                           n_samples=n_ran_samples, rank=rank, chk_step=wfn_chk_step,
                           chk_thr=wfn_chk_thr)

    def tbpm_dyn_pol(self, bes, beta, mu, s_indptr, s_indices, s_hop, h_rescale, s_dx, s_dy,
                     s_site_x, s_site_y, s_site_z, seed, n_timestep, n_ran_samples, nr_fermi,
                     fermi_precision, q_points, output_filename, rank, wfn_chk_step,
                     wfn_chk_thr):
        return tbpm_dyn_pol(bes, beta, mu, s_indptr, s_indices, s_hop, s_site_x, s_site_y,
                            s_site_z, q_points, n_timestep, wf0=self.states, seed=seed,
                            n_samples=n_ran_samples, nr_fermi=nr_fermi,
                            fermi_precision=fermi_precision, rank=rank,
                            chk_step=wfn_chk_step, chk_thr=wfn_chk_thr)

    def tbpm_eigenstates(self, bes, s_indptr, s_indices, s_hop, seed, n_timestep,
                         n_ran_samples, t_step, energies, rank, wfn_chk_step, wfn_chk_thr):
        return tbpm_eigenstates(bes, s_indptr, s_indices, s_hop, n_timestep, t_step, energies,
                                wf0=self.states, seed=seed, n_samples=n_ran_samples,
                                rank=rank, chk_step=wfn_chk_step, chk_thr=wfn_chk_thr)

    def tbpm_kbdc(self, seed, s_indptr, s_indices, s_hop, h_rescale, s_dx, s_dy,
                  n_ran_samples, n_kernel, direction, rank):
        return tbpm_kbdc(s_indptr, s_indices, s_hop, h_rescale, s_dx, s_dy, n_kernel,
                         direction, wf0=self.states, seed=seed, n_samples=n_ran_samples,
                         rank=rank)

    def cond_from_trace(self, mu_mn, mu, h_rescale, beta, ne_integral, fermi_precision, rank):
        return cond_from_trace(mu_mn, mu, h_rescale, beta, ne_integral)

    def ldos_haydock(self, site_indices, delta, e_range, s_indptr, s_indices, s_hop,
                     h_rescale, seed, n_depth, n_timestep, n_ran_samples, output_filename):
        sites = None if self.states is None else \
            np.asarray(self.states)[:, np.asarray(site_indices)]
        return ldos_haydock(site_indices, delta, e_range, s_indptr, s_indices, s_hop,
                            h_rescale, seed, n_depth, n_timestep, n_ran_samples,
                            wf_sites=sites)

    def tbpm_psi_t(self, bes, indptr, indices, hop, psi0, time_log, n_timestep, wfn_chk_step,
                   wfn_chk_thr):
        return tbpm_psi_t(bes, indptr, indices, hop, psi0, time_log, n_timestep,
                          chk_step=wfn_chk_step, chk_thr=wfn_chk_thr)

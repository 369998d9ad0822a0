"""Checkpoint and resume of long DOS and DC propagations.

The reference's TBPM drivers hold their state inside one Fortran call
(tbplas/fortran/tbpm.f90:6-93), so a run that is interrupted starts again from
t = 0.  `dos_checkpointed` runs the same computation as `f2py.tbpm_dos` as a
device-resident session and, every `every` time steps, writes what the run
needs to go on to one .npz file:

* the initial states of the current batch of states and their current states
  (tbpm_session_export), the correlation and norm rows recorded so far
  (tbpm_session_read);
* the correlation accumulated over the finished batches, the batch position
  and a fingerprint of every input (Bessel series, Hamiltonian, seed, sizes,
  precision, batch width, state distribution).

Called again with the same inputs and path, it resumes from that file
(tbpm_session_dos_resume) and returns exactly what an uninterrupted run
returns.  A file whose fingerprint does not match is ignored.  The file is
written atomically (temporary file + rename) and removed when the run ends.

`dc_checkpointed` does the same for f2py.tbpm_dccond (tbpm.f90:497-718) at the
boundaries between parts of the state list (the per-batch quasi-eigenstate
block is too large to write out mid-batch).
"""

import ctypes
import hashlib
import os
import zlib
from typing import Callable, Optional

import numpy as np

from . import _native as nat
from .fortran import f2py

__all__ = ["dos_checkpointed", "dc_checkpointed", "fingerprint"]


def _crc(a: np.ndarray) -> int:
    return zlib.crc32(np.ascontiguousarray(a).view(np.uint8).reshape(-1))


def fingerprint(bes, indptr, indices, hop, seed, n_timestep, n_samples, rank,
                backend: dict) -> str:
    """Hash of everything the correlation depends on."""
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(bes, dtype=np.float64).tobytes())
    if hasattr(indptr, "make_resident"):
        d = indptr.sample
        for a in (d.lat_vec, d.origin, d.pc_orb_pos, d.orb_eng, d.hop_ind, d.hop_eng,
                  d.vac_id_sc):
            h.update(str(_crc(a)).encode())
        if d.orb_eng_sc is not None:
            h.update(str(_crc(d.orb_eng_sc)).encode())
        h.update(repr((d.dim, d.pbc, d.b_field, d.gauge, d.rescale, indptr.layout,
                       indptr.cutoff)).encode())
    else:
        for a in (indptr, indices, hop):
            a = np.asarray(a)
            h.update(repr((a.dtype.str, a.shape, _crc(a))).encode())
    h.update(repr((int(seed), int(n_timestep), int(n_samples), int(rank),
                   backend["precision"], int(backend["batch"]),
                   backend["state_kind"])).encode())
    return h.hexdigest()


def _load(path: str, fp: str) -> Optional[dict]:
    if not os.path.exists(path):
        return None
    try:
        with np.load(path) as z:
            if str(z["fingerprint"]) != fp:
                return None
            return {k: z[k] for k in z.files}
    except Exception:
        return None


def _save(path: str, **arrays) -> None:
    tmp = path + ".tmp.npz"
    np.savez(tmp, **arrays)
    os.replace(tmp, path)


def dos_checkpointed(bes, s_indptr, s_indices, s_hop, seed, n_timestep, n_ran_samples, rank,
                     wfn_chk_step, wfn_chk_thr, path: str, every: int = 256,
                     on_checkpoint: Optional[Callable[[int, int], None]] = None) -> np.ndarray:
    """f2py.tbpm_dos (tbpm.f90:6-93) with a checkpoint file at `path`.

    :param every: time steps between checkpoints
    :param on_checkpoint: called as on_checkpoint(first_state, rows_done)
        after every checkpoint write
    :return: (n_timestep+1,) complex128 correlation, as f2py.tbpm_dos
    """
    if every < 1:
        raise ValueError("every must be >= 1")
    if int(n_timestep) < 1:
        raise ValueError("n_timestep must be >= 1 for a checkpointed run")
    be = f2py.get_backend()
    bes = nat.as_c(bes, np.float64)
    ctx = f2py._ctx()
    tnr, n_avg = int(n_timestep), int(n_ran_samples)
    if hasattr(s_indptr, "make_resident"):
        n, _ = s_indptr.make_resident(ctx)
    else:
        ip, ix, hv, n, nnz = f2py._csr(s_indptr, s_indices, s_hop)
        ctx.call("tbpm_ham_upload", nat.ptr(ip), nat.ptr(ix), nat.ptr(hv), n, nnz, None, None,
                 1.0)
    fp = fingerprint(bes, s_indptr, s_indices, s_hop, seed, tnr, n_avg, rank, be)
    state = _load(path, fp)
    B = max(1, min(int(be["batch"]), 64))
    corr = np.zeros(tnr + 1, dtype=np.complex128)
    s0, done = 0, 0
    if state is not None:
        corr = state["corr"].copy()
        s0, done = int(state["s0"]), int(state["done"])
    thr = float(wfn_chk_thr)
    if be["precision"] == "fp32":
        thr = max(thr, float(be["fp32_chk_thr"]))
    while s0 < n_avg:
        nb = min(B, n_avg - s0)
        if state is not None and done > 0:
            wf0 = np.ascontiguousarray(state["wf0"])
            psi = np.ascontiguousarray(state["psi"])
            rc = np.ascontiguousarray(state["rows_corr"])
            rn = np.ascontiguousarray(state["rows_norm"])
            ctx.call("tbpm_session_dos_resume", nat.ptr(bes), bes.size, nb, nat.ptr(wf0),
                     nat.ptr(psi), nat.ptr(rc), nat.ptr(rn), done, tnr)
        else:
            wf0 = f2py.random_states(n, int(seed), nb, rank=int(rank), n_ran_samples=n_avg,
                                     first_sample=s0 + 1)
            ctx.call("tbpm_session_dos_resume", nat.ptr(bes), bes.size, nb, nat.ptr(wf0), None,
                     None, None, 0, tnr)
            done = 1
        state = None
        rows_c = rows_n = None
        while done < tnr + 1:
            k = min(int(every), tnr + 1 - done)
            ctx.call("tbpm_session_advance", int(k))
            done += k
            rows_c = np.zeros((tnr + 1, nb), dtype=np.complex128)
            rows_n = np.zeros((tnr + 1, nb), dtype=np.float64)
            got = ctypes.c_int(0)
            ctx.call("tbpm_session_read", nat.ptr(rows_c), nat.ptr(rows_n), ctypes.byref(got))
            # tbpm.f90:71-79: at t == wfn_chk_step the state after t-1 steps is
            # checked against the norm after the first step
            chk = int(wfn_chk_step)
            if 2 <= chk <= tnr and done - k <= chk - 1 < done:
                d = np.abs(rows_n[chk - 1] - rows_n[1])
                if np.any(~np.isfinite(rows_n[chk - 1])) or np.any(~np.isfinite(d)):
                    raise nat.NanError(nat.TBPM_ERR_NAN,
                                       f"tbpm_dos: the wave function norm is NaN or infinite "
                                       f"at time step {chk}")
                if np.any(d > thr):
                    raise nat.NormError(nat.TBPM_ERR_NORM,
                                        f"tbpm_dos: wave function norm gets broken during "
                                        f"propagation (time step {chk})")
            if done < tnr + 1:
                psi = np.zeros((nb, n), dtype=np.complex128)
                ctx.call("tbpm_session_export", None, nat.ptr(psi))
                _save(path, fingerprint=np.array(fp), corr=corr, s0=np.array(s0),
                      done=np.array(done), wf0=wf0, psi=psi, rows_corr=rows_c[:done],
                      rows_norm=rows_n[:done])
                if on_checkpoint is not None:
                    on_checkpoint(s0, done)
        # tbpm.f90:58-86: corr(t) += corrval / n_ran_samples, state by state;
        # real and imaginary parts are divided as reals (a complex division by
        # (n, 0) rounds differently)
        acc = corr.view(np.float64)
        for b in range(nb):
            acc += np.ascontiguousarray(rows_c[:, b]).view(np.float64) / n_avg
        s0 += nb
        done = 0
        if s0 < n_avg:
            _save(path, fingerprint=np.array(fp), corr=corr, s0=np.array(s0),
                  done=np.array(0), wf0=np.zeros(0), psi=np.zeros(0),
                  rows_corr=np.zeros(0), rows_norm=np.zeros(0))
            if on_checkpoint is not None:
                on_checkpoint(s0, 0)
    if os.path.exists(path):
        os.remove(path)
    return corr


def dc_checkpointed(bes, s_indptr, s_indices, s_hop, h_rescale, s_dx, s_dy, seed, n_timestep,
                    n_ran_samples, t_step, energies, en_inds, rank, wfn_chk_step, wfn_chk_thr,
                    path: str, states_per_part: Optional[int] = None,
                    on_checkpoint: Optional[Callable[[int], None]] = None):
    """f2py.tbpm_dccond (tbpm.f90:497-718) with a checkpoint file at `path`.

    A DC run keeps, per batch of states, the quasi-eigenstate block (N x
    energies x states complex values, tens of GB at the largest samples) on
    the device, so it is checkpointed between parts of the state list: the
    run is taken in parts of `states_per_part` states (default: the backend's
    batch width), each added to the DOS and DC correlations by
    tbpm_dccond_accumulate, and after every part the two arrays and the
    number of finished states are written atomically with a fingerprint of
    every input.  A later call with the same inputs continues after the last
    finished part and returns what an uninterrupted call with the same parts
    returns, bit for bit.

    :param on_checkpoint: called as on_checkpoint(states_done) after each write
    :return: (dos_corr (n_timestep,), dc_corr (2, len(energies), n_timestep) F-order)
    """
    be = f2py.get_backend()
    bes = nat.as_c(bes, np.float64)
    en = nat.as_c(energies, np.float64)
    ei = nat.as_c(en_inds, np.int32)
    tnr, n_avg = int(n_timestep), int(n_ran_samples)
    if tnr < 1 or n_avg < 1:
        raise ValueError("n_timestep and n_ran_samples must be >= 1")
    part = int(states_per_part) if states_per_part else max(1, min(int(be["batch"]), 32))
    if part < 1:
        raise ValueError("states_per_part must be >= 1")
    ctx = f2py._ctx()
    if hasattr(s_indptr, "make_resident"):
        s_indptr.make_resident(ctx)
    else:
        ip, ix, hv, n, nnz = f2py._csr(s_indptr, s_indices, s_hop)
        dx, dy = f2py._real(s_dx, nnz), f2py._real(s_dy, nnz)
        ctx.call("tbpm_ham_upload", nat.ptr(ip), nat.ptr(ix), nat.ptr(hv), n, nnz, nat.ptr(dx),
                 nat.ptr(dy), float(h_rescale))
    h = hashlib.sha256()
    h.update(fingerprint(bes, s_indptr, s_indices, s_hop, seed, tnr, n_avg, rank, be).encode())
    if not hasattr(s_indptr, "make_resident"):
        for a in (s_dx, s_dy):
            h.update(str(_crc(np.ascontiguousarray(a, dtype=np.float64))).encode())
    h.update(repr((float(h_rescale), float(t_step), part, int(wfn_chk_step),
                   float(wfn_chk_thr))).encode())
    h.update(en.tobytes())
    h.update(ei.tobytes())
    fp = h.hexdigest()
    state = _load(path, fp)
    dos = np.zeros(tnr, dtype=np.complex128)
    dc = np.zeros((2, en.size, tnr), dtype=np.complex128, order="F")
    s0 = 0
    if state is not None:
        dos = np.ascontiguousarray(state["dos"])
        dc = np.asfortranarray(state["dc"])
        s0 = int(state["s0"])
    while s0 < n_avg:
        k = min(part, n_avg - s0)
        ctx.call("tbpm_dccond_accumulate", nat.ptr(bes), bes.size, None, int(seed), int(rank),
                 n_avg, s0, k, tnr, float(t_step), nat.ptr(en), en.size, nat.ptr(ei), ei.size,
                 int(wfn_chk_step), float(wfn_chk_thr), nat.ptr(dos), nat.ptr(dc))
        s0 += k
        if s0 < n_avg:
            _save(path, fingerprint=np.array(fp), s0=np.array(s0), dos=dos, dc=dc)
            if on_checkpoint is not None:
                on_checkpoint(s0)
    if os.path.exists(path):
        os.remove(path)
    return dos, dc

"""Drop-in for the TBPM entry points of the reference module `tbplas.fortran.f2py`.

The reference builds this module with numpy.f2py from tbplas/fortran/tbpm.f90;
tbplas/tbpm/solver.py calls it positionally (solver.py:271, :335, :422, :589).
Here every function keeps the f2py-visible argument list, argument meaning,
dtype casts (int32 indices, complex128 values) and return layout (Fortran-order
arrays for 2-D/3-D outputs), and runs on the GPU through libtbpm_b200.

Backend knobs that the reference does not have (precision, batch width,
device, random-state distribution) live in `set_backend`, so the reference
call sites stay unchanged.
"""

from typing import Optional, Tuple

import numpy as np

from .. import _native as nat

__all__ = ["tbpm_dos", "tbpm_accond", "tbpm_dccond", "tbpm_psi_t", "tbpm_ldos",
           "tbpm_dyn_pol", "tbpm_eigenstates", "tbpm_kbdc", "ldos_haydock", "cond_from_trace",
           "tbpm_dos_states", "tbpm_accond_states", "tbpm_dccond_states",
           "tbpm_dyn_pol_states", "tbpm_eigenstates_states", "tbpm_kbdc_states",
           "haydock_coef", "tbpm_dos_segmented", "set_backend", "get_backend"]

_INT32_MAX = np.iinfo(np.int32).max

_backend = {
    "precision": "fp64",     # "fp64" | "fp32"
    "batch": 16,             # states propagated as one block
    "device": None,          # CUDA device (None: LOCAL_RANK or 0)
    "state_kind": "exp",     # "exp" (reference distribution) | "unit"
    "threads_per_block": 0,  # 0: tuned default
    "rows_per_tile": 0,      # 0: tuned default
    "steps_per_graph": 16,
    "use_graphs": True,
    "fp32_chk_thr": 1.0e-4,
    "vector_width": 0,       # complex values per thread: 0 auto (32-byte accesses), 1, 2
    "term_kernel": 0,        # Chebyshev-term kernel: 0 auto (shared-memory ring), 1 grid-stride
    "dc_budget_gb": 0.0,     # DC quasi-eigenstate memory budget in GiB (0: free memory)
    "verbose": False,
}


def set_backend(**kw) -> None:
    """Set backend options (see the module docstring)."""
    for k, v in kw.items():
        if k not in _backend:
            raise ValueError(f"unknown backend option {k}")
        if v is not None:
            _backend[k] = v
    if _backend["precision"] not in ("fp64", "fp32"):
        raise ValueError("precision must be 'fp64' or 'fp32'")
    if _backend["state_kind"] not in ("exp", "unit"):
        raise ValueError("state_kind must be 'exp' or 'unit'")


def get_backend() -> dict:
    return dict(_backend)


def _ctx() -> nat.Context:
    ctx = nat.get_context(_backend["device"])
    ctx.set_options(
        precision=nat.PREC_FP64 if _backend["precision"] == "fp64" else nat.PREC_FP32,
        batch=int(_backend["batch"]),
        state_kind=nat.STATE_EXP if _backend["state_kind"] == "exp" else nat.STATE_UNIT,
        threads_per_block=int(_backend["threads_per_block"]),
        rows_per_tile=int(_backend["rows_per_tile"]),
        steps_per_graph=int(_backend["steps_per_graph"]),
        use_graphs=1 if _backend["use_graphs"] else 0,
        fp32_chk_thr=float(_backend["fp32_chk_thr"]),
        vector_width=int(_backend["vector_width"]),
        term_kernel=int(_backend["term_kernel"]),
        dc_budget_gb=float(_backend["dc_budget_gb"]),
    )
    return ctx


def _csr(indptr, indices, hop):
    """f2py casts: INTEGER (int32) index arrays, COMPLEX(KIND=8) values.

    In the place of indptr a handle of a device-assembled Hamiltonian
    (tbplas_b200.supercell.ResidentHam) may be given: it is assembled in the
    context and the drivers get NULL arrays (the resident Hamiltonian)."""
    if hasattr(indptr, "make_resident"):
        n, nnz = indptr.make_resident(_ctx())
        return None, None, None, n, nnz
    indptr = np.asarray(indptr)
    indices = np.asarray(indices)
    if indptr.size and int(indptr.max()) > _INT32_MAX:
        raise ValueError("indptr exceeds the int32 range")
    ip = nat.as_c(indptr, np.int32)
    ix = nat.as_c(indices, np.int32)
    hv = nat.as_c(hop, np.complex128)
    if ip.ndim != 1 or ip.size < 2:
        raise ValueError("indptr must be 1-D with at least 2 entries")
    if ix.size != hv.size:
        raise ValueError("indices and hop must have the same length")
    return ip, ix, hv, ip.size - 1, hv.size


def _real(a, n) -> Optional[np.ndarray]:
    if a is None:
        return None
    r = nat.as_c(a, np.float64)
    if r.size != n:
        raise ValueError("dx/dy must have the same length as hop")
    return r


def _say(rank: int, text: str) -> None:
    if _backend["verbose"] and rank == 0:
        print(text, flush=True)


def tbpm_dos(bes, s_indptr, s_indices, s_hop, seed, n_timestep, n_ran_samples,
             output_filename, rank, wfn_chk_step, wfn_chk_thr) -> np.ndarray:
    """DOS correlation function (tbpm.f90:6-93).

    :return: (n_timestep+1,) complex128, corr[t] = <psi0|exp(-iHt dt)|psi0>
        averaged over n_ran_samples random states
    """
    del output_filename  # only written by the reference's DEBUG build
    bes = nat.as_c(bes, np.float64)
    ip, ix, hv, n, nnz = _csr(s_indptr, s_indices, s_hop)
    corr = np.zeros(int(n_timestep) + 1, dtype=np.complex128)
    _say(rank, "Calculating DOS correlation function.")
    _ctx().call("tbpm_dos", nat.ptr(bes), bes.size, nat.ptr(ip), nat.ptr(ix), nat.ptr(hv),
                n, nnz, int(seed), int(n_timestep), int(n_ran_samples), int(rank),
                int(wfn_chk_step), float(wfn_chk_thr), nat.ptr(corr))
    return corr


def tbpm_dos_states(bes, s_indptr, s_indices, s_hop, wf0, n_timestep, wfn_chk_step,
                    wfn_chk_thr, per_state: bool = False):
    """tbpm_dos with caller-supplied initial states wf0 (n_states, n_orb).

    :return: averaged corr (n_timestep+1,), and with per_state=True also the
        unaveraged (n_states, n_timestep+1) correlations
    """
    bes = nat.as_c(bes, np.float64)
    ip, ix, hv, n, nnz = _csr(s_indptr, s_indices, s_hop)
    w = nat.as_c(np.atleast_2d(wf0), np.complex128)
    if w.shape[1] != n:
        raise ValueError("wf0 must have shape (n_states, n_orbitals)")
    corr = np.zeros(int(n_timestep) + 1, dtype=np.complex128)
    per = np.zeros((w.shape[0], int(n_timestep) + 1), dtype=np.complex128) if per_state else None
    _ctx().call("tbpm_dos_states", nat.ptr(bes), bes.size, nat.ptr(ip), nat.ptr(ix),
                nat.ptr(hv), n, nnz, nat.ptr(w), w.shape[0], int(n_timestep),
                int(wfn_chk_step), float(wfn_chk_thr), nat.ptr(corr), nat.ptr(per))
    return (corr, per) if per_state else corr


def tbpm_ldos(site_indices, bes, s_indptr, s_indices, s_hop, seed, n_timestep,
              n_ran_samples, output_filename, rank, wfn_chk_step, wfn_chk_thr) -> np.ndarray:
    """LDOS correlation function (tbpm.f90:97-189).

    The random state is restricted to site_indices and renormalised; then
    corr[k] = <wf0|wf_k> for k = 0..n_timestep with wf_0 = wf0.
    """
    del output_filename
    bes = nat.as_c(bes, np.float64)
    ip, ix, hv, n, nnz = _csr(s_indptr, s_indices, s_hop)
    sites = np.asarray(site_indices, dtype=np.int64)
    if sites.size == 0 or sites.min() < 0 or sites.max() >= n:
        raise ValueError("site_indices out of range")
    ctx = _ctx()
    full = np.zeros((int(n_ran_samples), n), dtype=np.complex128)
    kind = nat.STATE_EXP if _backend["state_kind"] == "exp" else nat.STATE_UNIT
    ctx.call("tbpm_random_states", n, int(seed), 1, int(n_ran_samples), int(rank),
             int(n_ran_samples), kind, nat.ptr(full))
    wf0 = np.zeros_like(full)
    wf0[:, sites] = full[:, sites]
    wf0 /= np.sqrt(np.sum(np.abs(wf0) ** 2, axis=1, keepdims=True))
    _say(rank, "Calculating LDOS correlation function.")
    corr = np.zeros(int(n_timestep) + 1, dtype=np.complex128)
    ctx.call("tbpm_dos_states", nat.ptr(bes), bes.size, nat.ptr(ip), nat.ptr(ix), nat.ptr(hv),
             n, nnz, nat.ptr(wf0), wf0.shape[0], int(n_timestep),
             int(wfn_chk_step), float(wfn_chk_thr), nat.ptr(corr), None)
    return corr


def tbpm_accond(bes, beta, mu, s_indptr, s_indices, s_hop, h_rescale, s_dx, s_dy, seed,
                n_timestep, n_ran_samples, nr_fermi, fermi_precision, output_filename, rank,
                wfn_chk_step, wfn_chk_thr) -> np.ndarray:
    """AC conductivity correlation function (tbpm.f90:193-351).

    :return: (4, n_timestep) complex128, Fortran order, rows xx, xy, yx, yy;
        column 0 is zero as in the reference
    """
    del output_filename
    bes = nat.as_c(bes, np.float64)
    ip, ix, hv, n, nnz = _csr(s_indptr, s_indices, s_hop)
    dx, dy = _real(s_dx, nnz), _real(s_dy, nnz)
    corr = np.zeros((4, int(n_timestep)), dtype=np.complex128, order="F")
    _say(rank, "Calculating AC conductivity correlation function.")
    _ctx().call("tbpm_accond", nat.ptr(bes), bes.size, float(beta), float(mu), nat.ptr(ip),
                nat.ptr(ix), nat.ptr(hv), n, nnz, float(h_rescale), nat.ptr(dx), nat.ptr(dy),
                int(seed), int(n_timestep), int(n_ran_samples), int(nr_fermi),
                float(fermi_precision), int(rank), int(wfn_chk_step), float(wfn_chk_thr),
                nat.ptr(corr))
    return corr


def tbpm_accond_states(bes, beta, mu, s_indptr, s_indices, s_hop, h_rescale, s_dx, s_dy,
                       wf0, n_timestep, nr_fermi, fermi_precision, wfn_chk_step,
                       wfn_chk_thr) -> np.ndarray:
    """tbpm_accond with caller-supplied initial states wf0 (n_states, n_orb)."""
    bes = nat.as_c(bes, np.float64)
    ip, ix, hv, n, nnz = _csr(s_indptr, s_indices, s_hop)
    dx, dy = _real(s_dx, nnz), _real(s_dy, nnz)
    w = nat.as_c(np.atleast_2d(wf0), np.complex128)
    if w.shape[1] != n:
        raise ValueError("wf0 must have shape (n_states, n_orbitals)")
    corr = np.zeros((4, int(n_timestep)), dtype=np.complex128, order="F")
    _ctx().call("tbpm_accond_states", nat.ptr(bes), bes.size, float(beta), float(mu),
                nat.ptr(ip), nat.ptr(ix), nat.ptr(hv), n, nnz, float(h_rescale), nat.ptr(dx),
                nat.ptr(dy), nat.ptr(w), w.shape[0], int(n_timestep), int(nr_fermi),
                float(fermi_precision), int(wfn_chk_step), float(wfn_chk_thr), nat.ptr(corr))
    return corr


def tbpm_dccond(bes, beta, mu, s_indptr, s_indices, s_hop, h_rescale, s_dx, s_dy, seed,
                n_timestep, n_ran_samples, t_step, energies, en_inds, output_filename_dos,
                output_filename_dc, rank, wfn_chk_step,
                wfn_chk_thr) -> Tuple[np.ndarray, np.ndarray]:
    """DC conductivity correlation functions (tbpm.f90:497-718).

    :return: (dos_corr, dc_corr): (n_timestep,) complex128 and
        (2, len(energies), n_timestep) complex128 Fortran order; only the first
        len(en_inds) rows of the energy axis are filled, as in the reference
    """
    del output_filename_dos, output_filename_dc
    bes = nat.as_c(bes, np.float64)
    ip, ix, hv, n, nnz = _csr(s_indptr, s_indices, s_hop)
    dx, dy = _real(s_dx, nnz), _real(s_dy, nnz)
    en = nat.as_c(energies, np.float64)
    ei = nat.as_c(en_inds, np.int32)
    dos = np.zeros(int(n_timestep), dtype=np.complex128)
    dc = np.zeros((2, en.size, int(n_timestep)), dtype=np.complex128, order="F")
    _say(rank, "Calculating DC conductivity correlation function.")
    _ctx().call("tbpm_dccond", nat.ptr(bes), bes.size, float(beta), float(mu), nat.ptr(ip),
                nat.ptr(ix), nat.ptr(hv), n, nnz, float(h_rescale), nat.ptr(dx), nat.ptr(dy),
                int(seed), int(n_timestep), int(n_ran_samples), float(t_step), nat.ptr(en),
                en.size, nat.ptr(ei), ei.size, int(rank), int(wfn_chk_step),
                float(wfn_chk_thr), nat.ptr(dos), nat.ptr(dc))
    return dos, dc


def tbpm_dccond_states(bes, s_indptr, s_indices, s_hop, h_rescale, s_dx, s_dy, wf0,
                       n_timestep, t_step, energies, en_inds, wfn_chk_step,
                       wfn_chk_thr) -> Tuple[np.ndarray, np.ndarray]:
    """tbpm_dccond with caller-supplied initial states wf0 (n_states, n_orb)."""
    bes = nat.as_c(bes, np.float64)
    ip, ix, hv, n, nnz = _csr(s_indptr, s_indices, s_hop)
    dx, dy = _real(s_dx, nnz), _real(s_dy, nnz)
    w = nat.as_c(np.atleast_2d(wf0), np.complex128)
    if w.shape[1] != n:
        raise ValueError("wf0 must have shape (n_states, n_orbitals)")
    en = nat.as_c(energies, np.float64)
    ei = nat.as_c(en_inds, np.int32)
    dos = np.zeros(int(n_timestep), dtype=np.complex128)
    dc = np.zeros((2, en.size, int(n_timestep)), dtype=np.complex128, order="F")
    _ctx().call("tbpm_dccond_states", nat.ptr(bes), bes.size, nat.ptr(ip), nat.ptr(ix),
                nat.ptr(hv), n, nnz, float(h_rescale), nat.ptr(dx), nat.ptr(dy), nat.ptr(w),
                w.shape[0], int(n_timestep), float(t_step), nat.ptr(en), en.size, nat.ptr(ei),
                ei.size, int(wfn_chk_step), float(wfn_chk_thr), nat.ptr(dos), nat.ptr(dc))
    return dos, dc


def tbpm_psi_t(bes, indptr, indices, hop, psi0, time_log, n_timestep, wfn_chk_step,
               wfn_chk_thr) -> np.ndarray:
    """Time-dependent wave function (tbpm.f90:1029-1093).

    :return: (n_psi0, n_time_log) complex128, Fortran order
    """
    bes = nat.as_c(bes, np.float64)
    ip, ix, hv, n, nnz = _csr(indptr, indices, hop)
    p0 = nat.as_c(psi0, np.complex128)
    if p0.size != n:
        raise ValueError("psi0 must have n_orbitals entries")
    tl = nat.as_c(time_log, np.int32)
    psi_t = np.zeros((n, tl.size), dtype=np.complex128, order="F")
    _ctx().call("tbpm_psi_t", nat.ptr(bes), bes.size, nat.ptr(ip), nat.ptr(ix), nat.ptr(hv), n,
                nnz, nat.ptr(p0), nat.ptr(tl), tl.size, int(n_timestep), int(wfn_chk_step),
                float(wfn_chk_thr), nat.ptr(psi_t))
    return psi_t



def _sites(site_x, site_y, site_z, n):
    xs = [nat.as_c(a, np.float64) for a in (site_x, site_y, site_z)]
    if any(a.size != n for a in xs):
        raise ValueError("site_x/y/z must have one entry per orbital")
    return xs


def _q_points(q_points) -> np.ndarray:
    q = nat.as_c(np.atleast_2d(np.asarray(q_points, dtype=np.float64)), np.float64)
    if q.ndim != 2 or q.shape[1] != 3:
        raise ValueError("q_points must have shape (n_q_points, 3)")
    return q


def tbpm_dyn_pol(bes, beta, mu, s_indptr, s_indices, s_hop, h_rescale, s_dx, s_dy, s_site_x,
                 s_site_y, s_site_z, seed, n_timestep, n_ran_samples, nr_fermi,
                 fermi_precision, q_points, output_filename, rank, wfn_chk_step,
                 wfn_chk_thr) -> np.ndarray:
    """Dynamical polarisation correlation function (tbpm.f90:355-493).

    :return: (n_q_points, n_timestep) float64, Fortran order
    """
    del output_filename
    bes = nat.as_c(bes, np.float64)
    ip, ix, hv, n, nnz = _csr(s_indptr, s_indices, s_hop)
    dx, dy = _real(s_dx, nnz), _real(s_dy, nnz)
    sx, sy, sz = _sites(s_site_x, s_site_y, s_site_z, n)
    q = _q_points(q_points)
    corr = np.zeros((q.shape[0], int(n_timestep)), dtype=np.float64, order="F")
    _say(rank, "Calculating dynamical polarization correlation function.")
    _ctx().call("tbpm_dyn_pol", nat.ptr(bes), bes.size, float(beta), float(mu), nat.ptr(ip),
                nat.ptr(ix), nat.ptr(hv), n, nnz, float(h_rescale), nat.ptr(dx), nat.ptr(dy),
                nat.ptr(sx), nat.ptr(sy), nat.ptr(sz), int(seed), int(n_timestep),
                int(n_ran_samples), int(nr_fermi), float(fermi_precision), nat.ptr(q),
                q.shape[0], int(rank), int(wfn_chk_step), float(wfn_chk_thr), nat.ptr(corr))
    return corr


def tbpm_dyn_pol_states(bes, beta, mu, s_indptr, s_indices, s_hop, site_x, site_y, site_z,
                        q_points, wf0, n_timestep, nr_fermi, fermi_precision, wfn_chk_step,
                        wfn_chk_thr) -> np.ndarray:
    """tbpm_dyn_pol with caller-supplied initial states wf0 (n_states, n_orb)."""
    bes = nat.as_c(bes, np.float64)
    ip, ix, hv, n, nnz = _csr(s_indptr, s_indices, s_hop)
    sx, sy, sz = _sites(site_x, site_y, site_z, n)
    q = _q_points(q_points)
    w = nat.as_c(np.atleast_2d(wf0), np.complex128)
    if w.shape[1] != n:
        raise ValueError("wf0 must have shape (n_states, n_orbitals)")
    corr = np.zeros((q.shape[0], int(n_timestep)), dtype=np.float64, order="F")
    _ctx().call("tbpm_dyn_pol_states", nat.ptr(bes), bes.size, float(beta), float(mu),
                nat.ptr(ip), nat.ptr(ix), nat.ptr(hv), n, nnz, nat.ptr(sx), nat.ptr(sy),
                nat.ptr(sz), nat.ptr(q), q.shape[0], nat.ptr(w), w.shape[0], int(n_timestep),
                int(nr_fermi), float(fermi_precision), int(wfn_chk_step), float(wfn_chk_thr),
                nat.ptr(corr))
    return corr


def tbpm_eigenstates(bes, s_indptr, s_indices, s_hop, seed, n_timestep, n_ran_samples, t_step,
                     energies, rank, wfn_chk_step, wfn_chk_thr) -> np.ndarray:
    """Quasi-eigenstates (tbpm.f90:721-830).

    :return: (n_energies, n_orbitals) float64, Fortran order
    """
    bes = nat.as_c(bes, np.float64)
    ip, ix, hv, n, nnz = _csr(s_indptr, s_indices, s_hop)
    en = nat.as_c(energies, np.float64).reshape(-1)
    out = np.zeros((en.size, n), dtype=np.float64, order="F")
    _say(rank, "Calculating quasi-eigenstates.")
    _ctx().call("tbpm_eigenstates", nat.ptr(bes), bes.size, nat.ptr(ip), nat.ptr(ix),
                nat.ptr(hv), n, nnz, int(seed), int(n_timestep), int(n_ran_samples),
                float(t_step), nat.ptr(en), en.size, int(rank), int(wfn_chk_step),
                float(wfn_chk_thr), nat.ptr(out))
    return out


def tbpm_eigenstates_states(bes, s_indptr, s_indices, s_hop, wf0, n_timestep, t_step,
                            energies, wfn_chk_step, wfn_chk_thr) -> np.ndarray:
    """tbpm_eigenstates with caller-supplied initial states wf0 (n_states, n_orb)."""
    bes = nat.as_c(bes, np.float64)
    ip, ix, hv, n, nnz = _csr(s_indptr, s_indices, s_hop)
    en = nat.as_c(energies, np.float64).reshape(-1)
    w = nat.as_c(np.atleast_2d(wf0), np.complex128)
    if w.shape[1] != n:
        raise ValueError("wf0 must have shape (n_states, n_orbitals)")
    out = np.zeros((en.size, n), dtype=np.float64, order="F")
    _ctx().call("tbpm_eigenstates_states", nat.ptr(bes), bes.size, nat.ptr(ip), nat.ptr(ix),
                nat.ptr(hv), n, nnz, nat.ptr(w), w.shape[0], int(n_timestep), float(t_step),
                nat.ptr(en), en.size, int(wfn_chk_step), float(wfn_chk_thr), nat.ptr(out))
    return out


def tbpm_kbdc(seed, s_indptr, s_indices, s_hop, h_rescale, s_dx, s_dy, n_ran_samples,
              n_kernel, direction, rank) -> np.ndarray:
    """Kubo-Bastin moments mu_mn (tbpm.f90:836-960).

    :return: (n_kernel, n_kernel) complex128, Fortran order
    """
    ip, ix, hv, n, nnz = _csr(s_indptr, s_indices, s_hop)
    dx, dy = _real(s_dx, nnz), _real(s_dy, nnz)
    mu = np.zeros((int(n_kernel), int(n_kernel)), dtype=np.complex128, order="F")
    _say(rank, "Calculating Kubo-Bastin moments.")
    _ctx().call("tbpm_kbdc", int(seed), nat.ptr(ip), nat.ptr(ix), nat.ptr(hv), n, nnz,
                float(h_rescale), nat.ptr(dx), nat.ptr(dy), int(n_ran_samples), int(n_kernel),
                int(direction), int(rank), nat.ptr(mu))
    return mu


def tbpm_kbdc_states(s_indptr, s_indices, s_hop, h_rescale, s_dx, s_dy, wf0, n_kernel,
                     direction) -> np.ndarray:
    """tbpm_kbdc with caller-supplied initial states wf0 (n_states, n_orb)."""
    ip, ix, hv, n, nnz = _csr(s_indptr, s_indices, s_hop)
    dx, dy = _real(s_dx, nnz), _real(s_dy, nnz)
    w = nat.as_c(np.atleast_2d(wf0), np.complex128)
    if w.shape[1] != n:
        raise ValueError("wf0 must have shape (n_states, n_orbitals)")
    mu = np.zeros((int(n_kernel), int(n_kernel)), dtype=np.complex128, order="F")
    _ctx().call("tbpm_kbdc_states", nat.ptr(ip), nat.ptr(ix), nat.ptr(hv), n, nnz,
                float(h_rescale), nat.ptr(dx), nat.ptr(dy), nat.ptr(w), w.shape[0],
                int(n_kernel), int(direction), nat.ptr(mu))
    return mu


def haydock_coef(site_indices, s_indptr, s_indices, s_hop, h_rescale, n_depth, wf_sites):
    """Sample-averaged Haydock coefficients (propagation.f90:85-155) for start
    vectors with amplitudes wf_sites (n_samples, n_sites) on site_indices.

    :return: (coefa complex128[n_depth], coefb float64[n_depth])
    """
    ip, ix, hv, n, nnz = _csr(s_indptr, s_indices, s_hop)
    sites = nat.as_c(site_indices, np.int32).reshape(-1)
    w = nat.as_c(np.atleast_2d(wf_sites), np.complex128)
    if w.shape[1] != sites.size:
        raise ValueError("wf_sites must have shape (n_samples, n_sites)")
    a = np.zeros(int(n_depth), dtype=np.complex128)
    b = np.zeros(int(n_depth), dtype=np.float64)
    _ctx().call("tbpm_haydock_coef", nat.ptr(ip), nat.ptr(ix), nat.ptr(hv), n, nnz,
                float(h_rescale), nat.ptr(sites), sites.size, nat.ptr(w), w.shape[0],
                int(n_depth), nat.ptr(a), nat.ptr(b))
    return a, b


def green_function(energies, delta, coefa, coefb) -> np.ndarray:
    """G00(E + i delta) of the Haydock continued fraction (funcs.f90:152-172),
    for all energies at once."""
    e = np.asarray(energies, dtype=np.float64) + 1j * float(delta)
    g = np.zeros(e.shape, dtype=np.complex128)
    for i in range(len(coefa) - 1, -1, -1):
        g = 1.0 / (e - coefa[i] - coefb[i] ** 2 * g)
    return g


def ldos_haydock(site_indices, delta, e_range, s_indptr, s_indices, s_hop, h_rescale, seed,
                 n_depth, n_timestep, n_ran_samples, output_filename):
    """LDOS by the Haydock recursion (tbpm.f90:963-1026).

    The random start vectors live on site_indices only and are drawn over those
    sites with the seed rule seed*i_sample (tbpm.f90:1004).

    :return: (energy, ldos), both float64[2*n_timestep+1]
    """
    del output_filename
    sites = np.asarray(site_indices, dtype=np.int64).reshape(-1)
    n_sites = sites.size
    if n_sites == 0:
        raise ValueError("site_indices must not be empty")
    wf = random_states(n_sites, int(seed), int(n_ran_samples), rank=0,
                       n_ran_samples=int(n_ran_samples))
    a, b = haydock_coef(sites, s_indptr, s_indices, s_hop, h_rescale, n_depth, wf)
    tnr = int(n_timestep)
    energy = np.array([0.5 * i * e_range / tnr for i in range(-tnr, tnr + 1)])
    g = green_function(energy, delta, a, b)
    return energy, -1.0 / np.pi * g.imag


def cond_from_trace(mu_mn, mu, h_rescale, beta, ne_integral, fermi_precision,
                    rank) -> np.ndarray:
    """Hall conductivity trace of analysis.f90:6-69 (before the Analyzer's
    prefactor), evaluated on the GPU.

    :return: float64[len(mu)]
    """
    m = np.asfortranarray(np.asarray(mu_mn, dtype=np.complex128))
    if m.ndim != 2 or m.shape[0] != m.shape[1]:
        raise ValueError("mu_mn must be a square (n_kernel, n_kernel) array")
    mus = nat.as_c(mu, np.float64).reshape(-1)
    cond = np.zeros(mus.size, dtype=np.float64)
    _ctx().call("tbpm_cond_from_trace", m.ctypes.data, m.shape[0], nat.ptr(mus), mus.size,
                float(h_rescale), float(beta), int(ne_integral), float(fermi_precision),
                int(rank), nat.ptr(cond))
    return cond

def random_states(n_orbitals: int, seed: int, n_states: int, rank: int = 0,
                  n_ran_samples: Optional[int] = None, first_sample: int = 1,
                  kind: Optional[str] = None) -> np.ndarray:
    """The random initial states the drivers use (random.f90:36-69 distribution,
    seed rule of tbpm.f90:57), as (n_states, n_orbitals) complex128."""
    k = _backend["state_kind"] if kind is None else kind
    out = np.zeros((int(n_states), int(n_orbitals)), dtype=np.complex128)
    nrs = int(n_states) if n_ran_samples is None else int(n_ran_samples)
    _ctx().call("tbpm_random_states", int(n_orbitals), int(seed), int(first_sample),
                int(n_states), int(rank), nrs,
                nat.STATE_EXP if k == "exp" else nat.STATE_UNIT, nat.ptr(out))
    return out


def tbpm_dos_segmented(bes, indptr, indices, hop, seg_offsets, n_states, seed, n_timestep,
                       wfn_chk_step=128, wfn_chk_thr=1.0e-9, per_state: bool = False):
    """DOS correlations of a batch of realisations packed block-diagonally
    (tbplas_b200.builder.pack_samples), propagated together.

    :param seg_offsets: (n_seg+1,) row offsets of the realisations
    :return: (n_seg, n_timestep+1) complex128, the state average per
        realisation; with per_state=True also (n_seg, n_states, n_timestep+1)
    """
    bes = nat.as_c(bes, np.float64)
    ip, ix, hv, n, nnz = _csr(indptr, indices, hop)
    off = nat.as_c(seg_offsets, np.int64)
    n_seg = off.size - 1
    corr = np.zeros((n_seg, int(n_timestep) + 1), dtype=np.complex128)
    per = (np.zeros((n_seg, int(n_states), int(n_timestep) + 1), dtype=np.complex128)
           if per_state else None)
    _ctx().call("tbpm_dos_segmented", nat.ptr(bes), bes.size, nat.ptr(ip), nat.ptr(ix),
                nat.ptr(hv), n, nnz, nat.ptr(off), n_seg, int(n_states), int(seed),
                int(n_timestep), int(wfn_chk_step), float(wfn_chk_thr), nat.ptr(corr),
                nat.ptr(per))
    return (corr, per) if per_state else corr

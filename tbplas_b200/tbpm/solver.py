"""TBPM Solver: the reference `tbplas.tbpm.Solver` API on the B200 backend.

Method names, arguments, returned shapes, output files and parameter handling
follow tbplas/tbpm/solver.py; the numeric core (the reference's f2py calls,
solver.py:271, :335, :422, :589) is tbplas_b200.fortran.f2py, i.e. the CUDA
library.  `sample` is any object with the TBPM-facing interface of
tbplas.Sample (build_ham_csr, build_ham_dxy, energy_range, rescale), e.g. a
tbplas Sample or tbplas_b200.builder.LatticeSample.
"""

import math
import os
import pickle
import time
from typing import List, Tuple

import numpy as np
import scipy.special as spec

from ..base import H_BAR_EV
from ..fortran import f2py
from ..parallel import MPIEnv
from .config import Config

__all__ = ["Solver"]


class Solver(MPIEnv):
    """Driver of the TBPM correlation functions.

    :param sample: sample for which TBPM calculations will be performed
    :param config: parameters controlling TBPM calculations
    :param enable_mpi: split random samples over the torch.distributed ranks
    :param echo_details: print parallelisation details
    :param backend: GPU backend options (see tbplas_b200.fortran.f2py.set_backend:
        precision 'fp64'/'fp32', batch, device, ...); not part of Config so that
        Config.check_params keeps the reference's key set
    :param checkpoint: optional {'path': file, 'every': time steps}: calc_corr_dos
        writes its state to path every `every` steps and resumes from it when
        called again with the same inputs (tbplas_b200.checkpoint); each rank
        uses path + '.rank<r>'.  calc_corr_dc_cond writes path + '.dc' after every
        'states_per_part' states (default: the batch width) and resumes from it
    :param kwargs: arguments of set_output
    """

    def __init__(self, sample, config: Config, enable_mpi: bool = False,
                 echo_details: bool = True, backend: dict = None, checkpoint: dict = None,
                 **kwargs) -> None:
        super().__init__(enable_mpi=enable_mpi, echo_details=echo_details)
        self._sample = sample
        self._config = config
        self._config.check_params()
        self._backend = dict(backend or {})
        self._checkpoint = dict(checkpoint) if checkpoint else None
        self._output = dict()
        self.set_output(**kwargs)

    # -- output files (solver.py:95-153) --------------------------------------
    def set_output(self, directory: str = "sim_data", prefix: str = None) -> None:
        self._output["directory"] = directory
        if prefix is None:
            prefix = str(int(time.time()))
        self._output["prefix"] = prefix
        if self.is_master and not os.path.exists(directory):
            os.makedirs(directory, exist_ok=True)
        self.barrier()
        for key in ("corr_DOS", "corr_LDOS", "corr_AC", "corr_dyn_pol", "corr_DC",
                    "hall_mu", "qe", "ldos_haydock", "psi_t"):
            self._output[key] = f"{directory}/{prefix}.{key}"
        spaces = " " * 2
        self.print("Output details:")
        self.print(f"{spaces}{'Directory':11s}: {directory}")
        self.print(f"{spaces}{'Prefix':11s}: {prefix}")
        self.print()
        self.save_config()

    def save_config(self, filename: str = "config.pkl") -> None:
        if self.is_master:
            directory, prefix = self._output["directory"], self._output["prefix"]
            with open(f"{directory}/{prefix}.{filename}", 'wb') as f:
                pickle.dump(self._config, f, pickle.HIGHEST_PROTOCOL)

    @property
    def output(self) -> dict:
        return self._output

    # -- parameter helpers (solver.py:155-254) ---------------------------------
    def _dist_sample(self) -> int:
        """Random samples of this rank; nr_random_samples padded to a multiple
        of the number of ranks (solver.py:155-173)."""
        num_sample_opt = self._config.generic["nr_random_samples"]
        if self.mpi_enabled:
            while num_sample_opt % self.size != 0:
                num_sample_opt += 1
            if num_sample_opt != self._config.generic["nr_random_samples"]:
                self.print(f"\nWARNING:\n  nr_random_samples adjusted to "
                           f"{num_sample_opt} for optimal balance")
                self._config.generic["nr_random_samples"] = num_sample_opt
            return num_sample_opt // self.size
        return num_sample_opt

    def _get_time_step(self) -> float:
        """time_step = 2*pi / energy_range in h_bar/eV (solver.py:175-182)."""
        return 2 * math.pi / self._sample.energy_range

    def _echo_time_step_fs(self, time_step: float) -> None:
        time_step_fs = time_step * H_BAR_EV * 1e15
        self.print(f"Time step for propagation: {time_step_fs:7.3f} fs\n")

    def _get_bessel_series(self, time_step: float) -> List[float]:
        """J_n(time_step*rescale) kept while |J_n| or |J_{n+1}| exceeds
        Bessel_precision (solver.py:194-224)."""
        bessel_max = self._config.generic["Bessel_max"]
        bessel_precision = self._config.generic["Bessel_precision"]
        time_scaled = time_step * self._sample.rescale
        series = []
        for i in range(bessel_max):
            val = spec.jv(i, time_scaled)
            if np.abs(val) > bessel_precision:
                series.append(val)
            elif np.abs(spec.jv(i + 1, time_scaled).item()) > bessel_precision:
                series.append(val)
            else:
                return series
        raise ValueError("Bessel_max too low")

    def _get_beta_mu_re(self) -> Tuple[float, float]:
        return (self._config.generic['beta'] * self._sample.rescale,
                self._config.generic['mu'] / self._sample.rescale)

    def _save_data(self, data: np.ndarray, file_name: str,
                   output_format: str = "numpy") -> None:
        if output_format not in ("numpy", "npy"):
            raise NotImplementedError(f"Unsupported format {output_format}")
        if self.is_master:
            np.save(f"{file_name}.npy", data)

    def _apply_backend(self) -> None:
        if self._backend:
            f2py.set_backend(**self._backend)

    # -- correlation functions --------------------------------------------------
    def calc_corr_dos(self) -> np.ndarray:
        """DOS correlation function, (nr_time_steps+1,) complex128 (solver.py:256-284)."""
        self._apply_backend()
        time_step = self._get_time_step()
        bessel_series = self._get_bessel_series(time_step)
        ham_csr = self._sample.build_ham_csr()
        num_sample = self._dist_sample()
        self._echo_time_step_fs(time_step)
        if self._checkpoint:
            from ..checkpoint import dos_checkpointed
            path = self._checkpoint["path"]
            if self.size > 1:
                path = f"{path}.rank{self.rank}"
            corr_dos = dos_checkpointed(
                bessel_series, ham_csr.indptr, ham_csr.indices, ham_csr.data,
                self._config.generic['seed'], self._config.generic['nr_time_steps'],
                num_sample, self.rank, self._config.generic['wfn_check_steps'],
                self._config.generic['wfn_check_thr'], path,
                every=int(self._checkpoint.get("every", 256)),
                on_checkpoint=self._checkpoint.get("on_checkpoint"))
        else:
            corr_dos = f2py.tbpm_dos(
                bessel_series, ham_csr.indptr, ham_csr.indices, ham_csr.data,
                self._config.generic['seed'], self._config.generic['nr_time_steps'],
                num_sample, self._output['corr_DOS'], self.rank,
                self._config.generic['wfn_check_steps'], self._config.generic['wfn_check_thr'])
        corr_dos = self.all_average(corr_dos)
        self._save_data(corr_dos, self._output["corr_DOS"])
        return corr_dos

    def calc_corr_ldos(self) -> np.ndarray:
        """LDOS correlation function, (nr_time_steps+1,) complex128."""
        self._apply_backend()
        time_step = self._get_time_step()
        bessel_series = self._get_bessel_series(time_step)
        ham_csr = self._sample.build_ham_csr()
        num_sample = self._dist_sample()
        self._echo_time_step_fs(time_step)
        corr_ldos = f2py.tbpm_ldos(
            self._config.LDOS['site_indices'], bessel_series,
            ham_csr.indptr, ham_csr.indices, ham_csr.data,
            self._config.generic['seed'], self._config.generic['nr_time_steps'],
            num_sample, self._output['corr_LDOS'], self.rank,
            self._config.generic['wfn_check_steps'], self._config.generic['wfn_check_thr'])
        corr_ldos = self.all_average(corr_ldos)
        self._save_data(corr_ldos, self._output["corr_LDOS"])
        return corr_ldos

    def calc_corr_ac_cond(self) -> np.ndarray:
        """AC conductivity correlation, (4, nr_time_steps) complex128 in the
        order xx, xy, yx, yy (solver.py:317-352)."""
        self._apply_backend()
        time_step = 0.5 * self._get_time_step()
        bessel_series = self._get_bessel_series(time_step)
        beta_re, mu_re = self._get_beta_mu_re()
        indptr, indices, hop, dx, dy = self._sample.build_ham_dxy()
        num_sample = self._dist_sample()
        self._echo_time_step_fs(time_step)
        corr_ac = f2py.tbpm_accond(
            bessel_series, beta_re, mu_re, indptr, indices, hop,
            self._sample.rescale, dx, dy,
            self._config.generic['seed'], self._config.generic['nr_time_steps'], num_sample,
            self._config.generic['nr_Fermi_fft_steps'],
            self._config.generic['Fermi_cheb_precision'],
            self._output['corr_AC'], self.rank,
            self._config.generic['wfn_check_steps'], self._config.generic['wfn_check_thr'])
        corr_ac = self.all_average(corr_ac)
        self._save_data(corr_ac, self._output["corr_AC"])
        return corr_ac

    def calc_corr_dc_cond(self) -> Tuple[np.ndarray, np.ndarray]:
        """DOS and DC conductivity correlations, (nr_time_steps,) and
        (2, 2*nr_time_steps, nr_time_steps) complex128 (solver.py:393-441)."""
        self._apply_backend()
        tnr = self._config.generic['nr_time_steps']
        en_range = self._sample.energy_range
        energies_dos = np.array([0.5 * i * en_range / tnr - en_range / 2.
                                 for i in range(tnr * 2)])
        en_limit = self._config.DC_conductivity['energy_limits']
        qe_indices = np.where((energies_dos >= en_limit[0]) &
                              (energies_dos <= en_limit[1]))[0]
        beta_re, mu_re = self._get_beta_mu_re()
        time_step = self._get_time_step()
        bessel_series = self._get_bessel_series(time_step)
        indptr, indices, hop, dx, dy = self._sample.build_ham_dxy()
        num_sample = self._dist_sample()
        self._echo_time_step_fs(time_step)
        if self._checkpoint:
            from ..checkpoint import dc_checkpointed
            path = self._checkpoint["path"] + ".dc"
            if self.size > 1:
                path = f"{path}.rank{self.rank}"
            corr_dos, corr_dc = dc_checkpointed(
                bessel_series, indptr, indices, hop, self._sample.rescale, dx, dy,
                self._config.generic['seed'], self._config.generic['nr_time_steps'],
                num_sample, time_step, energies_dos, qe_indices, self.rank,
                self._config.generic['wfn_check_steps'], self._config.generic['wfn_check_thr'],
                path, states_per_part=self._checkpoint.get("states_per_part"),
                on_checkpoint=self._checkpoint.get("on_dc_checkpoint"))
        else:
            corr_dos, corr_dc = f2py.tbpm_dccond(
                bessel_series, beta_re, mu_re, indptr, indices, hop,
                self._sample.rescale, dx, dy,
                self._config.generic['seed'], self._config.generic['nr_time_steps'], num_sample,
                time_step, energies_dos, qe_indices,
                self._output['corr_DOS'], self._output['corr_DC'], self.rank,
                self._config.generic['wfn_check_steps'], self._config.generic['wfn_check_thr'])
        corr_dos = self.all_average(corr_dos)
        corr_dc = self.all_average(corr_dc)
        self._save_data(corr_dos, self._output["corr_DOS"])
        self._save_data(corr_dc, self._output["corr_DC"])
        return corr_dos, corr_dc

    # names used by the TBPM literature / drop-in documentation
    calc_corr_ac = calc_corr_ac_cond
    calc_corr_dc = calc_corr_dc_cond

    def calc_psi_t(self, psi_0: np.ndarray, time_log: np.ndarray, dt_scale: float = 1.0,
                   save_data: bool = False) -> np.ndarray:
        """Propagate psi_0 and return psi at the steps in time_log,
        (num_time, num_orb) complex128 (solver.py:543-600)."""
        if self.size != 1:
            raise RuntimeError("Using more than 1 mpi process is not allowed"
                               " for wave function propagation")
        self._apply_backend()
        psi_0 = np.array(psi_0, dtype=np.complex128)
        psi_0 /= np.linalg.norm(psi_0)
        time_log = np.array(sorted(set(int(t) for t in time_log)), dtype=np.int64)
        for it in time_log:
            if it not in range(self._config.generic['nr_time_steps'] + 1):
                raise ValueError(f"time {it} out of range")
        time_step = self._get_time_step() * dt_scale
        bessel_series = self._get_bessel_series(time_step)
        ham_csr = self._sample.build_ham_csr()
        self._echo_time_step_fs(time_step)
        psi_t = f2py.tbpm_psi_t(
            bessel_series, ham_csr.indptr, ham_csr.indices, ham_csr.data, psi_0, time_log,
            self._config.generic['nr_time_steps'], self._config.generic['wfn_check_steps'],
            self._config.generic['wfn_check_thr'])
        psi_t = psi_t.T
        if save_data:
            self._save_data(psi_t, self._output['psi_t'])
        return psi_t

    def calc_corr_dyn_pol(self) -> np.ndarray:
        """Dynamical polarisation correlation, (n_q_points, nr_time_steps)
        float64 (solver.py:354-390)."""
        self._apply_backend()
        time_step = 0.5 * self._get_time_step()
        bessel_series = self._get_bessel_series(time_step)
        beta_re, mu_re = self._get_beta_mu_re()
        indptr, indices, hop, dx, dy = self._sample.build_ham_dxy()
        orb_pos = self._sample.orb_pos
        site_x, site_y, site_z = orb_pos[:, 0], orb_pos[:, 1], orb_pos[:, 2]
        num_sample = self._dist_sample()
        self._echo_time_step_fs(time_step)
        corr_dyn_pol = f2py.tbpm_dyn_pol(
            bessel_series, beta_re, mu_re, indptr, indices, hop, self._sample.rescale,
            dx, dy, site_x, site_y, site_z, self._config.generic['seed'],
            self._config.generic['nr_time_steps'], num_sample,
            self._config.generic['nr_Fermi_fft_steps'],
            self._config.generic['Fermi_cheb_precision'],
            self._config.dyn_pol['q_points'], self._output['corr_dyn_pol'], self.rank,
            self._config.generic['wfn_check_steps'], self._config.generic['wfn_check_thr'])
        corr_dyn_pol = self.all_average(corr_dyn_pol)
        self._save_data(corr_dyn_pol, self._output["corr_dyn_pol"])
        return corr_dyn_pol

    def calc_hall_mu(self) -> np.ndarray:
        """Kubo-Bastin moments mu_mn, (n_kernel, n_kernel) complex128
        (solver.py:443-472)."""
        self._apply_backend()
        indptr, indices, hop, dx, dy = self._sample.build_ham_dxy()
        num_sample = self._dist_sample()
        mu_mn = f2py.tbpm_kbdc(
            self._config.generic['seed'], indptr, indices, hop, self._sample.rescale, dx, dy,
            num_sample, self._config.dckb['n_kernel'], self._config.dckb['direction'],
            self.rank)
        mu_mn = self.all_average(mu_mn)
        self._save_data(mu_mn, self._output['hall_mu'])
        return mu_mn

    def calc_quasi_eigenstates(self, save_data: bool = False) -> np.ndarray:
        """Quasi-eigenstates, (n_energies, n_orbitals) float64
        (solver.py:474-507)."""
        self._apply_backend()
        time_step = self._get_time_step()
        bessel_series = self._get_bessel_series(time_step)
        num_sample = self._dist_sample()
        self._echo_time_step_fs(time_step)
        ham_csr = self._sample.build_ham_csr()
        states = f2py.tbpm_eigenstates(
            bessel_series, ham_csr.indptr, ham_csr.indices, ham_csr.data,
            self._config.generic['seed'], self._config.generic['nr_time_steps'], num_sample,
            time_step, self._config.quasi_eigenstates['energies'], self.rank,
            self._config.generic['wfn_check_steps'], self._config.generic['wfn_check_thr'])
        states = self.all_average(states)
        if save_data:
            self._save_data(states, self._output['qe'])
        return states

    def calc_ldos_haydock(self) -> Tuple[np.ndarray, np.ndarray]:
        """LDOS by the Haydock recursion: (energies, ldos), both
        (2*nr_time_steps+1,) float64 (solver.py:509-541)."""
        if self.size != 1:
            raise RuntimeError("Using more than 1 mpi process is not allowed"
                               " for ldos_haydock")
        self._apply_backend()
        ham_csr = self._sample.build_ham_csr()
        energies, ldos = f2py.ldos_haydock(
            self._config.LDOS['site_indices'], self._config.LDOS['delta'],
            self._sample.energy_range, ham_csr.indptr, ham_csr.indices, ham_csr.data,
            self._sample.rescale, self._config.generic['seed'],
            self._config.LDOS['recursion_depth'], self._config.generic['nr_time_steps'],
            self._config.generic['nr_random_samples'], self._output['ldos_haydock'])
        self._save_data(ldos, self._output["ldos_haydock"])
        return energies, ldos

"""Analyzer: correlation functions -> DOS, AC/DC/Hall conductivity,
dynamical polarisation and dielectric function.

Same API and formulas as tbplas/tbpm/analysis.py (window functions :20-51,
calc_dos :89-143, calc_ac_cond :161-243, calc_dyn_pol :245-308, _get_vq
:310-329, calc_epsilon :331-354, calc_epsilon_q0 :356-373, calc_dc_cond
:375-458, calc_diff_coeff :460-511, calc_hall_cond :513-575), with the
O(nr_time_steps^2) Python loops of the reference replaced by numpy array
expressions and the Kubo-Bastin trace (analysis.f90 cond_from_trace) run on
the GPU.  Results agree with the reference to floating-point summation order.
"""

from math import cos, exp, pi
from typing import Callable, Tuple

import numpy as np
from scipy.integrate import cumulative_trapezoid
from scipy.signal import hilbert

from ..base import EPSILON0
from ..parallel import MPIEnv
from .config import Config

__all__ = ["window_hanning", "window_exp", "window_exp_ten", "Analyzer"]


def window_hanning(i: int, tnr: int) -> float:
    """Hanning window 0.5*(1 + cos(pi*i/tnr))."""
    return 0.5 * (1 + cos(pi * i / tnr))


def window_exp(i: int, tnr: int) -> float:
    """Exponential window exp(-2*(i/tnr)^2)."""
    return exp(-2. * (i / tnr)**2)


def window_exp_ten(i: int, tnr: int) -> float:
    """Exponential window 10^(-2*(i/tnr)^2)."""
    power = -2 * (1. * i / tnr)**2
    return 10.**power


def _window_values(window: Callable, start: int, stop: int, tnr: int) -> np.ndarray:
    return np.array([window(i, tnr) for i in range(start, stop)], dtype=float)


def _trig_sums(ctx, w, a, b, x, dt, per_output: bool, phase_kdt: bool):
    """tbpm_trig_sums: (sum_k w a cos, sum_k w b sin) for every row of a / b
    (leading axes) and every x; either coefficient array may be None."""
    from .. import _native as nat
    w = np.ascontiguousarray(w, dtype=float)
    x = np.ascontiguousarray(x, dtype=float)
    ref = a if a is not None else b
    lead = ref.shape[:-2] if per_output else ref.shape[:-1]
    n_rows = int(np.prod(lead)) if len(lead) else 1
    shape = tuple(lead) + (x.size,)
    a = None if a is None else np.ascontiguousarray(a, dtype=float)
    b = None if b is None else np.ascontiguousarray(b, dtype=float)
    oc = np.zeros(shape) if a is not None else None
    os_ = np.zeros(shape) if b is not None else None
    ctx.call("tbpm_trig_sums", nat.ptr(w), w.size, nat.ptr(a), nat.ptr(b), n_rows, nat.ptr(x),
             x.size, float(dt), 1 if per_output else 0, 1 if phase_kdt else 0, nat.ptr(oc),
             nat.ptr(os_))
    return oc, os_


class Analyzer(MPIEnv):
    """Post-processing of TBPM correlation functions (see tbplas.tbpm.Analyzer).

    The trigonometric sums of calc_ac_cond, calc_dyn_pol, calc_dc_cond and
    calc_diff_coeff run on the GPU (tbpm_trig_sums, tbpm_trig_cumtrapz) when
    `backend` is "gpu", or "auto" and a GPU is visible; backend "host" (or
    "auto" without a GPU, e.g. post-processing saved correlations on a
    workstation) evaluates the same formulas with numpy.
    """

    def __init__(self, sample, config: Config, dimension: int = 3,
                 enable_mpi: bool = False, echo_details: bool = False,
                 backend: str = "auto") -> None:
        super().__init__(enable_mpi=enable_mpi, echo_details=echo_details)
        self._sample = sample
        self._config = config
        self._config.check_params()
        if dimension not in (2, 3):
            raise ValueError(f"Unsupported dimension: {dimension}")
        self._dimension = dimension
        if backend not in ("auto", "gpu", "host"):
            raise ValueError(f"Unsupported backend: {backend}")
        self._backend = backend
        self._dev = None

    def _device(self):
        """The library context the sums run on, or None for numpy."""
        if self._backend == "host":
            return None
        if self._dev is None:
            from .. import _native as nat
            try:
                self._dev = nat.get_context()
            except Exception:
                if self._backend == "gpu":
                    raise
                self._backend = "host"
                return None
        return self._dev

    def _energies(self) -> np.ndarray:
        tnr = self._config.generic['nr_time_steps']
        en_range = self._sample.energy_range
        return np.array([0.5 * i * en_range / tnr - en_range / 2. for i in range(tnr * 2)],
                        dtype=float)

    def calc_dos(self, corr_dos: np.ndarray,
                 window: Callable = window_hanning) -> Tuple[np.ndarray, np.ndarray]:
        """DOS from the DOS correlation function (analysis.py:89-143).

        :return: (energies, dos), both (2*nr_time_steps,) float64
        """
        tnr = self._config.generic['nr_time_steps']
        en_range = self._sample.energy_range
        en_step = 0.5 * en_range / tnr
        energies = self._energies()
        dos = np.zeros(tnr * 2, dtype=float)
        if self.is_master:
            c = np.asarray(corr_dos, dtype=complex).reshape(-1)
            w = _window_values(window, 0, tnr, tnr)
            neg = np.empty(tnr * 2, dtype=complex)
            neg[tnr - 1] = c[0]
            neg[2 * tnr - 1] = w[tnr - 1] * c[tnr]
            neg[tnr:2 * tnr - 1] = w[:tnr - 1] * c[1:tnr]
            neg[tnr - 2::-1] = w[:tnr - 1] * np.conj(c[1:tnr])
            fft = np.abs(np.fft.ifft(neg))
            dos[tnr:] = fft[:tnr]
            dos[:tnr] = fft[tnr:]
            dos = dos / (np.sum(dos) * en_step)
            if self._config.generic['correct_spin']:
                dos = 2. * dos
        self.bcast(dos)
        return energies, dos

    def calc_ldos(self, corr_ldos: np.ndarray,
                  window: Callable = window_hanning) -> Tuple[np.ndarray, np.ndarray]:
        """LDOS from the LDOS correlation function."""
        return self.calc_dos(corr_ldos, window)

    def calc_ac_cond(self, corr_ac: np.ndarray,
                     window: Callable = window_exp) -> Tuple[np.ndarray, np.ndarray]:
        """AC conductivity from its correlation function (analysis.py:161-243).

        :return: (omegas, ac_cond): (nr_time_steps,) float64 and
            (4, nr_time_steps) complex128 (xx, xy, yx, yy)
        """
        tnr = self._config.generic['nr_time_steps']
        en_range = self._sample.energy_range
        t_step = pi / en_range
        beta = self._config.generic['beta']
        if self._dimension == 2:
            prefactor = self._sample.nr_orbitals / (self._sample.area_unit_cell *
                                                    self._sample.extended)
        else:
            prefactor = self._sample.nr_orbitals / (self._sample.volume_unit_cell *
                                                    self._sample.extended)
        omegas = np.array([i * en_range / tnr for i in range(tnr)], dtype=float)
        ac_cond = np.zeros((4, tnr), dtype=complex)
        if self.is_master:
            corr = np.asarray(corr_ac)
            w = _window_values(window, 1, tnr + 1, tnr)
            dev = self._device()
            if dev is not None:
                _, ssum = _trig_sums(dev, w, None, np.imag(corr[:, :tnr]), omegas, t_step,
                                     per_output=False, phase_kdt=False)
                acv = 2. * ssum.T  # (tnr, 4)
            else:
                k = np.arange(tnr, dtype=float)
                # S[i, k] = 2 w(k+1) sin(omega_i k dt)
                s = 2. * w[None, :] * np.sin(np.outer(omegas, k) * t_step)
                acv = s @ np.imag(corr[:, :tnr]).T  # (tnr, 4)
            with np.errstate(divide="ignore", invalid="ignore"):
                fac = prefactor * t_step * (np.exp(-beta * omegas) - 1) / omegas
            fac[omegas == 0.] = 0.
            ac_real = (acv * fac[:, None]).T
            ac_real[:, omegas == 0.] = 0.
            ac_imag = np.zeros((4, tnr), dtype=float)
            for j in range(4):
                sigma = np.zeros(2 * tnr, dtype=float)
                sigma[tnr:] = ac_real[j]
                sigma[tnr - np.arange(tnr)] = ac_real[j]
                ac_imag[j, :] = np.imag(hilbert(sigma))[tnr:2 * tnr]
            ac_cond = ac_real + 1j * ac_imag
            if self._config.generic['correct_spin']:
                ac_cond = 2. * ac_cond
        self.bcast(ac_cond)
        return omegas, ac_cond

    def _qe_window(self):
        tnr = self._config.generic['nr_time_steps']
        energies = self._energies()
        en_limit = self._config.DC_conductivity['energy_limits']
        qe_indices = np.where((energies >= en_limit[0]) & (energies <= en_limit[1]))[0]
        return tnr, energies, qe_indices

    def calc_dc_cond(self, corr_dos: np.ndarray, corr_dc: np.ndarray,
                     window_dos: Callable = window_hanning,
                     window_dc: Callable = window_exp) -> Tuple[np.ndarray, np.ndarray]:
        """Zero-temperature DC conductivity (analysis.py:375-458).

        :return: (energies, dc): (n_energies,) float64 and (2, n_energies) float64
        """
        corr_dos = np.insert(np.asarray(corr_dos), 0, 1.0)
        _, dos = self.calc_dos(corr_dos, window_dos)
        tnr, energies_dos, qe_indices = self._qe_window()
        en_range = self._sample.energy_range
        t_step = 2 * pi / en_range
        n_energies = len(qe_indices)
        energies = energies_dos[qe_indices]
        if self._dimension == 2:
            prefactor = self._sample.nr_orbitals / self._sample.area_unit_cell
        else:
            prefactor = self._sample.nr_orbitals / self._sample.volume_unit_cell
        dc = np.zeros((2, n_energies))
        if self.is_master:
            w = _window_values(window_dc, 1, tnr + 1, tnr)
            corr = np.asarray(corr_dc)[:, :n_energies, :tnr]
            dev = self._device()
            if dev is not None and n_energies > 0:
                # Re(exp(-i E k dt) c) = Re(c) cos + Im(c) sin
                csum, ssum = _trig_sums(dev, w, np.real(corr), np.imag(corr), energies, t_step,
                                        per_output=True, phase_kdt=False)
                dc_val = csum + ssum
            else:
                k = np.arange(tnr, dtype=float)
                phi = np.outer(energies, k) * t_step  # (n_en, tnr)
                c_exp = np.cos(phi) - 1j * np.sin(phi)
                vals = np.real(c_exp[None, :, :] * corr) * w[None, None, :]
                dc_val = vals.sum(axis=2)
            dc = prefactor * t_step * dos[qe_indices][None, :] * dc_val
            if self._config.generic['correct_spin']:
                dc = 2. * dc
        self.bcast(dc)
        return energies, dc

    def calc_diff_coeff(self, corr_dc: np.ndarray,
                        window_dc: Callable = window_exp) -> Tuple[np.ndarray, np.ndarray]:
        """Diffusion coefficient from the DC correlation (analysis.py:460-511).

        :return: (time, diff_coeff): (nr_time_steps,) float64 and
            (2, n_energies, nr_time_steps) float64
        """
        tnr, energies_dos, qe_indices = self._qe_window()
        en_range = self._sample.energy_range
        t_step = 2 * pi / en_range
        n_energies = len(qe_indices)
        energies = energies_dos[qe_indices]
        time = np.linspace(0, tnr - 1, tnr) * t_step
        diff_coeff = np.zeros((2, n_energies, tnr))
        if self.is_master:
            w = _window_values(window_dc, 1, tnr + 1, tnr)
            corr = np.asarray(corr_dc)[:, :n_energies, :tnr]
            dev = self._device()
            if dev is not None and n_energies > 0:
                from .. import _native as nat
                a = np.ascontiguousarray(np.real(corr))
                b = np.ascontiguousarray(np.imag(corr))
                x = np.ascontiguousarray(np.tile(energies, 2))
                spacing = np.ascontiguousarray(np.diff(time))
                out = np.zeros((2, n_energies, tnr))
                dev.call("tbpm_trig_cumtrapz", nat.ptr(w), tnr, nat.ptr(a), nat.ptr(b),
                         2 * n_energies, nat.ptr(x), float(t_step), nat.ptr(spacing),
                         nat.ptr(out))
                diff_coeff = out
            else:
                k = np.arange(tnr, dtype=float)
                phi = np.outer(energies, k) * t_step
                c_exp = np.cos(phi) - 1j * np.sin(phi)
                temp = np.real(c_exp[None, :, :] * corr) * w[None, None, :]
                diff_coeff[:, :, 1:] = cumulative_trapezoid(temp, time, axis=2)
        self.bcast(diff_coeff)
        return time, diff_coeff

    def calc_dyn_pol(self, corr_dyn_pol: np.ndarray, window: Callable = window_exp_ten
                     ) -> Tuple[np.ndarray, np.ndarray, np.ndarray]:
        """Dynamical polarisation from its correlation function (analysis.py:245-308).

        :return: (q_points (n_q, 3), omegas (nr_time_steps,), dyn_pol
            (n_q, nr_time_steps) complex128)
        """
        tnr = self._config.generic['nr_time_steps']
        en_range = self._sample.energy_range
        t_step = pi / en_range
        q_points = np.array(self._config.dyn_pol['q_points'], dtype=float)
        if self._dimension == 2:
            prefactor = 2. * self._sample.nr_orbitals / (self._sample.area_unit_cell *
                                                         self._sample.extended)
        else:
            prefactor = 2. * self._sample.nr_orbitals / (self._sample.volume_unit_cell *
                                                         self._sample.extended)
        omegas = np.array([i * en_range / tnr for i in range(tnr)], dtype=float)
        dyn_pol = np.zeros((len(q_points), tnr), dtype=complex)
        if self.is_master:
            w = _window_values(window, 1, tnr + 1, tnr)
            corr = np.asarray(corr_dyn_pol, dtype=float)[:, :tnr]
            dev = self._device()
            if dev is not None:
                csum, ssum = _trig_sums(dev, w, corr, corr, omegas, t_step, per_output=False,
                                        phase_kdt=True)
                dyn_pol = prefactor * t_step * (csum + 1j * ssum)
            else:
                k = np.arange(tnr, dtype=float)
                phi = np.outer(omegas, k * t_step)  # phi[i, k] = k*dt*omega_i
                e = np.cos(phi) + 1j * np.sin(phi)
                dyn_pol = prefactor * t_step * ((corr * w[None, :]) @ e.T)
            if self._config.generic['correct_spin']:
                dyn_pol = 2. * dyn_pol
        self.bcast(dyn_pol)
        return q_points, omegas, dyn_pol

    def _get_vq(self, q_point: np.ndarray) -> float:
        """Coulomb interaction in momentum space in eV (analysis.py:310-329)."""
        factor = self._config.dyn_pol['coulomb_constant']
        back_epsilon = self._config.dyn_pol['background_dielectric_constant']
        factor /= (EPSILON0 * back_epsilon)
        q_norm = np.linalg.norm(q_point)
        if q_norm == 0.0:
            return 0.0
        if self._dimension == 2:
            return factor * 2 * pi / q_norm
        return factor * 4 * pi / q_norm**2

    def calc_epsilon(self, dyn_pol: np.ndarray) -> np.ndarray:
        """Dielectric function 1 - V(q) P(q, omega) (analysis.py:331-354)."""
        tnr = self._config.generic['nr_time_steps']
        q_points = self._config.dyn_pol['q_points']
        epsilon = np.zeros((len(q_points), tnr), dtype=complex)
        if self.is_master:
            for i, q_point in enumerate(q_points):
                epsilon[i] = 1 - self._get_vq(q_point) * dyn_pol[i]
        self.bcast(epsilon)
        return epsilon

    def calc_epsilon_q0(self, omegas: np.ndarray, ac_cond: np.ndarray) -> np.ndarray:
        """Dielectric function at q = 0 from the AC conductivity, 3-D only
        (analysis.py:356-373)."""
        if self._dimension != 3:
            raise ValueError(f"Unsupported dimension: {self._dimension}")
        back_epsilon = self._config.dyn_pol['background_dielectric_constant']
        prefactor = 4 * pi / (back_epsilon * EPSILON0)
        return 1 + 1j * prefactor * ac_cond / omegas

    def calc_hall_cond(self, mu_mn: np.ndarray,
                       unit: str = "h_bar") -> Tuple[np.ndarray, np.ndarray]:
        """Hall conductivity from the Kubo-Bastin moments (analysis.py:513-575);
        the trace over Gamma_mn(E) mu_mn runs on the GPU.

        :return: (energies, conductivity) for config.dckb['energies']
        """
        from ..fortran import f2py
        if unit not in ("h_bar", "h"):
            raise ValueError(f"Illegal unit {unit}")
        energies = np.array(self._config.dckb['energies'])
        if self.is_master:
            prefactor = 16 * self._sample.nr_orbitals / (pi * self._sample.energy_range ** 2)
            if self._dimension == 2:
                prefactor /= self._sample.area_unit_cell
            else:
                prefactor /= self._sample.volume_unit_cell
            if unit == "h":
                prefactor *= (2 * pi)
            conductivity = f2py.cond_from_trace(
                mu_mn, self._config.dckb['energies'], self._sample.rescale,
                self._config.generic['beta'], self._config.dckb['ne_integral'],
                self._config.generic['Fermi_cheb_precision'], self.rank)
            conductivity *= prefactor
            if self._config.generic['correct_spin']:
                conductivity *= 2
        else:
            conductivity = np.zeros(len(energies), dtype=float)
        self.bcast(conductivity)
        return energies, conductivity

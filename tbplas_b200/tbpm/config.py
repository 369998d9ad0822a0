"""TBPM parameters: the reference `Config` (tbplas/tbpm/config.py) kept as is.

Same attribute dictionaries, keys, defaults (config.py:86-120), legality
check (config.py:147-166) and pickle round trip (config.py:168-185).  Options
of the GPU backend are not stored here, so `check_params` keeps rejecting
unknown keys of the reference dictionaries.
"""

import pickle

from ..base import KB

__all__ = ["Config", "read_config"]


class Config:
    """Parameters controlling TBPM calculations (see tbplas.tbpm.Config)."""

    def __init__(self) -> None:
        self.generic = {'Bessel_max': 250,
                        'Bessel_precision': 1.0e-14,
                        'beta': 1.0 / (KB * 300),
                        'mu': 0.,
                        'correct_spin': False,
                        'nr_time_steps': 1024,
                        'nr_random_samples': 1,
                        'seed': 1337,
                        'wfn_check_steps': 128,
                        'wfn_check_thr': 1.0e-9,
                        'nr_Fermi_fft_steps': 2**15,
                        'Fermi_cheb_precision': 1.0e-12}
        self.LDOS = {'site_indices': [0],
                     'wf_weights': [1.0],
                     'delta': 0.01,
                     'recursion_depth': 2000}
        self.DC_conductivity = {'energy_limits': (-0.5, 0.5)}
        self.quasi_eigenstates = {'energies': [-0.1, 0., 0.1]}
        self.dyn_pol = {'q_points': [[1., 0., 0.]],
                        'coulomb_constant': 1.0,
                        'background_dielectric_constant': 1.0}
        self.dckb = {'energies': [i * 0.01 - 0.2 for i in range(0, 41)],
                     'n_kernel': 2048,
                     'direction': 1,
                     'ne_integral': 2048}
        self._legal_params = dict()
        self.set_legal_params()

    def set_temperature(self, temperature: float = 300.0) -> None:
        """Set beta = 1/(kB*T) for temperature T in Kelvin."""
        self.generic['beta'] = 1.0 / (KB * temperature)

    def set_legal_params(self) -> None:
        self._legal_params = {
            'generic': set(self.generic.keys()),
            'LDOS': set(self.LDOS.keys()),
            'dyn_pol': set(self.dyn_pol.keys()),
            'dckb': set(self.dckb.keys())
        }

    def check_params(self) -> None:
        """Raise ValueError on keys that are not defined (config.py:147-166)."""
        for name in ('generic', 'LDOS', 'dyn_pol', 'dckb'):
            unknown = set(getattr(self, name).keys()) - self._legal_params[name]
            for key in sorted(unknown):
                raise ValueError(f"Undefined parameter {key} in config.{name}")


def read_config(filename: str) -> Config:
    """Read a Config pickled by Solver.save_config."""
    with open(filename, 'rb') as f:
        loaded = pickle.load(f)
    config = Config()
    for name in ('generic', 'LDOS', 'dyn_pol', 'DC_conductivity', 'dckb',
                 'quasi_eigenstates'):
        setattr(config, name, getattr(loaded, name))
    config.set_legal_params()
    return config

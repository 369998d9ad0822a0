"""Physical constants used on the TBPM path (values of tbplas/base/constants.py)."""

KB = 8.617333262e-5  # Boltzmann constant in eV/K
H_BAR_EV = 6.582119514e-16  # reduced Planck constant in eV*s
EPSILON0 = 0.6944615417149689  # vacuum permittivity in eV/nm/q units
NM = 1.0

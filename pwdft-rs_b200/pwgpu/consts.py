"""Physical constants and numerical floors, in the engine's native units.

Energies are eV, lengths Å, densities e/Å³.  Values follow
pwdft/pwdft-core/src/consts.rs:15-49 and functionals/mod.rs:5 of the
reference so that every derived quantity (ħ²/2m, Coulomb prefactors,
unit conversions at the UPF boundary) rounds identically.
"""

import math

HA_TO_EV = 27.211386245988
RY_TO_EV = 13.605693122994
BOHR_TO_ANG = 0.529177210903
BOHR3_TO_ANG3 = BOHR_TO_ANG * BOHR_TO_ANG * BOHR_TO_ANG
E2_COULOMB = 14.399645351950548

G2_ZERO_THRESHOLD = 1e-12
G_ZERO_THRESHOLD = 1e-12
RHO_FLOOR = 1e-30

H_SI = 6.62607015e-34
HBAR_SI = H_SI / (2.0 * math.pi)
M_E = 9.1093837015e-31
EV_PER_J = 6.241509074e18
ANG_PER_M = 1e10
# ħ²/2m in eV·Å², same evaluation order as consts.rs:49
HBAR2_OVER_2M = HBAR_SI * HBAR_SI / (2.0 * M_E) * EV_PER_J * ANG_PER_M * ANG_PER_M

"""The plain-method SCF case: Si diamond 2-atom fcc primitive cell,
a = 10.26 bohr, atoms at crystal (0,0,0) and (1/4,1/4,1/4), PZ-LDA,
ecutwfc 20 Ry (ecutrho 4x), shifted 4x4x4 Monkhorst-Pack grid reduced by
the 48 operations + time reversal to 10 k-points, 8 bands.

"Fixed occupations" is read as the reference deck reads it:
SmearingScheme::Fixed with the deck's default smearing_width of 0.05 eV
(settings.rs:230), which occupies like Fermi-Dirac at that width
(smearing.rs:99).  Mixing: plain Anderson, beta 0.7, 8 history slots.
Convergence: energy change below 1e-10 Ry and density rms below 1e-8 e/Å³
(the reference's plain Anderson stalls near 2e-9 e/Å³ where its DIIS
matrix turns singular, so the rms threshold is set above that floor).
"""

from .consts import BOHR_TO_ANG, RY_TO_EV
from .context import build_system
from .crystal import diamond_primitive
from .symmetry import SymmetryInfo, reduce_kpoints

SCF_KW = dict(n_bands=8, max_iter=120, conv_threshold=1e-8, energy_threshold=1e-10 * RY_TO_EV, mixing_beta=0.7,
              mixing_ndim=8, smearing="fixed", sigma=0.05)


def config1_system(pp, ecut_ry: float = 20.0):
    cr = diamond_primitive("Si", 10.26 * BOHR_TO_ANG)
    sym = SymmetryInfo.from_crystal(cr, 1e-5)
    kp = reduce_kpoints((4, 4, 4), "mp1976", sym, cr.lattice)
    return build_system(cr, {"Si": pp}, ecut_ry * RY_TO_EV, kp, sym)

"""Batched k-points, collinear LSDA: the 8-atom conventional cubic diamond
cells of Si (a = 10.26 bohr; n_pw 3,791 on a 40^3 grid) and C (a = 6.74
bohr; n_pw 1,045 on 25^3), ecutwfc 35 Ry, Gamma-centred 6x6x6 mesh reduced
by the 48 point operations + time reversal (20 IBZ k-points each), 24 bands,
Fermi-Dirac 0.02 Ry, PZ-LSDA.

Starting magnetisation: 0 on Si; 0.5 mu_B on C, which the reference takes
as a per-species fraction of the valence charge (settings.rs:283-285):
0.5 / 4 = 0.125, applied as the atom average (driver_spin.rs:160-167).
Mixing and convergence use the reference's ScfParams defaults
(scf/mod.rs:228-252): plain Anderson beta 0.3, 8 history slots, density rms
1e-6 e/Å^3, energy change 1e-5 eV.

The only C LDA UPF at hand carries a core correction; `nlcc=False` strips it
in memory (a labelled variant, not a different pseudopotential file).
"""

import dataclasses

from .consts import BOHR_TO_ANG, RY_TO_EV
from .context import build_system
from .crystal import diamond_supercell
from .symmetry import SymmetryInfo, reduce_kpoints

CELLS = {"Si": 10.26, "C": 6.74}  # lattice constants, bohr
START_MAG = {"Si": 0.0, "C": 0.5 / 4.0}

SCF_KW = dict(n_bands=24, max_iter=100, conv_threshold=1e-6, energy_threshold=1e-5, mixing_beta=0.3,
              mixing_ndim=8, smearing="fermi_dirac", sigma=0.02 * RY_TO_EV)


def config4_system(species: str, pp, nlcc: bool = True, ecut_ry: float = 35.0, kgrid=(6, 6, 6)):
    """(ScfSystem, starting_magnetization) of one cell of the batched-k case."""
    if not nlcc and pp.has_nlcc():
        pp = dataclasses.replace(pp, core_charge=pp.core_charge[:0])
    cr = diamond_supercell(species, CELLS[species] * BOHR_TO_ANG)
    sym = SymmetryInfo.from_crystal(cr, 1e-5)
    kp = reduce_kpoints(kgrid, "gamma", sym, cr.lattice)
    return build_system(cr, {species: pp}, ecut_ry * RY_TO_EV, kp, sym, nspin=2), START_MAG[species]

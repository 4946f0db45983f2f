"""Copy the reference's test fixtures used by the parity tests into tests/golden/.

Run once in a checkout that has the reference tree available, giving the
root of that tree (the directory holding pseudopotentials/ and data/):

    python tests/golden/make_fixtures.py <reference-root>

Copied verbatim (data files, not source):
  * pseudopotentials/nc/lda/{Si,Si_hgh,C}.upf   -> tests/golden/upf/
  * pseudopotentials/nc/lda/{Al,As,Cl,Cu,Fe,Ga,Mg,Na,O}.upf (heavy-atom pins)
                                                 -> tests/golden/upf/
  * data/csv/{vloc_g_si,beta_q_si,dij_si,rho_core_g,vgcmp_phase4}_reference.csv,
    data/csv/vgch_{beta_l,vloc}_heavy.csv,
    data/csv/vgch_sad_heavy{,_samples}.csv (SAD start densities of seven cells)
                                                 -> tests/golden/csv/
  * data/qe/c_rho_qe.bin (QE's converged C-diamond density, VGCH2BIN bundle)
                                                 -> tests/golden/qe/
  * data/qe/{cu_fcc,fe_bcc_fm,nacl,c_diamond,mgo}_scf.out (QE's converged
    bands, weights and Fermi levels) and data/csv/vgch2c_fermi_reference.csv
    (the Fermi levels the reference's bisection finds on them)
                                                 -> tests/golden/qe/, tests/golden/csv/
The SCF goldens (E_total, E_F) are constants in tests/test_oracle_pins.py
with their reference file:line.
"""

import os
import shutil
import sys

UPFS = ["Si.upf", "Si_hgh.upf", "C.upf"] + [f"{e}.upf" for e in ("Al", "As", "Cl", "Cu", "Fe", "Ga", "Mg", "Na", "O")]
CSVS = ["vloc_g_si_reference.csv", "beta_q_si_reference.csv", "dij_si_reference.csv",
        "rho_core_g_reference.csv", "vgcmp_phase4_reference.csv", "vgch_beta_l_heavy.csv", "vgch_vloc_heavy.csv",
        "vgch_sad_heavy.csv", "vgch_sad_heavy_samples.csv", "vgch2c_fermi_reference.csv"]
QE_OUTS = [f"{n}_scf.out" for n in ("cu_fcc", "fe_bcc_fm", "nacl", "c_diamond", "mgo")]


def main(ref_root: str):
    here = os.path.dirname(os.path.abspath(__file__))
    os.makedirs(os.path.join(here, "upf"), exist_ok=True)
    os.makedirs(os.path.join(here, "csv"), exist_ok=True)
    for f in UPFS:
        shutil.copyfile(os.path.join(ref_root, "pseudopotentials", "nc", "lda", f), os.path.join(here, "upf", f))
    for f in CSVS:
        shutil.copyfile(os.path.join(ref_root, "data", "csv", f), os.path.join(here, "csv", f))
    os.makedirs(os.path.join(here, "qe"), exist_ok=True)
    for f in ["c_rho_qe.bin"] + QE_OUTS:
        shutil.copyfile(os.path.join(ref_root, "data", "qe", f), os.path.join(here, "qe", f))


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_fixtures.py <reference-root>")
    main(sys.argv[1])

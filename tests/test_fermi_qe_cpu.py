"""Fermi level of the library's host occupation code (pwgpu_occupations, the
find_fermi_energy bisection of scf/smearing.rs:49-90) on QE's converged band
structures of five cells (Cu fcc, Fe bcc ferromagnetic LSDA, NaCl, C diamond,
MgO; data/qe/*_scf.out), against:

* data/csv/vgch2c_fermi_reference.csv, rows `pwdft_bracket`: the level the
  reference's bracket-and-halve search finds on the same bands (written by
  the reference's pwdft-validation fermi generator), for Fermi-Dirac,
  Gaussian and first-order Methfessel-Paxton smearing at QE's width;
* the Fermi level QE itself reports (Fermi-Dirac, QE's own smearing).

Where the level is well defined (every scheme in a metal; Fermi-Dirac and
Methfessel-Paxton across a gap, whose tails keep a small slope) it must
agree. For Gaussian smearing inside an insulator's gap the electron count
is flat to rounding, so any level in the gap is a root: the test checks
the count and that the level lies in the gap.
"""

import csv
import os
import re

import numpy as np
import pytest

from conftest import GOLDEN
from pwgpu.consts import RY_TO_EV
from pwgpu.lib import occupations

CELLS = {"Cu_FCC": ("cu_fcc_scf.out", 1, True), "Fe_BCC_FM": ("fe_bcc_fm_scf.out", 2, True),
         "NaCl": ("nacl_scf.out", 1, False), "C_diamond": ("c_diamond_scf.out", 1, False),
         "MgO": ("mgo_scf.out", 1, False)}
SCHEMES = {"fermi_dirac": "fermi_dirac", "gaussian": "gaussian", "mp1": "methfessel_paxton"}
_NUM = re.compile(r"-?\d+\.\d+")


def qe_bands(fname, nspin):
    """(eigenvalues [sets, nbnd] eV, weights [sets], n_electrons, degauss Ry,
    QE's Fermi level eV) from a QE pw.x output: the last band listing, one
    set per k-point (spin up sets then spin down for LSDA); weights are QE's
    wk of the first (Cartesian) k-point list, repeated for each spin."""
    text = open(os.path.join(GOLDEN, "qe", fname)).read()
    nel = float(re.search(r"number of electrons\s*=\s*(\S+)", text).group(1))
    degauss = float(re.search(r"width \(Ry\)=\s*(\S+)", text).group(1))
    ef_qe = float(re.search(r"the Fermi energy is\s+(\S+)\s+ev", text).group(1))
    wk = {}
    for idx, w in re.findall(r"k\(\s*(\d+)\)\s*=\s*\([^)]*\),\s*wk\s*=\s*(\S+)", text):
        wk.setdefault(int(idx), float(w))
    weights = [wk[i] for i in sorted(wk)] * nspin
    tail = text[text.rindex("End of self-consistent calculation"):]
    sets = []
    for chunk in tail.split("bands (ev):")[1:]:
        cut = min([i for i in (chunk.find(s) for s in ("occupation numbers", "k =", "the Fermi", "------"))
                   if i >= 0] + [len(chunk)])
        sets.append([float(x) for x in _NUM.findall(chunk[:cut])])
    assert len(sets) == len(weights), fname
    assert len({len(s) for s in sets}) == 1, fname
    return np.array(sets), np.array(weights), nel, degauss, ef_qe


def reference_rows():
    with open(os.path.join(GOLDEN, "csv", "vgch2c_fermi_reference.csv")) as fh:
        return {(r["system"], r["smearing"]): float(r["ef_ev"]) for r in csv.DictReader(fh)
                if r["bisection_style"] == "pwdft_bracket"}


@pytest.mark.parametrize("scheme", sorted(SCHEMES))
@pytest.mark.parametrize("cell", sorted(CELLS))
def test_fermi_level_on_qe_bands(cell, scheme):
    fname, nspin, metal = CELLS[cell]
    ev, w, nel, degauss, _ = qe_bands(fname, nspin)
    ef, occ, _ = occupations(ev, w, nel, degauss * RY_TO_EV, SCHEMES[scheme], spin_factor=1.0)
    assert abs(float(np.sum(w[:, None] * occ)) - nel) < 1e-9 * nel
    ref = reference_rows()[(cell, scheme)]
    if metal:
        # the count's slope is states per eV: the roots agree to rounding
        assert abs(ef - ref) < 1e-9, (cell, scheme, ef, ref)
    elif scheme != "gaussian":
        # Fermi-Dirac tails and the Methfessel-Paxton term keep a small slope
        # across the gap, so the root is still defined (observed <= 3e-9 eV)
        assert abs(ef - ref) < 1e-8, (cell, scheme, ef, ref)
    else:
        # Gaussian tails vanish inside the gap: any level there is a root
        n_occ = int(round(nel / 2))
        assert ev[:, n_occ - 1].max() < ef < ev[:, n_occ].min(), (cell, ef)


@pytest.mark.parametrize("cell", sorted(CELLS))
def test_fermi_dirac_level_matches_qe_report(cell):
    """QE's cells use Fermi-Dirac smearing (or report its level): the
    library's level on QE's bands is QE's printed level (4 decimals)."""
    fname, nspin, _ = CELLS[cell]
    ev, w, nel, degauss, ef_qe = qe_bands(fname, nspin)
    ef, _, _ = occupations(ev, w, nel, degauss * RY_TO_EV, "fermi_dirac", spin_factor=1.0)
    assert abs(ef - ef_qe) < 2.5e-4, (cell, ef, ef_qe)


def test_parser_reads_the_whole_listing():
    ev, w, nel, degauss, ef = qe_bands("fe_bcc_fm_scf.out", 2)
    assert ev.shape == (58, 12) and nel == 16.0 and degauss == 0.02 and ef == 26.2006
    assert ev[0, 0] == -122.5041 and ev[0, -1] == 45.4725
    assert abs(w.sum() - 2.0 * w[:29].sum()) < 1e-15

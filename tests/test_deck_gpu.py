"""A YAML deck run end to end on the device (pwgpu.deck.run_deck): the
reference's golden SCF case (tests/cpu_scf_baseline.rs:43-44: Si primitive
cell, 100 eV, 16^3 grid, Γ, 4 bands, Fermi-Dirac 0.05 eV, identity-only
symmetry; E = -213.028339 eV, E_F = 8.052064 eV, within 1e-3 eV) written as
a deck, with both output files the deck asks for."""

import os

import numpy as np
import pytest

from conftest import GOLDEN
from pwgpu.deck import run_deck
from pwgpu.output import read_bands, read_density

pytestmark = pytest.mark.gpu

DECK = """
system:
  lattice:
    - [0.0, 2.7155, 2.7155]
    - [2.7155, 0.0, 2.7155]
    - [2.7155, 2.7155, 0.0]
  atoms:
    - {symbol: Si, position: [0.0, 0.0, 0.0]}
    - {symbol: Si, position: [0.25, 0.25, 0.25]}
basis:
  ecutwfc: 100.0
  fft_grid: [16, 16, 16]
kpoints:
  type: monkhorst_pack
  grid: [1, 1, 1]
scf:
  n_bands: 4
  max_iter: 40
  mixing_beta: 0.3
  mixing_ndim: 4
  smearing: fermi_dirac
  smearing_width: 0.05
symmetry:
  enabled: false
output:
  write_density: true
"""


def test_deck_reproduces_reference_golden(tmp_path):
    path = tmp_path / "si.yaml"
    path.write_text(DECK)
    res, ev, rho, s = run_deck(str(path), os.path.join(GOLDEN, "upf"), output_dir=str(tmp_path / "out"))
    assert res["converged"] == 1
    assert abs(res["total_energy"] - (-213.028339)) < 1e-3
    assert abs(res["fermi_energy"] - 8.052064) < 1e-3
    b = read_bands(str(tmp_path / "out" / "bands.txt"))
    assert np.max(np.abs(b["eigenvalues"] - ev)) < 1e-9 and b["fermi_energy"] == pytest.approx(res["fermi_energy"])
    ck = read_density(str(tmp_path / "out" / "density.npz"))
    assert np.array_equal(ck["rho_r"].ravel(), rho)

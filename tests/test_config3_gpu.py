"""The mixed-precision SCF case against the FP64 oracle.

1. The 8-atom cell of the same physics (Si cubic conventional cell with
   seeded ±0.05 bohr displacements, Si.upf, 30 Ry, Γ, 20 bands, Gaussian
   0.01 Ry, Anderson beta 0.4 + Kerker): the full SCF of the dense oracle is
   the committed fixture (tests/golden/make_config3_fixtures.py, converged to
   drho 1e-9 e/Å³).  The plain FP64 form, converged as tightly, is held to
   1e-8 Ha in the total energy and 1e-7 Ha in the eigenvalues, with real
   (Gamma-packed) and complex bands; the mixed form, run at the benchmark's
   own thresholds (drho 1e-6, FP64 switch at 1e-6), to 1e-6 Ha per atom and
   1e-5 Ha.
2. The benchmarked 64-atom cell itself, too large for the dense loop: the
   device solves it (FP64, drho 1e-8), then runs one transplanted FP64
   iteration from the converged density, whose input density, bands,
   eigenvalues, output density and energies are all read back.  The oracle
   rebuilds V_eff from that input density, applies its FFT-form H to the
   bands, and builds occupations, the output density and the total energy
   from its own Rayleigh quotients (oracle.fixed_point_check).  The device's
   eigenvalues must equal the oracle's Rayleigh quotients and its energy the
   oracle's, at the plain form's bars; the residuals must vanish, the two
   output densities agree and the map be at its fixed point.  The mixed
   solve, at the benchmark's own thresholds, is held to the mixed bars
   against that oracle-verified state.
"""

import json
import os

import numpy as np
import pytest

from conftest import GOLDEN
from oracle import pwdft_oracle as O
from pwgpu.config3 import FP64_SWITCH, SCF_KW, SI8_SCF_KW, SOLVER_KW, config3_si8_system, config3_system
from pwgpu.lib import PRECISION_FP64, PRECISION_MIXED, PwGpu

pytestmark = pytest.mark.gpu

HA = O.HA_TO_EV
E_TOL_FP64 = 1e-8 * HA      # total energy, plain form
EV_TOL_FP64 = 1e-7 * HA     # eigenvalues, plain form
E_TOL_MIXED_ATOM = 1e-6 * HA
EV_TOL_MIXED = 1e-5 * HA


def fixture():
    with open(os.path.join(GOLDEN, "config3_si8_oracle.json")) as f:
        return json.load(f)


def run(s, kw, precision, gamma_complex=False, **extra):
    kw = dict(kw)
    nb = kw.pop("n_bands")
    with PwGpu(s, gamma_complex=gamma_complex) as dev:
        res, ev, rho, _ = dev.scf_run(s.rho_init_r, nb, precision=precision, fp64_switch=FP64_SWITCH, **kw, **extra)
        psi = dev.get_bands(nb)
    return res, ev, rho, psi


# the library's default eigen-residual schedule and the one the Si64 bench uses
SCHEDULES = {"default": {}, "si64": SOLVER_KW}


@pytest.mark.parametrize("schedule", sorted(SCHEDULES))
@pytest.mark.parametrize("gamma_complex", [False, True])
def test_si8_fp64_matches_oracle(si_pp, gamma_complex, schedule):
    ref = fixture()
    s = config3_si8_system(si_pp)
    assert (s.n_pw, list(s.dims)) == (ref["n_pw"], ref["dims"])
    res, ev, _, _ = run(s, SI8_SCF_KW, PRECISION_FP64, gamma_complex, diag_tol=1e-10, **SCHEDULES[schedule])
    assert res["converged"] == 1
    assert abs(res["total_energy"] - ref["total_energy"]) < E_TOL_FP64
    assert abs(res["harris_foulkes_energy"] - ref["harris_foulkes_energy"]) < E_TOL_FP64
    assert abs(res["fermi_energy"] - ref["fermi_energy"]) < EV_TOL_FP64
    assert np.max(np.abs(ev[0] - np.array(ref["eigenvalues"][0]))) < EV_TOL_FP64
    for k in ("e_kinetic", "e_local", "e_nonlocal"):
        assert abs(res[k] - ref["components"][k]) < 1e-6, k


@pytest.mark.parametrize("schedule", sorted(SCHEDULES))
def test_si8_mixed_matches_oracle(si_pp, schedule):
    ref = fixture()
    s = config3_si8_system(si_pp)
    kw = dict(SCF_KW, n_bands=SI8_SCF_KW["n_bands"], **SCHEDULES[schedule])
    res, ev, _, _ = run(s, kw, PRECISION_MIXED)
    assert res["converged"] == 1
    assert abs(res["total_energy"] - ref["total_energy"]) / ref["n_atoms"] < E_TOL_MIXED_ATOM
    assert np.max(np.abs(ev[0] - np.array(ref["eigenvalues"][0]))) < EV_TOL_MIXED


def test_schedule_reaches_the_eigensolver(si_pp):
    """pwgpu_scf_params.diag_tol_per_drho / diag_tol_cap change the work of
    the solve (band applications) but not its converged energy."""
    s = config3_si8_system(si_pp)
    kw = dict(SCF_KW, n_bands=SI8_SCF_KW["n_bands"])
    r0, _, _, _ = run(s, kw, PRECISION_FP64)
    r1, _, _, _ = run(s, dict(kw, diag_tol_per_drho=20.0, diag_tol_cap=0.2), PRECISION_FP64)
    assert r0["converged"] == 1 and r1["converged"] == 1
    assert r0["h_applications"] != r1["h_applications"]
    assert abs(r0["total_energy"] - r1["total_energy"]) / 8 < E_TOL_MIXED_ATOM


def _si64_state(s):
    """The benchmarked cell solved on the device, then one transplanted FP64
    iteration from its converged density (pwgpu_scf_iter1_from_rho_g): the
    iteration's input density is known exactly, its bands are eigenvectors
    of H[rho_in], its energies are built on its output density."""
    nb = SCF_KW["n_bands"]
    kw = dict(SCF_KW, conv_threshold=1e-8, energy_threshold=1e-8, max_iter=120)
    kw.pop("n_bands")
    with PwGpu(s) as dev:
        res, ev, rho, _ = dev.scf_run(s.rho_init_r, nb, precision=PRECISION_FP64, **kw)
        r1, ev1, rho_out1, _, rho_in1 = dev.scf_iter1_from_rho_g(
            O.density_r_to_g(rho, s.dims), nb, smearing=SCF_KW["smearing"], sigma=SCF_KW["sigma"], diag_tol=1e-9,
            diag_max_iter=300)
        psi = dev.get_bands(nb)
    return res, ev, r1, ev1, rho_out1, rho_in1, psi


def test_si64_fp64_iteration_is_the_oracles(si_pp):
    s = config3_system(si_pp)
    res, _, r1, ev1, rho_out1, rho_in1, psi = _si64_state(s)
    assert res["converged"] == 1
    chk = O.fixed_point_check(s, rho_in1, psi, SCF_KW["smearing"], SCF_KW["sigma"])
    assert np.max(np.abs(chk["rayleigh"] - ev1[0])) < EV_TOL_FP64
    assert np.max(chk["residual"]) < 1e-6
    assert abs(chk["fermi_energy"] - r1["fermi_energy"]) < EV_TOL_FP64
    assert np.max(np.abs(chk["rho_out"] - rho_out1)) < 1e-10 * np.max(np.abs(rho_out1))
    assert abs(chk["total_energy"] - r1["total_energy"]) < E_TOL_FP64
    # at the converged density the iteration maps rho to itself (the fixed point of both)
    assert chk["drho_in_out"] < 1e-7


def test_si64_mixed_form_against_oracle(si_pp):
    """The benchmarked mixed solve (its own thresholds and eigen-residual
    schedule) against the oracle's energy and eigenvalues at the FP64 fixed
    point."""
    s = config3_system(si_pp)
    _, _, r1, ev1, _, rho_in1, psi = _si64_state(s)
    chk = O.fixed_point_check(s, rho_in1, psi, SCF_KW["smearing"], SCF_KW["sigma"])
    assert abs(chk["total_energy"] - r1["total_energy"]) < E_TOL_FP64
    kw = dict(SCF_KW, **SOLVER_KW)
    nb = kw.pop("n_bands")
    with PwGpu(s) as dev:
        rm, evm, _, _ = dev.scf_run(s.rho_init_r, nb, precision=PRECISION_MIXED, fp64_switch=FP64_SWITCH, **kw)
    assert rm["converged"] == 1
    n_at = len(s.crystal.atoms)
    assert abs(rm["total_energy"] - chk["total_energy"]) / n_at < E_TOL_MIXED_ATOM
    assert np.max(np.abs(evm[0] - chk["rayleigh"])) < EV_TOL_MIXED

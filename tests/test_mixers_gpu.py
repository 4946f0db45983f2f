"""Density mixers on the device (Mixer kinds of mixing/mod.rs:186-287:
Anderson, modified Broyden, Periodic Pulay; each with and without Kerker)
against the oracle restatements: step by step through pwgpu_mix, and whole
SCF runs (unpolarised and CCMX spin) through pwgpu_scf_run.

Tolerances: mixing steps 1e-12 relative (same arithmetic, different
summation order); converged SCF energies 1e-5 eV (first order in drho at
drho < 1e-8), Harris-Foulkes 1e-6 eV, eigenvalues 1e-5 eV."""

import numpy as np
import pytest

from conftest import rng
from oracle import pwdft_oracle as O
from pwgpu.context import build_system
from pwgpu.crystal import diamond_primitive, gamma_only
from pwgpu.lib import PwGpu

pytestmark = pytest.mark.gpu

MIXERS = [(m, k) for m in ("anderson", "broyden", "periodic_pulay") for k in (False, True)]


def si2(pp, nspin=1):
    return build_system(diamond_primitive("Si", 5.431), {"Si": pp}, 100.0, gamma_only(), fft_grid=(16, 16, 16),
                        nspin=nspin)


def kerker_weights(s):
    q2 = O.auto_q_tf_squared(s.n_electrons, s.omega)
    return np.where(s.g_squared < O.G2_ZERO_THRESHOLD, 0.0, s.g_squared / (s.g_squared + q2))


@pytest.mark.parametrize("mixer,kerker", MIXERS)
def test_mix_steps_match_oracle(si_pp, mixer, kerker):
    """12 steps through a depth-4 history (wrap-around), period 3."""
    s = si2(si_pp)
    g = rng(23)
    n = s.n_grid
    ref = O.make_mixer(mixer, 0.35, 4, s.dims, kerker_weights(s) if kerker else None, period=3)
    rho = s.rho_init_r.copy()
    with PwGpu(s) as dev:
        dev.mix_reset()
        for step in range(12):
            out = rho + 1e-3 * (g.standard_normal(n) + np.cos(np.arange(n) * (0.013 * (step + 1))))
            want = ref.mix(rho, out)
            got = dev.mix(rho, out, 0.35, 4, kerker=kerker, mixer=mixer, period=3)
            assert np.max(np.abs(got - want)) < 1e-12 * np.max(np.abs(want)), step
            rho = want


@pytest.mark.parametrize("mixer,kerker", [("broyden", True), ("periodic_pulay", False), ("periodic_pulay", True)])
def test_scf_with_mixer_matches_oracle(si_pp, mixer, kerker):
    s = si2(si_pp)
    kw = dict(n_bands=6, max_iter=150, conv_threshold=1e-8, energy_threshold=1e-7, mixing_beta=0.3,
              smearing="fermi_dirac", sigma=0.05, kerker=kerker, mixer=mixer, mixing_period=3)
    ref = O.run_scf_unpolarized(s, **kw)
    with PwGpu(s) as dev:
        res, ev, rho, _ = dev.scf_run(s.rho_init_r, **kw)
    assert res["converged"] == 1
    assert abs(res["total_energy"] - ref.total_energy) < 1e-5
    assert abs(res["harris_foulkes_energy"] - ref.harris_foulkes_energy) < 1e-6
    assert np.max(np.abs(ev - np.array(ref.eigenvalues))) < 1e-5


def test_spin_scf_periodic_pulay_matches_oracle(si_pp):
    s = si2(si_pp, nspin=2)
    kw = dict(n_bands=6, max_iter=200, conv_threshold=1e-8, energy_threshold=1e-7, mixing_beta=0.3,
              smearing="fermi_dirac", sigma=0.05, mixer="periodic_pulay", mixing_period=3,
              starting_magnetization=0.2)
    ref = O.run_scf_spin(s, **kw)
    with PwGpu(s) as dev:
        res, ev, rho, _ = dev.scf_run(s.rho_init_r, **kw)
    assert res["converged"] == 1
    assert abs(res["total_energy"] - ref.total_energy) < 1e-5
    assert abs(res["harris_foulkes_energy"] - ref.harris_foulkes_energy) < 1e-6
    assert abs(res["magnetization"] - ref.magnetization) < 1e-6

"""Occupations through the library's host code (pwgpu_occupations; no GPU
work): the reference's smearing unit tests (scf/smearing.rs:268-461) as
known answers, and E_F, occupations and TS against the oracle's
restatement (smearing.rs:38-252) on seeded spectra of several (spin, k)
sets, every scheme."""

import numpy as np
import pytest

from conftest import rng
from oracle import pwdft_oracle as O
from pwgpu.lib import occupations

SCHEMES = ("fermi_dirac", "gaussian", "methfessel_paxton", "cold")


def occ_at(scheme, e, ef, sigma, spin_factor):
    _, occ, _ = occupations([[e]], [1.0], 0.0, sigma, scheme, spin_factor, fermi_energy=ef)
    return occ[0, 0]


def test_fermi_dirac_occupation_by_spin_factor():
    for sf, full in ((2.0, 2.0), (1.0, 1.0)):
        assert abs(occ_at("fermi_dirac", -1.0, 0.0, 0.01, sf) - full) < 1e-10
        assert abs(occ_at("fermi_dirac", 1.0, 0.0, 0.01, sf)) < 1e-10
        assert abs(occ_at("fermi_dirac", 0.0, 0.0, 0.01, sf) - full / 2) < 1e-10


def test_all_schemes_spin_factor_consistency():
    for scheme in SCHEMES:
        for e in (-0.5, -0.1, 0.0, 0.1, 0.5):
            f1 = occ_at(scheme, e, 0.0, 0.1, 1.0)
            f2 = occ_at(scheme, e, 0.0, 0.1, 2.0)
            assert abs(f2 - 2.0 * f1) <= 1e-12 * max(abs(f2), 1e-300) or f2 == 2.0 * f1, (scheme, e)


def test_fermi_energy_nspin1_nspin2():
    evs = [-2.0, -1.0, 1.0, 2.0]
    ef1, occ1, _ = occupations([evs], [1.0], 4.0, 0.05, "fermi_dirac", 2.0)
    assert -1.5 < ef1 < 1.5
    assert abs(occ1.sum() - 4.0) < 4.0 * 1e-6
    ef2, occ2, _ = occupations([evs, evs], [1.0, 1.0], 4.0, 0.05, "fermi_dirac", 1.0)
    assert -1.5 < ef2 < 1.5
    assert abs(occ2.sum() - 4.0) < 4.0 * 1e-6
    assert abs(ef1 - ef2) < 1e-10


def test_entropy():
    for scheme in SCHEMES:
        _, _, ts = occupations([[-1.0, 0.0, 1.0]], [1.0], 0.0, 0.0, scheme, 2.0, fermi_energy=0.0)
        assert abs(ts) < 1e-15, scheme
    evs = [-0.5, -0.1, 0.1, 0.5]
    _, _, ts = occupations([evs], [1.0], 4.0, 0.1, "fermi_dirac", 2.0)
    assert ts > 0.0
    _, _, ts1 = occupations([evs], [1.0], 0.0, 0.1, "fermi_dirac", 2.0, fermi_energy=0.0)
    _, _, ts2 = occupations([evs, evs], [1.0, 1.0], 0.0, 0.1, "fermi_dirac", 1.0, fermi_energy=0.0)
    assert abs(ts1 - ts2) < 1e-10


def test_zero_temperature_all_schemes():
    for scheme in SCHEMES:
        for sf in (2.0, 1.0):
            assert occ_at(scheme, -1.0, 0.0, 0.0, sf) == sf
            assert occ_at(scheme, 1.0, 0.0, 0.0, sf) == 0.0
            assert occ_at(scheme, 0.0, 0.0, 0.0, sf) == sf / 2


@pytest.mark.parametrize("scheme", SCHEMES + ("fixed",))
@pytest.mark.parametrize("spin_factor", (2.0, 1.0))
def test_matches_oracle(scheme, spin_factor):
    g = rng(31)
    n_sets, nb = 6, 12
    ev = np.sort(g.uniform(-8.0, 6.0, (n_sets, nb)), axis=1)
    w = g.uniform(0.5, 2.0, n_sets)
    w /= w.sum()
    n_el = 9.0 * spin_factor
    sigma = 0.12
    ef, occ, ts = occupations(ev, w, n_el, sigma, scheme, spin_factor)
    ef_o = O.find_fermi_energy(list(ev), list(w), n_el, sigma, scheme, spin_factor)
    assert abs(ef - ef_o) < 1e-12
    occ_o = spin_factor * O.occupation01(scheme, ev, ef_o, sigma)
    assert np.max(np.abs(occ - occ_o)) < 1e-13
    assert abs(ts - O.entropy_ts(list(ev), list(w), ef_o, sigma, scheme, spin_factor)) < 1e-12
    assert abs(float(np.sum(w[:, None] * occ)) - n_el) < 1e-9


def test_rejects_bad_arguments():
    from pwgpu.lib import PwGpuError
    with pytest.raises(PwGpuError):
        occupations([[0.0]], [1.0], 1.0, -0.1, "fermi_dirac", 2.0)
    with pytest.raises(PwGpuError):
        occupations([[0.0]], [1.0], 1.0, 0.1, "fermi_dirac", 0.0)

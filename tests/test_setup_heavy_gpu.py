"""Context setup on the device for heavier atoms (the reference's LDA UPFs
of Cu, Fe, Ga, As, Na, Cl: Z_val 7-19, s/p/d projectors, NLCC on all but
Na) against the host construction at a general k-point. Compared are the
projector matrix B (NonlocalPotential::new, nonlocal.rs:190-382), V_loc(G),
the core density and the start density (potentials.rs:18-115,
initial_density.rs:64-166), each within 1e-12 of its maximum."""

import numpy as np
import pytest

from conftest import upf_path
from pwgpu.context import build_system
from pwgpu.crystal import Atom, Crystal, KPoint, Lattice, fcc_primitive
from pwgpu.lib import PwGpu
from pwgpu.symmetry import SymmetryInfo
from pwgpu.upf import load_upf

pytestmark = pytest.mark.gpu


def bcc_primitive(a):
    return Lattice(a / 2 * np.array([-1.0, 1.0, 1.0]), a / 2 * np.array([1.0, -1.0, 1.0]),
                   a / 2 * np.array([1.0, 1.0, -1.0]))


CASES = {
    "cu_fcc": (lambda: Crystal(fcc_primitive(3.61), [Atom("Cu", (0.0, 0.0, 0.0))]), ("Cu",)),
    "fe_bcc": (lambda: Crystal(bcc_primitive(2.87), [Atom("Fe", (0.0, 0.0, 0.0))]), ("Fe",)),
    "gaas_zincblende": (lambda: Crystal(fcc_primitive(5.65), [Atom("Ga", (0.0, 0.0, 0.0)),
                                                              Atom("As", (0.25, 0.25, 0.25))]), ("Ga", "As")),
    "nacl_rocksalt": (lambda: Crystal(fcc_primitive(5.64), [Atom("Na", (0.0, 0.0, 0.0)),
                                                            Atom("Cl", (0.5, 0.5, 0.5))]), ("Na", "Cl")),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_device_setup_matches_host_heavy(name):
    make, elements = CASES[name]
    pps = {e: load_upf(upf_path(f"{e}.upf")) for e in elements}
    kp = [KPoint(np.array([0.13, -0.21, 0.07]), 1.0)]
    host = build_system(make(), pps, 250.0, kp, SymmetryInfo.identity_only())
    dev_sys = build_system(make(), pps, 250.0, kp, SymmetryInfo.identity_only(), projectors_on_device=True,
                           local_on_device=True)
    with PwGpu(dev_sys) as dev:
        b = dev.projectors(0)
        v, rc = dev.local_potential()
        rho0 = dev.initial_density()
    bh = host.projectors[0].b
    assert b.shape == bh.shape
    assert np.max(np.abs(b - bh)) < 1e-12 * np.max(np.abs(bh))
    assert np.max(np.abs(v - host.v_local_g)) < 1e-12 * np.max(np.abs(host.v_local_g))
    assert np.max(np.abs(rc - host.rho_core_r)) < 1e-12 * np.max(np.abs(host.rho_core_r))
    assert np.max(np.abs(rho0 - host.rho_init_r)) < 1e-12 * np.max(host.rho_init_r)
    assert abs(rho0.sum() * host.omega / host.n_grid - host.n_electrons) < 1e-10 * host.n_electrons

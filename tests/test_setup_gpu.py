"""Context setup on the device from the UPF radial data against the host
construction: projector matrices (NonlocalPotential::new, nonlocal.rs:
190-382) column by column, the local potential V_loc(G), the NLCC core
density and the start density (ScfContext::new, potentials.rs:18-115;
generate_initial_density, initial_density.rs:64-166) point by point, all
within 1e-12 of their maximum (Simpson summation order, libm rounding and
the order of the structure-factor sums differ); SCF results identical to
the host-built form, and Gamma handles still recognised as Gamma-real."""

import numpy as np
import pytest

from pwgpu.context import build_system
from pwgpu.crystal import KPoint, diamond_primitive, diamond_supercell, gamma_only
from pwgpu.lib import PwGpu
from pwgpu.symmetry import SymmetryInfo

pytestmark = pytest.mark.gpu


def cases(si_pp, c_pp):
    c8 = diamond_supercell("C", 3.5667, displacement_ang=0.03, rng=np.random.default_rng(3))
    return {
        "si2_k": lambda dev: build_system(diamond_primitive("Si", 5.431), {"Si": si_pp}, 150.0,
                                          [KPoint(np.array([0.11, -0.23, 0.31]), 0.5),
                                           KPoint(np.array([0.0, 0.2, 0.1]), 0.5)],
                                          SymmetryInfo.identity_only(), projectors_on_device=dev),
        "c8_gamma": lambda dev: build_system(c8, {"C": c_pp}, 250.0, gamma_only(), SymmetryInfo.identity_only(),
                                             projectors_on_device=dev),
    }


@pytest.mark.parametrize("name", ["si2_k", "c8_gamma"])
def test_device_projectors_match_host(si_pp, c_pp, name):
    build = cases(si_pp, c_pp)[name]
    host = build(False)
    dev_sys = build(True)
    with PwGpu(dev_sys) as dev:
        for ik in range(len(host.kpoints)):
            b_dev = dev.projectors(ik)
            b_host = host.projectors[ik].b
            assert b_dev.shape == b_host.shape
            assert np.max(np.abs(b_dev - b_host)) < 1e-13 * np.max(np.abs(b_host))


def test_scf_with_device_projectors_matches_host(si_pp):
    kw = dict(n_bands=6, max_iter=80, conv_threshold=1e-8, energy_threshold=1e-7, mixing_beta=0.3, sigma=0.05)
    out = []
    for on_device in (False, True):
        s = build_system(diamond_primitive("Si", 5.431), {"Si": si_pp}, 100.0, gamma_only(), fft_grid=(16, 16, 16),
                         projectors_on_device=on_device)
        with PwGpu(s) as dev:
            res, ev, _, _ = dev.scf_run(s.rho_init_r, **kw)
            # Gamma-real bands (the real path ran): eigenvectors come back Gamma-real
            e2, psi, _, _ = dev.eigensolve(4, tol=1e-8, max_iter=200)
        m = s.basis.miller
        where = {tuple(x): i for i, x in enumerate(m.tolist())}
        neg = np.array([where[tuple((-x).tolist())] for x in m])
        assert np.max(np.abs(psi[neg] - psi.conj())) < 1e-12
        out.append((res["total_energy"], ev))
    assert abs(out[0][0] - out[1][0]) < 1e-9
    assert np.max(np.abs(out[0][1] - out[1][1])) < 1e-9


def local_cases(si_pp, si_hgh_pp, c_pp):
    c8 = diamond_supercell("C", 3.5667, displacement_ang=0.03, rng=np.random.default_rng(3))
    return {
        # NLCC and PP_RHOATOM
        "c8_gamma": lambda dev: build_system(c8, {"C": c_pp}, 250.0, gamma_only(), SymmetryInfo.identity_only(),
                                             local_on_device=dev),
        # no NLCC, no PP_RHOATOM: the Gaussian start density
        "si2_hgh": lambda dev: build_system(diamond_primitive("Si", 5.431), {"Si": si_hgh_pp}, 150.0, gamma_only(),
                                            local_on_device=dev),
        "si2_k": lambda dev: build_system(diamond_primitive("Si", 5.431), {"Si": si_pp}, 120.0,
                                          [KPoint(np.array([0.11, -0.23, 0.31]), 1.0)], SymmetryInfo.identity_only(),
                                          local_on_device=dev, projectors_on_device=dev),
    }


@pytest.mark.parametrize("name", ["c8_gamma", "si2_hgh", "si2_k"])
def test_device_local_potential_matches_host(si_pp, si_hgh_pp, c_pp, name):
    build = local_cases(si_pp, si_hgh_pp, c_pp)[name]
    host = build(False)
    dev_sys = build(True)
    assert dev_sys.v_local_g is None and dev_sys.rho_init_r is None
    with PwGpu(dev_sys) as dev:
        v, rc = dev.local_potential()
        rho0 = dev.initial_density()
    assert np.max(np.abs(v - host.v_local_g)) < 1e-12 * np.max(np.abs(host.v_local_g))
    if host.rho_core_r.size:
        assert np.max(np.abs(rc - host.rho_core_r)) < 1e-12 * np.max(np.abs(host.rho_core_r))
    else:
        assert not np.any(rc)
    assert np.max(np.abs(rho0 - host.rho_init_r)) < 1e-12 * np.max(host.rho_init_r)
    assert abs(rho0.sum() * host.omega / host.n_grid - host.n_electrons) < 1e-10 * host.n_electrons


def test_scf_with_device_local_potential_matches_host(c_pp):
    kw = dict(n_bands=20, max_iter=80, conv_threshold=1e-7, energy_threshold=1e-6, mixing_beta=0.3, sigma=0.05)
    c8 = diamond_supercell("C", 3.5667, displacement_ang=0.03, rng=np.random.default_rng(3))
    out = []
    for on_device in (False, True):
        s = build_system(c8, {"C": c_pp}, 250.0, gamma_only(), SymmetryInfo.identity_only(),
                         local_on_device=on_device, projectors_on_device=on_device)
        with PwGpu(s) as dev:
            rho0 = dev.initial_density() if on_device else s.rho_init_r
            res, ev, _, _ = dev.scf_run(rho0, **kw)
        out.append((res, ev))
    assert out[0][0]["converged"] == 1 and out[1][0]["converged"] == 1
    # same inputs to 1e-12: the two loops take the same path
    assert abs(out[0][0]["total_energy"] - out[1][0]["total_energy"]) < 1e-7
    assert np.max(np.abs(out[0][1] - out[1][1])) < 1e-7


def test_initial_density_needs_device_local_build(si_pp):
    s = build_system(diamond_primitive("Si", 5.431), {"Si": si_pp}, 100.0, gamma_only(), fft_grid=(16, 16, 16))
    with PwGpu(s) as dev:
        with pytest.raises(Exception):
            dev.initial_density()

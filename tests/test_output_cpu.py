"""Density checkpoint and band table (the reference's write_density /
write_bands flags, settings.rs:435-454) written and read back, and the
oracle's transplanted iteration (scf/transplant.rs:114-376) against the
first iteration of its own SCF loop from the same density.  CPU only."""

import numpy as np
import pytest

from oracle import pwdft_oracle as O
from pwgpu.context import build_system
from pwgpu.crystal import KPoint, diamond_primitive, gamma_only
from pwgpu.output import read_bands, read_density, restart_rho_g, write_bands, write_density


def si2(pp, nspin=1, kpts=None):
    return build_system(diamond_primitive("Si", 5.431), {"Si": pp}, 100.0, kpts or gamma_only(),
                        fft_grid=(16, 16, 16), nspin=nspin)


@pytest.mark.parametrize("nspin", [1, 2])
def test_density_checkpoint_round_trip(tmp_path, si_pp, nspin):
    s = si2(si_pp, nspin)
    n = s.n_grid
    rho = np.concatenate([s.rho_init_r * 0.6, s.rho_init_r * 0.4]) if nspin == 2 else s.rho_init_r
    path = str(tmp_path / "rho.npz")
    write_density(path, s, rho)
    ck = read_density(path)
    assert ck["dims"] == s.dims and ck["nspin"] == nspin
    assert np.array_equal(ck["rho_r"].ravel(), rho)
    total = rho.reshape(nspin, n).sum(axis=0)
    ref_g = O.density_r_to_g(total, s.dims)
    assert np.max(np.abs(ck["rho_g_fft"] - ref_g)) < 1e-15 * n
    assert np.array_equal(ck["rho_g_basis"], ck["rho_g_fft"][s.g_to_fft])
    assert np.array_equal(ck["miller"], s.basis.miller)
    # back to real space through the transplant's inverse transform
    back = O.ifft3(restart_rho_g(s, ck), s.dims).real
    assert np.max(np.abs(back - total)) < 1e-12 * np.max(total)
    other = build_system(diamond_primitive("Si", 5.431), {"Si": si_pp}, 100.0, gamma_only(), fft_grid=(18, 18, 18))
    with pytest.raises(ValueError):
        restart_rho_g(other, ck)


def test_band_table_round_trip(tmp_path, si_pp):
    kp = [KPoint(np.array([0.1, 0.0, -0.2]), 0.25), KPoint(np.array([0.0, 0.3, 0.1]), 0.75)]
    s = si2(si_pp, 2, kp)
    ev = np.sort(np.random.default_rng(1).normal(size=(4, 6)), axis=1) * 5.0
    path = str(tmp_path / "bands.txt")
    write_bands(path, s, ev, 3.25)
    b = read_bands(path)
    assert b["fermi_energy"] == 3.25
    assert np.max(np.abs(b["eigenvalues"] - ev)) < 1e-10
    assert list(b["spin"]) == [0, 0, 1, 1] and list(b["ik"]) == [0, 1, 0, 1]
    assert np.allclose(b["weight"], [0.25, 0.75, 0.25, 0.75])
    assert np.allclose(b["k"][1], [0.0, 0.3, 0.1])
    with pytest.raises(ValueError):
        write_bands(path, s, ev[:3], 0.0)


def test_oracle_transplant_is_the_first_scf_iteration(si_pp):
    """The transplanted iteration replicates iteration 0 of the driver from
    the same density (transplant.rs:21-28)."""
    s = si2(si_pp)
    kw = dict(smearing="fermi_dirac", sigma=0.05)
    it1 = O.run_scf_iter1_from_rho_g(s, 4, O.density_r_to_g(s.rho_init_r, s.dims), **kw)
    full = O.run_scf_unpolarized(s, 4, max_iter=40, conv_threshold=1e-6, energy_threshold=1e-5, mixing_beta=0.3,
                                 mixing_ndim=4, **kw)
    _, e0, d0 = full.history[0]
    assert abs(it1.total_energy - e0) < 1e-9
    assert abs(it1.delta_rho - d0) < 1e-12
    assert np.max(np.abs(it1.rho_r_in - s.rho_init_r)) < 1e-12 * np.max(s.rho_init_r)
    # from the converged density the iteration stays there
    again = O.run_scf_iter1_from_rho_g(s, 4, O.density_r_to_g(full.rho_r, s.dims), **kw)
    assert again.delta_rho < 1e-5
    assert abs(again.total_energy - full.total_energy) < 1e-4
    with pytest.raises(ValueError):
        O.run_scf_iter1_from_rho_g(s, 4, np.zeros(10, dtype=complex), **kw)


def test_qe_density_bundle_reads_and_integrates():
    """The reference's QE C-diamond density (data/qe/c_rho_qe.bin) parses
    and rho(G = 0) Omega = 8 electrons to 0.01 on its 20^3 grid
    (tests/vgch_transplant_c.rs:188-237)."""
    import os
    from conftest import GOLDEN
    from pwgpu.crystal import fcc_primitive
    from pwgpu.output import qe_rho_g_on_grid, read_qe_density_bundle
    b = read_qe_density_bundle(os.path.join(GOLDEN, "qe", "c_rho_qe.bin"))
    assert b["nspin"] == 1 and b["miller"].shape == (1687, 3)
    g = qe_rho_g_on_grid(b, (20, 20, 20))
    assert abs(g[0].real * fcc_primitive(3.567).volume() - 8.0) < 0.01


def test_qe_density_bundle_rejects_bad_files(tmp_path):
    from pwgpu.output import read_qe_density_bundle
    p = tmp_path / "bad.bin"
    p.write_bytes(b"NOTABUNDLE" + bytes(100))
    with pytest.raises(ValueError):
        read_qe_density_bundle(str(p))

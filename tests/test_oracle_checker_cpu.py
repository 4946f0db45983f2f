"""The oracle's fixed-point checker (oracle.fixed_point_check, used by the
GPU tests and the bench on cells too large for the dense loop) against the
dense oracle loop itself, on CPU: an 8-atom displaced Si cell at 10 Ry, Γ,
converged by run_scf_unpolarized to drho 1e-10; the checker, given that
run's output density and the dense eigenvectors of H at it, reproduces the
loop's total energy, Fermi level and eigenvalues, and finds residuals at
the eigensolver's rounding and an output density equal to its input."""

import numpy as np

from oracle import pwdft_oracle as O
from pwgpu.config3 import SI8_SCF_KW, config3_si8_system


def test_fixed_point_check_reproduces_dense_loop(si_pp):
    s = config3_si8_system(si_pp, ecut_ry=10.0)
    kw = dict(SI8_SCF_KW, conv_threshold=1e-10, energy_threshold=1e-10)
    nb = kw.pop("n_bands")
    r = O.run_scf_unpolarized(s, nb, smearing=kw.pop("smearing"), sigma=kw.pop("sigma"), **kw)
    rho = r.rho_r
    dims = s.dims
    rho_g = O.density_r_to_g(rho, dims)
    _, vxc = O.lda_xc(O.add_core(rho, s.rho_core_r))
    veff = s.v_local_g + O.hartree(rho_g, s.g_squared) + O.density_r_to_g(vxc, dims)
    p = s.projectors[0]
    h = O.dense_hamiltonian(s.basis.miller, s.kinetic[0], veff, dims, p.b, p.d_dense())
    w, v = O.lowest_eigenpairs(h, nb)
    chk = O.fixed_point_check(s, rho, v, SI8_SCF_KW["smearing"], SI8_SCF_KW["sigma"])
    assert np.max(np.abs(chk["rayleigh"] - w)) < 1e-9
    assert np.max(chk["residual"]) < 1e-8
    assert chk["drho_in_out"] < 1e-9
    assert abs(chk["fermi_energy"] - r.fermi_energy) < 1e-7
    assert abs(chk["total_energy"] - r.total_energy) < 1e-7
    assert np.max(np.abs(chk["rayleigh"] - np.asarray(r.eigenvalues[0]))) < 1e-7

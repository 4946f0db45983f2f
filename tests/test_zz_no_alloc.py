"""The allocation-free local H|psi> entry point.

pwgpu_apply_h_local_noalloc serves callers that cannot call cudaMalloc (a
host framework whose memory manager owns the device memory, or a serving
loop that cannot take cudaMalloc's device-wide synchronisation); its FFT
intermediates live in a fixed 32 MiB array inside the library.  Here it is
called through the C-ABI twice in a row and each result is compared with
the allocating entry point pwgpu_apply_h_device on a system without
projectors (so both compute the same local operator), at the tolerances of
the other H|psi> tests: a block of 7 bands that fits one scratch chunk,
and a block of 70 bands with padded leading dimensions that needs two
chunks.  A grid whose single band needs more than the 32 MiB scratch is
refused with PWGPU_E_INVALID before anything is written.  The file sorts
last so that a run stopping at the first failure has already run every
other test; it also passes alone in a fresh process, where its first call
is the one that sets the scratch up.
"""

import ctypes as ct

import numpy as np
import pytest

from conftest import rng
from oracle import pwdft_oracle as O
from pwgpu.consts import RY_TO_EV
from pwgpu.context import Projectors, ScfSystem, build_system
from pwgpu.crystal import BasisSet, KPoint, diamond_primitive, grid_dims_for, miller_to_idx
from pwgpu.lib import PRECISION_FP64, PRECISION_MIXED, PwGpu, load_library
from pwgpu.symmetry import SymmetryInfo

pytestmark = pytest.mark.gpu


def _local_only(s):
    """The same system with the Kleinman-Bylander channels removed."""
    s.projectors = [Projectors(np.zeros((s.n_pw, 0), dtype=np.complex128), [], np.array([0], dtype=np.int32))
                    for _ in s.kpoints]
    return s


def _noalloc_fn():
    lib = load_library()
    fn = lib.pwgpu_apply_h_local_noalloc
    fn.argtypes = [ct.c_void_p, ct.c_int32, ct.c_int32, ct.c_void_p, ct.c_int64, ct.c_int32, ct.c_void_p,
                   ct.c_int64, ct.c_void_p]
    fn.restype = ct.c_int32
    return lib, fn


@pytest.mark.parametrize("precision,tol,nb,pad", [(PRECISION_FP64, 1e-12, 7, 0), (PRECISION_MIXED, 3e-6, 7, 0),
                                                  (PRECISION_FP64, 1e-12, 70, 5), (PRECISION_MIXED, 3e-6, 70, 3)])
def test_noalloc_local_apply_matches_allocating_entry_point(si_pp, precision, tol, nb, pad):
    import torch

    s = build_system(diamond_primitive("Si", 5.431), {"Si": si_pp}, 150.0,
                     [KPoint(np.array([0.1, -0.2, 0.15]), 1.0)], SymmetryInfo.identity_only())
    rho_g = O.density_r_to_g(s.rho_init_r, s.dims)
    _, vxc = O.lda_xc(O.add_core(s.rho_init_r, s.rho_core_r))
    veff = s.v_local_g + O.hartree(rho_g, s.g_squared) + O.density_r_to_g(vxc, s.dims)
    s = _local_only(s)
    lib, fn = _noalloc_fn()
    g = rng(17)
    n = s.n_pw
    ldpsi, ldh = n + pad, n + 2 * pad  # padded columns: row b = band b, first n entries used
    psi = np.zeros((nb, ldpsi), dtype=np.complex128)
    psi[:, :n] = g.standard_normal((nb, n)) + 1j * g.standard_normal((nb, n))
    with PwGpu(s, precision=precision) as dev:
        dev.set_veff_g(veff)
        d_psi = torch.from_numpy(psi).cuda()
        d_ref = torch.empty((nb, ldh), dtype=torch.complex128, device="cuda")
        dev.apply_h_device(d_psi.data_ptr(), ldpsi, nb, d_ref.data_ptr(), ldh)
        torch.cuda.synchronize()
        ref = d_ref.cpu().numpy()[:, :n]
        for _ in range(2):
            d_out = torch.full((nb, ldh), complex(float("nan"), float("nan")), dtype=torch.complex128, device="cuda")
            rc = fn(dev.h, 0, 0, ct.c_void_p(d_psi.data_ptr()), ldpsi, nb, ct.c_void_p(d_out.data_ptr()), ldh, None)
            assert rc == 0, lib.pwgpu_last_error()
            torch.cuda.synchronize()
            got = d_out.cpu().numpy()
            out = got[:, :n]
            err = np.max(np.abs(out - ref)) / np.max(np.abs(ref))
            assert err < tol, f"no-alloc vs allocating entry point: rel err {err:.3e}"
            if pad:  # the padding of each output column is left as it was
                assert np.all(np.isnan(got[:, n:].real))


def test_noalloc_refuses_grid_larger_than_scratch():
    """Si2 at 1300 Ry (144^3 grid, 71 compact x-planes): one FP64 band needs
    more than 32 MiB of intermediates; the call fails with PWGPU_E_INVALID
    before any launch, so the output keeps its contents."""
    import torch

    cr = diamond_primitive("Si", 5.431)
    basis = BasisSet(cr.lattice, 1300.0 * RY_TO_EV)
    dims = grid_dims_for(basis, 4)
    m = np.abs(basis.miller).max(axis=0)
    xp, yp = 2 * int(m[0]) + 1, 2 * int(m[1]) + 1
    assert 16 * xp * dims[2] * (yp + dims[1]) > 32 << 20
    n = int(np.prod(dims))
    k = KPoint(np.array([0.1, -0.2, 0.15]), 1.0)
    g_to_fft = miller_to_idx(dims, *(basis.miller[:, i].astype(np.int64) for i in range(3)))
    s = ScfSystem(cr, basis, dims, g_to_fft, [k], [basis.kinetic(k.k)],
                  [Projectors(np.zeros((len(basis), 0), dtype=np.complex128), [], np.array([0], dtype=np.int32))],
                  np.zeros(n, dtype=np.complex128), np.zeros(n), np.zeros(0), 8.0, cr.lattice.volume(), 0.0,
                  SymmetryInfo.identity_only(), np.zeros(0))
    lib, fn = _noalloc_fn()
    with PwGpu(s, precision=PRECISION_FP64) as dev:
        dev.set_veff_g(np.zeros(n, dtype=np.complex128))
        d_psi = torch.ones((1, s.n_pw), dtype=torch.complex128, device="cuda")
        d_out = torch.full_like(d_psi, 7.0)
        rc = fn(dev.h, 0, 0, ct.c_void_p(d_psi.data_ptr()), s.n_pw, 1, ct.c_void_p(d_out.data_ptr()), s.n_pw, None)
        torch.cuda.synchronize()
        assert rc == -1
        assert b"32 MiB" in lib.pwgpu_last_error()
        assert torch.all(d_out == 7.0)

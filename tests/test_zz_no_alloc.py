"""The allocation-free local H|psi> entry point.

pwgpu_apply_h_local_noalloc serves callers that cannot call cudaMalloc (a
host framework whose memory manager owns the device memory, or a serving
loop that cannot take cudaMalloc's device-wide synchronisation); its FFT
intermediates live in a fixed 32 MiB array inside the library.  Here it is
called through the C-ABI twice in a row and each result is compared with
the allocating entry point pwgpu_apply_h_device on a system without
projectors (so both compute the same local operator), at the tolerances of
the other H|psi> tests.  The file sorts last so that a run stopping at the
first failure has already run every other test; it also passes alone in a
fresh process, where its first call is the one that sets the scratch up.
"""

import ctypes as ct

import numpy as np
import pytest

from conftest import rng
from oracle import pwdft_oracle as O
from pwgpu.context import Projectors, build_system
from pwgpu.crystal import KPoint, diamond_primitive
from pwgpu.lib import PRECISION_FP64, PRECISION_MIXED, PwGpu, load_library
from pwgpu.symmetry import SymmetryInfo

pytestmark = pytest.mark.gpu


def _local_only(s):
    """The same system with the Kleinman-Bylander channels removed."""
    s.projectors = [Projectors(np.zeros((s.n_pw, 0), dtype=np.complex128), [], np.array([0], dtype=np.int32))
                    for _ in s.kpoints]
    return s


@pytest.mark.parametrize("precision,tol", [(PRECISION_FP64, 1e-12), (PRECISION_MIXED, 3e-6)])
def test_noalloc_local_apply_matches_allocating_entry_point(si_pp, precision, tol):
    import torch

    s = build_system(diamond_primitive("Si", 5.431), {"Si": si_pp}, 150.0,
                     [KPoint(np.array([0.1, -0.2, 0.15]), 1.0)], SymmetryInfo.identity_only())
    rho_g = O.density_r_to_g(s.rho_init_r, s.dims)
    _, vxc = O.lda_xc(O.add_core(s.rho_init_r, s.rho_core_r))
    veff = s.v_local_g + O.hartree(rho_g, s.g_squared) + O.density_r_to_g(vxc, s.dims)
    s = _local_only(s)
    lib = load_library()
    fn = lib.pwgpu_apply_h_local_noalloc
    fn.argtypes = [ct.c_void_p, ct.c_int32, ct.c_int32, ct.c_void_p, ct.c_int64, ct.c_int32, ct.c_void_p,
                   ct.c_int64, ct.c_void_p]
    fn.restype = ct.c_int32
    g = rng(17)
    nb = 7
    psi = g.standard_normal((nb, s.n_pw)) + 1j * g.standard_normal((nb, s.n_pw))  # row b = band b
    with PwGpu(s, precision=precision) as dev:
        dev.set_veff_g(veff)
        d_psi = torch.from_numpy(psi).cuda()
        d_ref = torch.empty_like(d_psi)
        dev.apply_h_device(d_psi.data_ptr(), s.n_pw, nb, d_ref.data_ptr(), s.n_pw)
        torch.cuda.synchronize()
        ref = d_ref.cpu().numpy()
        for _ in range(2):
            d_out = torch.full_like(d_psi, complex(float("nan"), float("nan")))
            rc = fn(dev.h, 0, 0, ct.c_void_p(d_psi.data_ptr()), s.n_pw, nb, ct.c_void_p(d_out.data_ptr()), s.n_pw,
                    None)
            assert rc == 0, lib.pwgpu_last_error()
            torch.cuda.synchronize()
            out = d_out.cpu().numpy()
            err = np.max(np.abs(out - ref)) / np.max(np.abs(ref))
            assert err < tol, f"no-alloc vs allocating entry point: rel err {err:.3e}"

"""ctypes binding of libpwgpu.so (include/pwgpu.h).

`PwGpu(system)` uploads an ScfSystem (pwgpu.context) and exposes the C-ABI
entry points with numpy arrays.  Loading fails loudly when the shared
library is missing: there is no CPU fallback in the product path.
"""

from __future__ import annotations

import ctypes as ct
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libpwgpu.so")

PWGPU_OK = 0
PRECISION_FP64 = 0
PRECISION_MIXED = 1

ERROR_NAMES = {
    -1: "PWGPU_E_INVALID", -2: "PWGPU_E_CUDA", -3: "PWGPU_E_OOM", -4: "PWGPU_E_NOT_CONVERGED",
    -5: "PWGPU_E_TIMEOUT", -6: "PWGPU_E_NOT_IMPLEMENTED", -7: "PWGPU_E_STATE", -8: "PWGPU_E_PARSE",
}
PWGPU_E_PARSE = -8

# pwgpu_upf_get_array selectors (PWGPU_UPF_*)
UPF_R, UPF_RAB, UPF_LOCAL, UPF_BETA, UPF_DIJ, UPF_RHOATOM, UPF_NLCC = range(7)


class PwGpuError(RuntimeError):
    """A pwgpu entry point returned a negative status (PwdftError analogue)."""

    def __init__(self, code, msg):
        super().__init__(f"{ERROR_NAMES.get(code, code)}: {msg}")
        self.code = code


_i32p = ct.POINTER(ct.c_int32)
_f64p = ct.POINTER(ct.c_double)


class PwgpuSystem(ct.Structure):
    _fields_ = [
        ("dims", ct.c_int32 * 3),
        ("n_pw", ct.c_int32),
        ("miller", _i32p),
        ("n_k", ct.c_int32),
        ("k_weights", _f64p),
        ("kinetic", _f64p),
        ("n_ch", ct.c_int32),
        ("proj_b", _f64p),
        ("n_atoms", ct.c_int32),
        ("atom_ch_start", _i32p),
        ("d_blocks", _f64p),
        ("v_local_g", _f64p),
        ("g_squared", _f64p),
        ("rho_core_r", _f64p),
        ("n_sym", ct.c_int32),
        ("sym_src", _i32p),
        ("sym_arg", _f64p),
        ("n_electrons", ct.c_double),
        ("omega", ct.c_double),
        ("e_ewald", ct.c_double),
        ("nspin", ct.c_int32),
        ("g_cart", _f64p),
        ("k_cart", _f64p),
        ("atom_tau", _f64p),
        ("atom_species", _i32p),
        ("n_species", ct.c_int32),
        ("species_mesh", _i32p),
        ("radial_r", _f64p),
        ("radial_rab", _f64p),
        ("species_nbeta", _i32p),
        ("beta_l", _i32p),
        ("beta_r", _f64p),
        ("recip", _f64p), ("species_zval", _f64p), ("vloc_r", _f64p), ("core_r", _f64p),
        ("rho_atom_r", _f64p), ("species_flags", _i32p), ("gaussian_sigma", ct.c_double),
    ]


class PwgpuOptions(ct.Structure):
    _fields_ = [("device", ct.c_int32), ("precision", ct.c_int32), ("lanes", ct.c_int32), ("gamma_complex", ct.c_int32)]


SMEARING = {"fermi_dirac": 0, "gaussian": 1, "methfessel_paxton": 2, "cold": 3, "fixed": 4}


class PwgpuScfParams(ct.Structure):
    _fields_ = [
        ("n_bands", ct.c_int32), ("max_iter", ct.c_int32), ("conv_threshold", ct.c_double),
        ("energy_threshold", ct.c_double), ("mixing_beta", ct.c_double), ("mixing_ndim", ct.c_int32),
        ("mixing_mode", ct.c_int32), ("kerker_q_tf", ct.c_double), ("smearing", ct.c_int32),
        ("smearing_sigma", ct.c_double), ("diag_tol", ct.c_double), ("diag_max_iter", ct.c_int32),
        ("diag_extra_bands", ct.c_int32), ("precision", ct.c_int32), ("fp64_switch", ct.c_double),
        ("verbose", ct.c_int32), ("starting_magnetization", ct.c_double), ("fixed_magnetization", ct.c_int32),
        ("tot_magnetization", ct.c_double), ("mixing_period", ct.c_int32), ("diag_tol_per_drho", ct.c_double),
        ("diag_tol_cap", ct.c_double),
    ]


class PwgpuScfResult(ct.Structure):
    _fields_ = [
        ("total_energy", ct.c_double), ("harris_foulkes_energy", ct.c_double), ("free_energy", ct.c_double),
        ("energy_sigma0", ct.c_double), ("entropy_ts", ct.c_double), ("fermi_energy", ct.c_double),
        ("final_delta", ct.c_double), ("e_band", ct.c_double), ("e_hartree", ct.c_double), ("e_xc", ct.c_double),
        ("e_vxc", ct.c_double), ("e_ewald", ct.c_double), ("n_iterations", ct.c_int32), ("converged", ct.c_int32),
        ("nspin", ct.c_int32), ("magnetization", ct.c_double), ("h_applications", ct.c_int64),
        ("max_residual", ct.c_double), ("e_kinetic", ct.c_double), ("e_local", ct.c_double),
        ("e_nonlocal", ct.c_double),
    ]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


class PwgpuServerOptions(ct.Structure):
    _fields_ = [("device", ct.c_int32), ("workers", ct.c_int32), ("precision", ct.c_int32),
                ("lanes_per_job", ct.c_int32), ("hbm_budget_bytes", ct.c_int64)]


class PwgpuJobInfo(ct.Structure):
    _fields_ = [("state", ct.c_int32), ("status", ct.c_int32), ("queue_s", ct.c_double), ("run_s", ct.c_double),
                ("footprint_bytes", ct.c_int64)]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


class PwgpuServerStats(ct.Structure):
    _fields_ = [(name, ct.c_int64) for name in ("submitted", "queued", "running", "done", "failed", "bytes_in_use",
                                                "peak_bytes", "budget_bytes")]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


class PwgpuUpfInfo(ct.Structure):
    _fields_ = [("element", ct.c_char * 8), ("z_valence", ct.c_double), ("l_max", ct.c_int32),
                ("n_proj", ct.c_int32), ("mesh", ct.c_int32), ("has_nlcc", ct.c_int32), ("has_rho_atom", ct.c_int32)]


class PwgpuDeckSettings(ct.Structure):
    _fields_ = [("lattice", ct.c_double * 9), ("n_atoms", ct.c_int32), ("ecutwfc", ct.c_double),
                ("ecutrho_ratio", ct.c_int32), ("fft_grid", ct.c_int32 * 3), ("kpoints_type", ct.c_int32),
                ("mp_grid", ct.c_int32 * 3), ("mp_shift", ct.c_int32 * 3), ("n_path", ct.c_int32),
                ("band_npoints", ct.c_int32), ("max_iter", ct.c_int32), ("conv_threshold", ct.c_double),
                ("energy_threshold", ct.c_double), ("n_bands", ct.c_int32), ("eigensolver", ct.c_int32),
                ("wfrx_subspace", ct.c_int32), ("mixing_beta", ct.c_double), ("mixing_ndim", ct.c_int32),
                ("mixing_mode", ct.c_int32), ("pulay_period", ct.c_int32), ("adaptive_beta", ct.c_int32),
                ("smearing", ct.c_int32), ("smearing_width", ct.c_double), ("spin_polarized", ct.c_int32),
                ("n_starting_magnetization", ct.c_int32), ("has_tot_magnetization", ct.c_int32),
                ("tot_magnetization", ct.c_double), ("occupations", ct.c_int32), ("functional", ct.c_int32),
                ("symmetry_enabled", ct.c_int32), ("time_reversal", ct.c_int32), ("symmetry_tolerance", ct.c_double),
                ("verbosity", ct.c_int32), ("write_density", ct.c_int32), ("write_bands", ct.c_int32),
                ("gaussian_sigma", ct.c_double)]


MIXERS = {"anderson": 0, "broyden": 2, "periodic_pulay": 4}


def mixing_mode(mixer: str = "anderson", kerker: bool = False) -> int:
    """pwgpu mixing_mode code of a MixingMode (mixer kind + Kerker flag)."""
    return MIXERS[mixer] + (1 if kerker else 0)


def scf_params(n_bands: int, max_iter: int = 100, conv_threshold: float = 1e-6, energy_threshold: float = 1e-5,
               mixing_beta: float = 0.3, mixing_ndim: int = 8, kerker: bool = False, q_tf: float = 0.0,
               smearing: str = "fermi_dirac", sigma: float = 0.01, diag_tol: float = 1e-8, diag_max_iter: int = 60,
               diag_extra_bands: int = -1, precision: int = 0, fp64_switch: float = 1e-6, verbose: bool = False,
               starting_magnetization: float = 0.0, tot_magnetization=None, mixer: str = "anderson",
               mixing_period: int = 3, diag_tol_per_drho: float = 0.0, diag_tol_cap: float = 0.0) -> "PwgpuScfParams":
    """The pwgpu_scf_params POD (ScfParams fields, reference defaults; the eigen-residual
    schedule of the SCF steps at 0 selects 3 eV per e/Å^3 of delta rho, capped at 3e-2 eV)."""
    return PwgpuScfParams(n_bands, max_iter, conv_threshold, energy_threshold, mixing_beta, mixing_ndim,
                          mixing_mode(mixer, kerker), q_tf, SMEARING[smearing], sigma, diag_tol, diag_max_iter,
                          diag_extra_bands, precision, fp64_switch, 1 if verbose else 0, starting_magnetization,
                          0 if tot_magnetization is None else 1,
                          0.0 if tot_magnetization is None else tot_magnetization, mixing_period,
                          diag_tol_per_drho, diag_tol_cap)


_lib = None


def load_library(path: str = LIB_PATH):
    """Load libpwgpu.so; raises OSError if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise OSError(f"libpwgpu.so not found at {path}; build it with `python -m pwgpu.build`")
    lib = ct.CDLL(path)
    vp = ct.c_void_p
    lib.pwgpu_last_error.restype = ct.c_char_p
    lib.pwgpu_version.restype = ct.c_char_p
    lib.pwgpu_create.argtypes = [ct.POINTER(PwgpuSystem), ct.POINTER(PwgpuOptions), ct.POINTER(vp)]
    lib.pwgpu_destroy.argtypes = [vp]
    lib.pwgpu_set_veff_g.argtypes = [vp, ct.c_int32, _f64p]
    lib.pwgpu_apply_h.argtypes = [vp, ct.c_int32, ct.c_int32, _f64p, ct.c_int32, _f64p]
    lib.pwgpu_apply_h_device.argtypes = [vp, ct.c_int32, ct.c_int32, vp, ct.c_int64, ct.c_int32, vp, ct.c_int64, vp]
    lib.pwgpu_set_precision.argtypes = [vp, ct.c_int32]
    lib.pwgpu_profile_apply_h.argtypes = [vp, ct.c_int32, ct.c_int32, vp, ct.c_int64, ct.c_int32, vp, ct.c_int64,
                                          _f64p, _i32p]
    lib.pwgpu_get_dims.argtypes = [vp, _i32p, ct.POINTER(ct.c_int64), _i32p]
    lib.pwgpu_scf_run.argtypes = [vp, ct.POINTER(PwgpuScfParams), _f64p, ct.POINTER(PwgpuScfResult), _f64p, _f64p,
                                  _f64p]
    lib.pwgpu_eigensolve.argtypes = [vp, ct.c_int32, ct.c_int32, ct.c_int32, ct.c_double, ct.c_int32, _f64p, _f64p,
                                     _f64p, _i32p, _f64p]
    lib.pwgpu_get_bands.argtypes = [vp, ct.c_int32, ct.c_int32, ct.c_int32, _f64p]
    lib.pwgpu_apply_h_packed.argtypes = [vp, ct.c_int32, _f64p, ct.c_int32, _f64p]
    lib.pwgpu_dense_eigh.argtypes = [ct.c_int32, ct.c_int32, ct.c_int32, _f64p, _f64p, _f64p, _i32p, _f64p]
    lib.pwgpu_dense_cholesky_inverse.argtypes = [ct.c_int32, ct.c_int32, _f64p, _f64p, _f64p, _i32p, _i32p, _f64p]
    lib.pwgpu_density.argtypes = [vp, ct.c_int32, _f64p, _f64p, _f64p]
    lib.pwgpu_symmetrize.argtypes = [vp, _f64p]
    lib.pwgpu_potentials.argtypes = [vp, _f64p, _f64p, _f64p]
    lib.pwgpu_mix.argtypes = [vp, ct.c_int32, ct.c_int32, _f64p, _f64p, _f64p, ct.c_double, ct.c_int32, ct.c_int32,
                              ct.c_double]
    lib.pwgpu_mix_reset.argtypes = [vp]
    lib.pwgpu_get_projectors.argtypes = [vp, ct.c_int32, _f64p]
    lib.pwgpu_initial_density.argtypes = [vp, _f64p]
    lib.pwgpu_get_local_potential.argtypes = [vp, _f64p, _f64p]
    lib.pwgpu_small_geneig.argtypes = [ct.c_int32, ct.c_int32, ct.c_int32, _f64p, _f64p, _f64p, _f64p]
    lib.pwgpu_occupations.argtypes = [ct.c_int32, ct.c_int32, _f64p, _f64p, ct.c_double, ct.c_double, ct.c_int32,
                                      ct.c_double, ct.c_int32, _f64p, _f64p, _f64p]
    lib.pwgpu_get_stream.argtypes = [vp, ct.POINTER(vp)]
    lib.pwgpu_get_stream.restype = ct.c_int32
    lib.pwgpu_kernel_launches.argtypes = [ct.POINTER(ct.c_int64)]
    lib.pwgpu_kernel_launches.restype = ct.c_int32
    lib.pwgpu_server_create.argtypes = [ct.POINTER(PwgpuServerOptions), ct.POINTER(vp)]
    lib.pwgpu_server_destroy.argtypes = [vp]
    lib.pwgpu_scf_iter1_from_rho_g.argtypes = [vp, ct.POINTER(PwgpuScfParams), _f64p, ct.POINTER(PwgpuScfResult),
                                               _f64p, _f64p, _f64p, _f64p]
    lib.pwgpu_server_submit.argtypes = [vp, ct.POINTER(PwgpuSystem), ct.POINTER(PwgpuScfParams), _f64p,
                                        ct.POINTER(ct.c_int64)]
    lib.pwgpu_server_poll.argtypes = [vp, ct.c_int64, ct.POINTER(PwgpuJobInfo)]
    lib.pwgpu_server_wait.argtypes = [vp, ct.c_int64, ct.c_double, ct.POINTER(PwgpuJobInfo)]
    lib.pwgpu_server_wait_any.argtypes = [vp, ct.c_double, ct.POINTER(ct.c_int64)]
    lib.pwgpu_server_result.argtypes = [vp, ct.c_int64, ct.POINTER(PwgpuScfResult), _f64p, ct.POINTER(ct.c_char_p)]
    lib.pwgpu_server_release.argtypes = [vp, ct.c_int64]
    lib.pwgpu_server_get_stats.argtypes = [vp, ct.POINTER(PwgpuServerStats)]
    lib.pwgpu_upf_parse.argtypes = [ct.c_char_p, ct.c_int64, ct.POINTER(vp)]
    lib.pwgpu_upf_load.argtypes = [ct.c_char_p, ct.POINTER(vp)]
    lib.pwgpu_upf_get_info.argtypes = [vp, ct.POINTER(PwgpuUpfInfo)]
    lib.pwgpu_upf_get_array.argtypes = [vp, ct.c_int32, ct.c_int32, _f64p, ct.c_int64]
    lib.pwgpu_upf_get_beta_l.argtypes = [vp, _i32p]
    lib.pwgpu_upf_free.argtypes = [vp]
    lib.pwgpu_deck_parse.argtypes = [ct.c_char_p, ct.c_int64, ct.POINTER(vp)]
    lib.pwgpu_deck_get_settings.argtypes = [vp, ct.POINTER(PwgpuDeckSettings)]
    lib.pwgpu_deck_get_atoms.argtypes = [vp, ct.c_char_p, _f64p]
    lib.pwgpu_deck_get_starting_magnetization.argtypes = [vp, ct.c_char_p, _f64p]
    lib.pwgpu_deck_get_band_path.argtypes = [vp, ct.c_char_p, _f64p]
    lib.pwgpu_deck_free.argtypes = [vp]
    for name in ("pwgpu_create", "pwgpu_destroy", "pwgpu_set_veff_g", "pwgpu_apply_h", "pwgpu_apply_h_device",
                 "pwgpu_set_precision", "pwgpu_get_dims", "pwgpu_profile_apply_h", "pwgpu_scf_run", "pwgpu_scf_iter1_from_rho_g",
                 "pwgpu_eigensolve", "pwgpu_density", "pwgpu_symmetrize", "pwgpu_potentials",
                 "pwgpu_small_geneig", "pwgpu_occupations", "pwgpu_mix", "pwgpu_mix_reset", "pwgpu_get_projectors", "pwgpu_initial_density",
                 "pwgpu_get_local_potential", "pwgpu_server_create", "pwgpu_server_destroy",
                 "pwgpu_server_submit", "pwgpu_server_poll", "pwgpu_server_wait", "pwgpu_server_wait_any",
                 "pwgpu_server_result", "pwgpu_server_release", "pwgpu_server_get_stats", "pwgpu_upf_parse",
                 "pwgpu_upf_load", "pwgpu_upf_get_info", "pwgpu_upf_get_array", "pwgpu_upf_get_beta_l",
                 "pwgpu_upf_free", "pwgpu_deck_parse", "pwgpu_deck_get_settings", "pwgpu_deck_get_atoms",
                 "pwgpu_deck_get_starting_magnetization", "pwgpu_deck_get_band_path", "pwgpu_deck_free"):
        getattr(lib, name).restype = ct.c_int32
    _lib = lib
    return lib


def _upf_from_handle(lib, h):
    from .upf import Upf
    info = PwgpuUpfInfo()
    _check(lib, lib.pwgpu_upf_get_info(h, ct.byref(info)))
    mesh, nproj = info.mesh, info.n_proj

    def arr(which, index=0, n=mesh):
        out = np.zeros(n)
        _check(lib, lib.pwgpu_upf_get_array(h, which, index, _f64(out), n))
        return out

    ls = np.zeros(max(nproj, 1), dtype=np.int32)
    _check(lib, lib.pwgpu_upf_get_beta_l(h, _i32(ls)))
    core = arr(UPF_NLCC) if info.has_nlcc else np.zeros(0)
    return Upf(info.element.decode(), info.z_valence, info.l_max, arr(UPF_R), arr(UPF_RAB), arr(UPF_LOCAL),
               [int(x) for x in ls[:nproj]], [arr(UPF_BETA, i) for i in range(nproj)], arr(UPF_DIJ, n=nproj * nproj),
               arr(UPF_RHOATOM), core)


def load_upf_native(path: str = None, text: str = None):
    """A UPF read by the library's own parser (pwgpu_upf_load / pwgpu_upf_parse,
    parse_upf_body, upf/parse.rs:20-135), returned as the same Upf object the
    Python reader gives; raises PwGpuError(PWGPU_E_PARSE) on a malformed file."""
    lib = load_library()
    h = ct.c_void_p()
    if text is not None:
        raw = text.encode()
        _check(lib, lib.pwgpu_upf_parse(raw, len(raw), ct.byref(h)))
    else:
        _check(lib, lib.pwgpu_upf_load(os.fsencode(path), ct.byref(h)))
    try:
        return _upf_from_handle(lib, h)
    finally:
        lib.pwgpu_upf_free(h)


def _check(lib, rc):
    if rc != PWGPU_OK:
        raise PwGpuError(rc, lib.pwgpu_last_error().decode(errors="replace"))


def _f64(a):
    return a.ctypes.data_as(_f64p)


def _i32(a):
    return a.ctypes.data_as(_i32p)


def pack_system(sys_) -> tuple:
    """Flatten an ScfSystem into the pwgpu_system POD.  Returns (struct, keepalive)."""
    keep = []

    def hold(a):
        keep.append(a)
        return a

    n_pw = sys_.n_pw
    miller = hold(np.ascontiguousarray(sys_.basis.miller, dtype=np.int32))
    kw = hold(np.ascontiguousarray(sys_.kpt_weights, dtype=np.float64))
    kin = hold(np.ascontiguousarray(np.stack(sys_.kinetic), dtype=np.float64))
    projs = sys_.projectors
    n_ch = projs[0].n_ch if projs else 0
    s = PwgpuSystem()
    s.dims[:] = list(sys_.dims)
    s.n_pw = n_pw
    s.miller = _i32(miller)
    s.n_k = len(sys_.kpoints)
    s.k_weights = _f64(kw)
    s.kinetic = _f64(kin)
    s.n_ch = n_ch
    packed = []

    def species_radial():
        """Atoms and species meshes shared by the device builds (packed once)."""
        cr, pps = sys_.crystal, sys_.extra["pps"]
        species = list(dict.fromkeys(a.symbol for a in cr.atoms))
        if not packed:
            s.atom_tau = _f64(hold(np.ascontiguousarray(np.array([a.cart(cr.lattice) for a in cr.atoms]),
                                                        dtype=np.float64)))
            s.atom_species = _i32(hold(np.array([species.index(a.symbol) for a in cr.atoms], dtype=np.int32)))
            s.n_species = len(species)
            s.species_mesh = _i32(hold(np.array([pps[sp].r.size for sp in species], dtype=np.int32)))
            s.radial_r = _f64(hold(np.concatenate([pps[sp].r for sp in species]).astype(np.float64)))
            s.radial_rab = _f64(hold(np.concatenate([pps[sp].rab for sp in species]).astype(np.float64)))
            packed.append(True)
        return species

    if n_ch:
        starts = hold(np.ascontiguousarray(projs[0].atom_ch_start, dtype=np.int32))
        blocks = hold(np.concatenate([blk.ravel() for blk in projs[0].d_blocks]).astype(np.float64))
        s.n_atoms = len(projs[0].d_blocks)
        s.atom_ch_start = _i32(starts)
        s.d_blocks = _f64(blocks)
        if projs[0].b is not None:
            b = hold(np.concatenate([np.asfortranarray(p.b).ravel(order="F") for p in projs]).astype(np.complex128))
            s.proj_b = b.view(np.float64).ctypes.data_as(_f64p)
        else:
            # radial form: the device builds B (NonlocalPotential::new on the GPU)
            pps = sys_.extra["pps"]
            species = species_radial()
            s.g_cart = _f64(hold(np.ascontiguousarray(sys_.basis.g, dtype=np.float64)))
            s.k_cart = _f64(hold(np.ascontiguousarray(np.array([kp.k for kp in sys_.kpoints]), dtype=np.float64)))
            s.species_nbeta = _i32(hold(np.array([len(pps[sp].beta_l) for sp in species], dtype=np.int32)))
            s.beta_l = _i32(hold(np.array([l for sp in species for l in pps[sp].beta_l], dtype=np.int32)))
            betas = [np.asarray(pps[sp].beta[i], dtype=np.float64) for sp in species for i in range(len(pps[sp].beta_l))]
            s.beta_r = _f64(hold(np.concatenate(betas) if betas else np.zeros(1)))
    if sys_.v_local_g is not None:
        vl = hold(np.ascontiguousarray(sys_.v_local_g, dtype=np.complex128))
        s.v_local_g = vl.view(np.float64).ctypes.data_as(_f64p)
        if sys_.rho_core_r.size:
            rc = hold(np.ascontiguousarray(sys_.rho_core_r, dtype=np.float64))
            s.rho_core_r = _f64(rc)
    else:
        # radial form: the device builds V_loc(G), the core density and the start density
        pps = sys_.extra["pps"]
        species = species_radial()
        s.n_atoms = len(sys_.crystal.atoms)
        rec = sys_.crystal.lattice.reciprocal()
        s.recip = _f64(hold(np.ascontiguousarray(np.array([rec.a, rec.b, rec.c]), dtype=np.float64)))
        s.species_zval = _f64(hold(np.array([pps[sp].z_valence for sp in species], dtype=np.float64)))
        s.vloc_r = _f64(hold(np.concatenate([pps[sp].v_local for sp in species]).astype(np.float64)))
        flags = np.array([(1 if pps[sp].has_nlcc() else 0) | (2 if pps[sp].has_rho_atom() else 0)
                          for sp in species], dtype=np.int32)
        s.species_flags = _i32(hold(flags))
        if np.any(flags & 1):
            s.core_r = _f64(hold(np.concatenate([pps[sp].core_charge if pps[sp].has_nlcc() else np.zeros(pps[sp].r.size)
                                                 for sp in species]).astype(np.float64)))
        if np.any(flags & 2):
            s.rho_atom_r = _f64(hold(np.concatenate([pps[sp].rho_atom if pps[sp].has_rho_atom()
                                                     else np.zeros(pps[sp].r.size) for sp in species])
                                     .astype(np.float64)))
        s.gaussian_sigma = sys_.extra["gaussian_sigma"]
    g2 = hold(np.ascontiguousarray(sys_.g_squared, dtype=np.float64))
    s.g_squared = _f64(g2)
    n_sym = sys_.symmetry.n_ops
    s.n_sym = n_sym
    if n_sym > 1:
        from .symmetry import g_space_gather_map
        src, arg = g_space_gather_map(sys_.dims, sys_.symmetry)
        src = hold(np.ascontiguousarray(src, dtype=np.int32))
        arg = hold(np.ascontiguousarray(arg, dtype=np.float64))
        s.sym_src = _i32(src)
        s.sym_arg = _f64(arg)
    s.n_electrons = sys_.n_electrons
    s.omega = sys_.omega
    s.e_ewald = sys_.e_ewald
    s.nspin = sys_.nspin
    return s, keep


class PwGpu:
    """One device handle (pwgpu_create .. pwgpu_destroy)."""

    def __init__(self, sys_, precision: int = PRECISION_FP64, device: int = 0, lanes: int = 0,
                 gamma_complex: bool = False):
        self.lib = load_library()
        self.sys = sys_
        st, keep = pack_system(sys_)
        opt = PwgpuOptions(device, precision, lanes, 1 if gamma_complex else 0)
        h = ct.c_void_p()
        _check(self.lib, self.lib.pwgpu_create(ct.byref(st), ct.byref(opt), ct.byref(h)))
        self.h = h
        self.n_pw = sys_.n_pw

    def close(self):
        if self.h:
            self.lib.pwgpu_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def stream(self) -> int:
        """cudaStream_t of the handle (as an integer)."""
        s = ct.c_void_p()
        _check(self.lib, self.lib.pwgpu_get_stream(self.h, ct.byref(s)))
        return s.value or 0

    def set_precision(self, precision: int):
        _check(self.lib, self.lib.pwgpu_set_precision(self.h, precision))

    def set_veff_g(self, veff_g: np.ndarray, spin: int = 0):
        v = np.ascontiguousarray(veff_g, dtype=np.complex128)
        _check(self.lib, self.lib.pwgpu_set_veff_g(self.h, spin, v.view(np.float64).ctypes.data_as(_f64p)))

    def apply_h(self, psi: np.ndarray, ik: int = 0, spin: int = 0) -> np.ndarray:
        p = np.asfortranarray(psi, dtype=np.complex128)
        if p.ndim == 1:
            p = p[:, None]
        nb = p.shape[1]
        out = np.empty((self.n_pw, nb), dtype=np.complex128, order="F")
        _check(self.lib, self.lib.pwgpu_apply_h(self.h, spin, ik, p.ravel(order="F").view(np.float64).ctypes.data_as(_f64p),
                                                nb, out.ravel(order="F").view(np.float64).ctypes.data_as(_f64p)))
        return out

    def apply_h_device(self, psi_ptr: int, ldpsi: int, nb: int, hpsi_ptr: int, ldh: int, ik: int = 0, spin: int = 0,
                       stream: int = 0):
        _check(self.lib, self.lib.pwgpu_apply_h_device(self.h, spin, ik, ct.c_void_p(psi_ptr), ldpsi, nb,
                                                       ct.c_void_p(hpsi_ptr), ldh, ct.c_void_p(stream or None)))

    def profile_apply_h(self, psi_ptr: int, ldpsi: int, nb: int, hpsi_ptr: int, ldh: int, ik: int = 0, spin: int = 0):
        """Per-stage device ms and launch counts of one H|psi> call (8 stages)."""
        ms = np.zeros(8)
        n = np.zeros(8, dtype=np.int32)
        _check(self.lib, self.lib.pwgpu_profile_apply_h(self.h, spin, ik, ct.c_void_p(psi_ptr), ldpsi, nb,
                                                        ct.c_void_p(hpsi_ptr), ldh, _f64(ms), _i32(n)))
        return ms, n

    # -- SCF pieces ---------------------------------------------------------

    def scf_run(self, rho_init: np.ndarray, n_bands: int, max_iter: int = 100, conv_threshold: float = 1e-6,
                energy_threshold: float = 1e-5, mixing_beta: float = 0.3, mixing_ndim: int = 8, kerker: bool = False,
                q_tf: float = 0.0, smearing: str = "fermi_dirac", sigma: float = 0.01, diag_tol: float = 1e-8,
                diag_max_iter: int = 60, diag_extra_bands: int = -1, precision: int = PRECISION_FP64,
                fp64_switch: float = 1e-6, verbose: bool = False, raise_on_unconverged: bool = True,
                starting_magnetization: float = 0.0, tot_magnetization=None, mixer: str = "anderson",
                mixing_period: int = 3, diag_tol_per_drho: float = 0.0, diag_tol_cap: float = 0.0):
        """run_scf_unpolarized / run_scf_spin on the device; returns (result dict, eigenvalues
        [nspin * n_k, n_bands] (spin up k-points first), rho_r [nspin * N] (up then down),
        total rho_g in basis order [n_pw])."""
        p = scf_params(n_bands, max_iter, conv_threshold, energy_threshold, mixing_beta, mixing_ndim, kerker, q_tf,
                       smearing, sigma, diag_tol, diag_max_iter, diag_extra_bands, precision, fp64_switch, verbose,
                       starting_magnetization, tot_magnetization, mixer, mixing_period, diag_tol_per_drho,
                       diag_tol_cap)
        rho0 = np.ascontiguousarray(rho_init, dtype=np.float64)
        res = PwgpuScfResult()
        ns = self.sys.nspin
        nk = len(self.sys.kpoints)
        ev = np.zeros((ns * nk, n_bands))
        rho = np.zeros(ns * self.sys.n_grid)
        rg = np.zeros(self.n_pw, dtype=np.complex128)
        rc = self.lib.pwgpu_scf_run(self.h, ct.byref(p), _f64(rho0), ct.byref(res), _f64(ev), _f64(rho),
                                    rg.view(np.float64).ctypes.data_as(_f64p))
        if rc != PWGPU_OK and (raise_on_unconverged or rc != -4):
            raise PwGpuError(rc, self.lib.pwgpu_last_error().decode(errors="replace"))
        return res.as_dict(), ev, rho, rg

    def apply_h_packed(self, u: np.ndarray, spin: int = 0) -> np.ndarray:
        """H on Gamma-packed real bands (n_pw, nb) at the handle's precision."""
        uf = np.asfortranarray(u, dtype=np.float64)
        if uf.ndim == 1:
            uf = uf[:, None]
        out = np.empty_like(uf, order="F")
        _check(self.lib, self.lib.pwgpu_apply_h_packed(self.h, spin, uf.ravel(order="F").ctypes.data_as(_f64p),
                                                       uf.shape[1], out.ravel(order="F").ctypes.data_as(_f64p)))
        return out

    def get_bands(self, n_bands: int, ik: int = 0, spin: int = 0) -> np.ndarray:
        """Eigenvectors of (spin, ik) left by the last SCF run or eigensolve: (n_pw, n_bands) complex."""
        out = np.zeros((n_bands, self.n_pw), dtype=np.complex128)  # row b = band b (column-major n_pw x nb)
        _check(self.lib, self.lib.pwgpu_get_bands(self.h, spin, ik, n_bands, out.view(np.float64).ctypes.data_as(_f64p)))
        return out.T

    def scf_iter1_from_rho_g(self, rho_g_fft: np.ndarray, n_bands: int, smearing: str = "fermi_dirac",
                             sigma: float = 0.01, diag_tol: float = 1e-10, diag_max_iter: int = 60,
                             diag_extra_bands: int = -1, precision: int = PRECISION_FP64):
        """One SCF iteration seeded from rho(G) on the full FFT grid (run_scf_iter1_from_rho_g_fft,
        scf/transplant.rs:114-376); returns (result dict, eigenvalues [n_k, n_bands], rho_r_out [N],
        rho_g_fft_out [N] complex, rho_r_in [N])."""
        p = scf_params(n_bands, 1, 0.0, 0.0, 0.3, 1, False, 0.0, smearing, sigma, diag_tol, diag_max_iter,
                       diag_extra_bands, precision, 1e-6, False)
        rg = np.ascontiguousarray(rho_g_fft, dtype=np.complex128).ravel()
        n = self.sys.n_grid
        if rg.size != n:
            raise ValueError(f"rho_g_fft has {rg.size} entries; the FFT grid has {n}")
        res = PwgpuScfResult()
        ev = np.zeros((len(self.sys.kpoints), n_bands))
        rho = np.zeros(n)
        rg_out = np.zeros(n, dtype=np.complex128)
        rho_in = np.zeros(n)
        _check(self.lib, self.lib.pwgpu_scf_iter1_from_rho_g(
            self.h, ct.byref(p), rg.view(np.float64).ctypes.data_as(_f64p), ct.byref(res), _f64(ev), _f64(rho),
            rg_out.view(np.float64).ctypes.data_as(_f64p), _f64(rho_in)))
        return res.as_dict(), ev, rho, rg_out, rho_in

    def mix(self, rho_in: np.ndarray, rho_out: np.ndarray, beta: float, ndim: int, kerker: bool = False,
            q_tf: float = 0.0, channel: int = 0, mixer: str = "anderson", period: int = 3) -> np.ndarray:
        """One mixing step (Anderson / Broyden / Periodic Pulay, optional Kerker) on the device
        history `channel`; returns the next input density."""
        a = np.ascontiguousarray(rho_in, dtype=np.float64)
        b = np.ascontiguousarray(rho_out, dtype=np.float64)
        out = np.empty_like(a)
        _check(self.lib, self.lib.pwgpu_mix(self.h, channel, mixing_mode(mixer, kerker), _f64(a), _f64(b),
                                            _f64(out), beta, ndim, period, q_tf))
        return out

    def initial_density(self) -> np.ndarray:
        """The device-built start density (N,) of a system whose local part is built on the device."""
        out = np.zeros(self.sys.n_grid)
        _check(self.lib, self.lib.pwgpu_initial_density(self.h, _f64(out)))
        return out

    def local_potential(self):
        """(V_loc(G) (N,) complex, rho_core(r) (N,)) as held on the device."""
        n = self.sys.n_grid
        v = np.zeros(n, dtype=np.complex128)
        rc = np.zeros(n)
        _check(self.lib, self.lib.pwgpu_get_local_potential(self.h, v.view(np.float64).ctypes.data_as(_f64p),
                                                           _f64(rc)))
        return v, rc

    def projectors(self, ik: int = 0) -> np.ndarray:
        """The device copy of B at k-point ik (n_pw x n_ch complex)."""
        n_ch = self.sys.projectors[ik].n_ch
        out = np.zeros((self.n_pw, n_ch), dtype=np.complex128, order="F")
        _check(self.lib, self.lib.pwgpu_get_projectors(self.h, ik,
                                                       out.ravel(order="F").view(np.float64).ctypes.data_as(_f64p)))
        return out

    def mix_reset(self):
        _check(self.lib, self.lib.pwgpu_mix_reset(self.h))

    def eigensolve(self, n_bands: int, ik: int = 0, spin: int = 0, tol: float = 1e-9, max_iter: int = 300,
                   psi_in=None):
        ev = np.zeros(n_bands)
        psi = np.zeros((self.n_pw, n_bands), dtype=np.complex128, order="F")
        it = ct.c_int32()
        mr = ct.c_double()
        pin = None
        if psi_in is not None:
            pin = np.asfortranarray(psi_in, dtype=np.complex128)
            pin = pin.ravel(order="F").view(np.float64).ctypes.data_as(_f64p)
        _check(self.lib, self.lib.pwgpu_eigensolve(self.h, spin, ik, n_bands, tol, max_iter, pin, _f64(ev),
                                                   psi.ravel(order="F").view(np.float64).ctypes.data_as(_f64p),
                                                   ct.byref(it), ct.byref(mr)))
        return ev, psi, it.value, mr.value

    def density(self, occ: np.ndarray, psis) -> np.ndarray:
        """occ [n_k, n_bands]; psis: list of n_k blocks (n_pw, n_bands)."""
        occ = np.ascontiguousarray(occ, dtype=np.float64)
        nb = occ.shape[1]
        allp = np.concatenate([np.asfortranarray(p, dtype=np.complex128).ravel(order="F") for p in psis])
        rho = np.zeros(self.sys.n_grid)
        _check(self.lib, self.lib.pwgpu_density(self.h, nb, _f64(occ), allp.view(np.float64).ctypes.data_as(_f64p),
                                                _f64(rho)))
        return rho

    def symmetrize(self, rho: np.ndarray) -> np.ndarray:
        r = np.ascontiguousarray(rho, dtype=np.float64).copy()
        _check(self.lib, self.lib.pwgpu_symmetrize(self.h, _f64(r)))
        return r

    def potentials(self, rho: np.ndarray):
        r = np.ascontiguousarray(rho, dtype=np.float64)
        vg = np.zeros(self.sys.n_grid, dtype=np.complex128)
        en = np.zeros(3)
        _check(self.lib, self.lib.pwgpu_potentials(self.h, _f64(r), vg.view(np.float64).ctypes.data_as(_f64p),
                                                   _f64(en)))
        return vg, {"e_hartree": en[0], "e_xc": en[1], "e_vxc": en[2]}


def kernel_launches() -> int:
    """This library's kernel launches since load (pwgpu_kernel_launches)."""
    lib = load_library()
    n = ct.c_int64()
    _check(lib, lib.pwgpu_kernel_launches(ct.byref(n)))
    return n.value


def occupations(eigenvalues, weights, n_electrons: float, sigma: float, smearing: str = "fermi_dirac",
                spin_factor: float = 2.0, fermi_energy: float | None = None):
    """Fermi level, occupations and TS through the library's host code
    (pwgpu_occupations; find_fermi_energy / occupation / entropy_ts,
    scf/smearing.rs:38-252).  eigenvalues: (n_sets, nb); weights: (n_sets,).
    fermi_energy None: searched for n_electrons; else used as given.
    Returns (fermi_energy, occ [n_sets, nb] = spin_factor f, TS)."""
    lib = load_library()
    ev = np.ascontiguousarray(np.atleast_2d(eigenvalues), dtype=np.float64)
    w = np.ascontiguousarray(weights, dtype=np.float64)
    ef = np.array([0.0 if fermi_energy is None else float(fermi_energy)])
    occ = np.zeros_like(ev)
    ts = np.zeros(1)
    _check(lib, lib.pwgpu_occupations(ev.shape[0], ev.shape[1], _f64(ev), _f64(w), float(n_electrons), float(sigma),
                                      SMEARING[smearing], float(spin_factor), 1 if fermi_energy is None else 0,
                                      _f64(ef), _f64(occ), _f64(ts)))
    return float(ef[0]), occ, float(ts[0])


def small_geneig(H: np.ndarray, S: np.ndarray, nev: int):
    """Batched generalized Hermitian eigensolve through the device kernel.
    H, S: (batch, m, m) complex.  Returns (evals [batch, nev], C [batch, m, nev])."""
    lib = load_library()
    b, m, _ = H.shape
    hf = np.ascontiguousarray(np.transpose(H, (0, 2, 1)), dtype=np.complex128)  # column-major per matrix
    sf = np.ascontiguousarray(np.transpose(S, (0, 2, 1)), dtype=np.complex128)
    ev = np.zeros((b, nev))
    c = np.zeros((b, nev, m), dtype=np.complex128)
    _check(lib, lib.pwgpu_small_geneig(b, m, nev, hf.view(np.float64).ctypes.data_as(_f64p),
                                       sf.view(np.float64).ctypes.data_as(_f64p), _f64(ev),
                                       c.view(np.float64).ctypes.data_as(_f64p)))
    return ev, np.transpose(c, (0, 2, 1))


def dense_eigh(A: np.ndarray, nev: int, timed: bool = False):
    """Lowest nev eigenpairs of a dense Hermitian or real symmetric matrix
    through the device's cluster eigensolver.  Returns (w [nev], Z [m, nev],
    cluster CTAs used), plus the kernel's device ms when timed."""
    lib = load_library()
    m = A.shape[0]
    cpx = np.iscomplexobj(A)
    dt = np.complex128 if cpx else np.float64
    af = np.asfortranarray(A, dtype=dt)
    w = np.zeros(nev)
    z = np.zeros((nev, m), dtype=dt)  # row j = eigenvector j (column-major m x nev)
    nc = ct.c_int32(0)
    ms = ct.c_double(0.0)
    _check(lib, lib.pwgpu_dense_eigh(m, nev, 1 if cpx else 0, af.ravel(order="F").view(np.float64).ctypes.data_as(_f64p),
                                     _f64(w), z.view(np.float64).ctypes.data_as(_f64p), ct.byref(nc),
                                     ct.byref(ms) if timed else None))
    return (w, z.T, nc.value, ms.value) if timed else (w, z.T, nc.value)


def dense_cholesky_inverse(G: np.ndarray, timed: bool = False):
    """Cholesky factor G = R^H R of a Hermitian / real symmetric positive
    definite matrix through the device's cluster kernel.  Returns (Ri = R^-1,
    diag(R), info, cluster CTAs used), plus the kernel's device ms when
    timed; info = 1 + the first failing pivot row, 0 on success."""
    lib = load_library()
    q = G.shape[0]
    cpx = np.iscomplexobj(G)
    dt = np.complex128 if cpx else np.float64
    gf = np.asfortranarray(G, dtype=dt)
    ri = np.zeros((q, q), dtype=dt)  # filled column-major: transposed view below
    rd = np.zeros(q)
    info = ct.c_int32(0)
    nc = ct.c_int32(0)
    ms = ct.c_double(0.0)
    _check(lib, lib.pwgpu_dense_cholesky_inverse(q, 1 if cpx else 0,
                                                 gf.ravel(order="F").view(np.float64).ctypes.data_as(_f64p),
                                                 ri.view(np.float64).ctypes.data_as(_f64p), _f64(rd),
                                                 ct.byref(info), ct.byref(nc), ct.byref(ms) if timed else None))
    out = (ri.T.copy(), rd, info.value, nc.value)
    return out + (ms.value,) if timed else out

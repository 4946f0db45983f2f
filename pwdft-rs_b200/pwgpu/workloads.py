"""Seeded synthetic workloads with the shapes of the named benchmark configs.

si64_hpsi: 64-atom Si cubic supercell (2x2x2 conventional cells of
a = 10.26 bohr, i.e. 20.52 bohr box), diamond sites with seeded uniform
±0.05 bohr Cartesian displacements, Γ point, ecutwfc 30 Ry (n_pw = 23,847 on
a 72^3 grid by the reference's basis and grid rules).  160 bands of seeded
complex Gaussian coefficients normalised per band; V_eff(r) seeded uniform
in [-1, 0] Ha; 256 Kleinman-Bylander channels (one s and one p radial
projector per atom, Gaussian form factors F_0(q) = A e^{-q²r_c²/2},
F_1(q) = A q r_c e^{-q²r_c²/2}, r_c = 1 bohr, A = 1) entering B exactly as
the reference's NonlocalPotential::new does (1/√Ω, e^{-iG·τ}, real Y_lm);
D diagonal per (atom, l), seeded uniform in [0.1, 2] Ha, equal across m.
"""

from __future__ import annotations

import math

import numpy as np

from .consts import BOHR_TO_ANG, HA_TO_EV, RY_TO_EV
from .context import Projectors, ScfSystem, build_projectors, forward_fft_unnormalized
from .crystal import BasisSet, Crystal, KPoint, diamond_supercell, grid_dims_for, miller_to_idx
from .symmetry import SymmetryInfo

SEED = 20261203


def si64_crystal(seed: int = SEED) -> Crystal:
    rng = np.random.default_rng(seed)
    return diamond_supercell("Si", 10.26 * BOHR_TO_ANG, (2, 2, 2), 0.05 * BOHR_TO_ANG, rng)


def gaussian_projector_table(rc_ang: float, amp: float = 1.0):
    def ff(i, q):
        x = q * rc_ang
        g = amp * np.exp(-0.5 * x * x)
        return g if i == 0 else g * x
    return ([0, 1], ff, np.zeros(4))


def hpsi_system(crystal: Crystal, ecut_ry: float = 30.0, n_bands: int = 160, seed: int = SEED,
                k=(0.0, 0.0, 0.0)):
    """ScfSystem + V_eff(G) + ψ block for the synthetic H|ψ> benchmark."""
    rng = np.random.default_rng(seed + 1)
    basis = BasisSet(crystal.lattice, ecut_ry * RY_TO_EV)
    dims = grid_dims_for(basis, 4)
    n = int(np.prod(dims))
    kp = [KPoint(np.asarray(k, dtype=np.float64), 1.0)]
    table = {"Si": gaussian_projector_table(1.0 * BOHR_TO_ANG)}
    proj = build_projectors(crystal, basis, kp[0].k, {sp: table["Si"] for sp in crystal.species()})
    blocks = []
    for _ in crystal.atoms:
        ds, dp = rng.uniform(0.1, 2.0, 2) * HA_TO_EV
        blocks.append(np.diag([ds, dp, dp, dp]))
    proj = Projectors(proj.b, blocks, proj.atom_ch_start)
    g_to_fft = miller_to_idx(dims, basis.miller[:, 0].astype(np.int64), basis.miller[:, 1].astype(np.int64),
                             basis.miller[:, 2].astype(np.int64))
    v_r = rng.uniform(-1.0, 0.0, n) * HA_TO_EV
    veff_g = forward_fft_unnormalized(v_r.astype(np.complex128), dims) / n
    psi = rng.standard_normal((len(basis), n_bands)) + 1j * rng.standard_normal((len(basis), n_bands))
    psi /= np.linalg.norm(psi, axis=0)
    sys_ = ScfSystem(crystal, basis, dims, g_to_fft, kp, [basis.kinetic(kp[0].k)], [proj],
                     np.zeros(n, dtype=np.complex128), np.zeros(n), np.zeros(0), 256.0,
                     crystal.lattice.volume(), 0.0, SymmetryInfo.identity_only(), np.zeros(0))
    return sys_, veff_g, np.asfortranarray(psi)


def hpsi_algorithmic_bytes(n_pw: int, n_grid: int, c_bytes: int) -> float:
    """Local H|ψ> bytes per band: ψ read + Hψ write (2 c n_pw), inverse and
    forward full-grid FFT as one read+write each (4 c N), V_eff(r) read (c/2 N)."""
    return 2.0 * c_bytes * n_pw + 4.0 * c_bytes * n_grid + 0.5 * c_bytes * n_grid


def nonlocal_flops(n_pw: int, n_ch: int, n_b: int) -> float:
    """Two complex GEMMs, 8 n_pw n_ch n_b flops each."""
    return 2.0 * 8.0 * n_pw * n_ch * n_b


def fft_flops(n_grid: int) -> float:
    return 2.0 * 5.0 * n_grid * math.log2(n_grid)

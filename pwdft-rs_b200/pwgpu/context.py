"""Per-calculation invariants consumed by the SCF hot path (the data contract).

Host-side mirror of ScfContext::new (pwdft/pwdft-core/src/scf/context.rs:102-231):
FFT grid and index maps, V_loc(G) on the full grid, NLCC core density,
Kleinman-Bylander projector matrices B per k-point with their
block-diagonal D, Ewald energy, k-point weights and the SAD start density.
None of this is on the per-iteration path; the GPU library consumes the
arrays built here.
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from .consts import E2_COULOMB, HBAR2_OVER_2M
from .crystal import BasisSet, Crystal, grid_dims_for, grid_g_vectors, miller_to_idx
from .symmetry import SymmetryInfo, g_space_gather_map
from .upf import Upf, beta_form_factor, sinc_transform, v_local_of_g


def inverse_fft_unnormalized(x_flat, dims):
    """f(r) = Σ_G f(G) e^{+iG·r}, no 1/N (fft.rs:89-114)."""
    return np.fft.ifftn(x_flat.reshape(dims), norm="forward").ravel()


def forward_fft_unnormalized(x_flat, dims):
    """f(G) = Σ_r f(r) e^{-iG·r}, no 1/N (fft.rs:62-87)."""
    return np.fft.fftn(x_flat.reshape(dims)).ravel()


def real_sph_harmonics(q: np.ndarray, lmax: int) -> np.ndarray:
    """Real Y_lm(q̂) for all q rows, order (0,0),(1,0),(1,+1),(1,-1),(2,0),(2,+1),(2,-1),...

    Same recurrence and conventions as nonlocal.rs:469-552: Y_lm = 0 for l>0
    when |q| < 1e-9; φ = atan2(qy, qx); the +m slot carries cos(mφ), the −m
    slot sin(mφ), both with a √2 normalisation.
    """
    n = q.shape[0]
    out = np.zeros((n, (lmax + 1) ** 2))
    fpi = 4.0 * math.pi
    out[:, 0] = math.sqrt(1.0 / fpi)
    if lmax == 0:
        return out
    gmod = np.sqrt((q[:, 0] * q[:, 0] + q[:, 1] * q[:, 1]) + q[:, 2] * q[:, 2])
    ok = gmod >= 1e-9
    gm = np.where(ok, gmod, 1.0)
    cost = q[:, 2] / gm
    sint = np.sqrt(np.maximum(1.0 - cost * cost, 0.0))
    phi = np.arctan2(q[:, 1], q[:, 0])
    Q = {}
    Q[(0, 0)] = np.ones(n)
    Q[(1, 0)] = cost
    Q[(1, 1)] = -sint / math.sqrt(2.0)
    c1 = math.sqrt(3.0 / fpi)
    out[:, 1] = c1 * Q[(1, 0)]
    out[:, 2] = c1 * math.sqrt(2.0) * Q[(1, 1)] * np.cos(phi)
    out[:, 3] = c1 * math.sqrt(2.0) * Q[(1, 1)] * np.sin(phi)
    lm = 4
    for l in range(2, lmax + 1):
        c = math.sqrt((2 * l + 1) / fpi)
        for m in range(0, l - 1):
            llmm = math.sqrt(l * l - m * m)
            llm1 = math.sqrt((l - 1) * (l - 1) - m * m)
            Q[(l, m)] = (cost * (2.0 * l - 1.0) * Q[(l - 1, m)] - llm1 * Q[(l - 2, m)]) / llmm
        Q[(l, l - 1)] = cost * math.sqrt(2.0 * l - 1.0) * Q[(l - 1, l - 1)]
        Q[(l, l)] = -math.sqrt((2.0 * l - 1.0) / (2.0 * l)) * sint * Q[(l - 1, l - 1)]
        out[:, lm] = c * Q[(l, 0)]
        for m in range(1, l + 1):
            out[:, lm + 2 * m - 1] = c * math.sqrt(2.0) * Q[(l, m)] * np.cos(m * phi)
            out[:, lm + 2 * m] = c * math.sqrt(2.0) * Q[(l, m)] * np.sin(m * phi)
        lm += 2 * l + 1
    out[~ok, 1:] = 0.0
    return out


@dataclass
class Projectors:
    """Expanded KB projector matrix of one k-point (nonlocal.rs:190-382).

    b[G, c]  = (1/√Ω) e^{−iG·τ_a(c)} F_i(c)(|k+G|) Y_{l m}(c)(k+G)   (n_pw x n_ch)
    H_NL     = B · D · B^H with D block-diagonal over (atom, l, m).
    D is stored per atom as a dense n_ch_atom x n_ch_atom real block;
    atom_ch_start[a] is the first channel of atom a.
    """
    b: np.ndarray                  # complex128 (n_pw, n_ch), column-major friendly
    d_blocks: list                 # per atom, (nc, nc) float64
    atom_ch_start: np.ndarray      # int32 (n_atoms + 1,)

    @property
    def n_ch(self):
        return int(self.atom_ch_start[-1]) if self.b is None else self.b.shape[1]

    def d_dense(self) -> np.ndarray:
        n = self.n_ch
        d = np.zeros((n, n))
        for a, blk in enumerate(self.d_blocks):
            s = self.atom_ch_start[a]
            d[s:s + blk.shape[0], s:s + blk.shape[0]] = blk
        return d


def _atom_d_block(ls, dij):
    """D[(i,m),(j,m')] = D_ij if l_i == l_j and m == m' (nonlocal.rs:346-379)."""
    nproj = len(ls)
    starts, nc = [], 0
    for l in ls:
        starts.append(nc)
        nc += 2 * l + 1
    blk = np.zeros((nc, nc))
    for i in range(nproj):
        for j in range(nproj):
            if ls[i] != ls[j]:
                continue
            dv = dij[i * nproj + j]
            if abs(dv) < 1e-20:
                continue
            for mo in range(2 * ls[i] + 1):
                blk[starts[i] + mo, starts[j] + mo] += dv
    return blk


def build_projectors(crystal: Crystal, basis: BasisSet, k, radial_tables) -> Projectors:
    """radial_tables: species -> (ls, form_factor(q)->array per projector, dij row-major)."""
    omega = crystal.lattice.volume()
    inv_sqrt_omega = 1.0 / math.sqrt(omega)
    g = basis.g
    q = np.asarray(k, dtype=np.float64)[None, :] + g
    qn = np.sqrt((q[:, 0] * q[:, 0] + q[:, 1] * q[:, 1]) + q[:, 2] * q[:, 2])
    lmax = 0
    for sp, (ls, _, _) in radial_tables.items():
        if ls:
            lmax = max(lmax, max(ls))
    ylm = real_sph_harmonics(q, lmax)
    ff_cache = {}
    cols, blocks, starts = [], [], [0]
    for at in crystal.atoms:
        ls, ffun, dij = radial_tables[at.symbol]
        if at.symbol not in ff_cache:
            # F_i(|k+G|) on the distinct |k+G| only (bit-identical: same inputs)
            ff_cache[at.symbol] = [_per_unique(qn, lambda u, i=i: ffun(i, u)) for i in range(len(ls))]
        ffs = ff_cache[at.symbol]
        tau = at.cart(crystal.lattice)
        phase_arg = -((g[:, 0] * tau[0] + g[:, 1] * tau[1]) + g[:, 2] * tau[2])
        phase = np.cos(phase_arg) + 1j * np.sin(phase_arg)
        for ip, l in enumerate(ls):
            scale = inv_sqrt_omega * ffs[ip]
            for mo in range(2 * l + 1):
                cols.append(phase * (scale * ylm[:, l * l + mo]))
        blk = _atom_d_block(ls, dij)
        blocks.append(blk)
        starts.append(starts[-1] + blk.shape[0])
    b = np.stack(cols, axis=1) if cols else np.zeros((len(basis), 0), dtype=np.complex128)
    return Projectors(np.asfortranarray(b), blocks, np.array(starts, dtype=np.int32))


def projector_layout(crystal: Crystal, radial_tables) -> Projectors:
    """D blocks and channel starts of the projectors, without B (b = None):
    the device builds B from the radial data (pwgpu_system radial fields)."""
    blocks, starts = [], [0]
    for at in crystal.atoms:
        ls, _, dij = radial_tables[at.symbol]
        blk = _atom_d_block(ls, dij)
        blocks.append(blk)
        starts.append(starts[-1] + blk.shape[0])
    return Projectors(None, blocks, np.array(starts, dtype=np.int32))


def upf_radial_table(pp: Upf):
    return (list(pp.beta_l), lambda i, q, pp=pp: beta_form_factor(pp, i, q), np.asarray(pp.dij))


def ewald_energy(crystal: Crystal, charges) -> float:
    """Ion-ion Ewald sum in eV (ewald.rs:43-200), η = (N_at π/Ω)^{1/3}."""
    from scipy.special import erfc
    lat = crystal.lattice
    omega = lat.volume()
    pos = np.array([a.cart(lat) for a in crystal.atoms])
    z = np.asarray(charges, dtype=np.float64)
    nat = len(z)
    eta = (nat * math.pi / omega) ** (1.0 / 3.0)
    eta2 = eta * eta
    rec = lat.reciprocal()
    gmax = 10.0 * eta
    nm = [int(math.ceil(gmax / np.linalg.norm(v))) for v in (rec.a, rec.b, rec.c)]
    r1 = np.arange(-nm[0], nm[0] + 1); r2 = np.arange(-nm[1], nm[1] + 1); r3 = np.arange(-nm[2], nm[2] + 1)
    a1, a2, a3 = np.meshgrid(r1, r2, r3, indexing="ij")
    a1 = a1.ravel(); a2 = a2.ravel(); a3 = a3.ravel()
    keep = ~((a1 == 0) & (a2 == 0) & (a3 == 0))
    a1, a2, a3 = a1[keep], a2[keep], a3[keep]
    gv = np.outer(a1, rec.a) + np.outer(a2, rec.b) + np.outer(a3, rec.c)
    g2 = np.einsum("ij,ij->i", gv, gv)
    ok = g2 >= 1e-12
    gv, g2 = gv[ok], g2[ok]
    s = (np.exp(1j * (gv @ pos.T)) * z[None, :]).sum(axis=1)
    e_rec = float(np.sum(np.abs(s) ** 2 * np.exp(-g2 / (4.0 * eta2)) / g2)) * 2.0 * math.pi * E2_COULOMB / omega
    rmax = 10.0 / eta
    lm = [int(math.ceil(rmax / np.linalg.norm(v))) for v in (lat.a, lat.b, lat.c)]
    e_real = 0.0
    for l1 in range(-lm[0], lm[0] + 1):
        for l2 in range(-lm[1], lm[1] + 1):
            for l3 in range(-lm[2], lm[2] + 1):
                t = l1 * lat.a + l2 * lat.b + l3 * lat.c
                d = pos[:, None, :] - pos[None, :, :] + t[None, None, :]
                rn = np.sqrt(np.einsum("ijk,ijk->ij", d, d))
                m = rn >= 1e-10
                e_real += float(np.sum((z[:, None] * z[None, :])[m] * erfc(eta * rn[m]) / rn[m]))
    e_real *= 0.5 * E2_COULOMB
    e_self = -eta / math.sqrt(math.pi) * float(np.sum(z * z)) * E2_COULOMB
    e_bg = -math.pi * float(np.sum(z)) ** 2 * E2_COULOMB / (2.0 * omega * eta2)
    return e_real + e_rec + e_self + e_bg


def _per_unique(values: np.ndarray, fn):
    """Evaluate fn on the distinct entries of values (exact float equality)."""
    u, inv = np.unique(values, return_inverse=True)
    return fn(u)[inv]


@dataclass
class ScfSystem:
    """Everything the GPU hot path needs, in the reference's units (eV, Å)."""
    crystal: Crystal
    basis: BasisSet
    dims: tuple
    g_to_fft: np.ndarray          # int64 (n_pw,)
    kpoints: list                 # KPoint list
    kinetic: list                 # per k: (n_pw,) eV
    projectors: list              # per k: Projectors
    v_local_g: np.ndarray         # complex (N,) eV, G=0 kept
    g_squared: np.ndarray         # (N,) Å⁻²
    rho_core_r: np.ndarray        # (N,) e/Å³ or empty
    n_electrons: float
    omega: float
    e_ewald: float
    symmetry: SymmetryInfo
    rho_init_r: np.ndarray        # SAD start density (N,)
    nspin: int = 1
    extra: dict = field(default_factory=dict)

    @property
    def n_grid(self):
        return int(np.prod(self.dims))

    @property
    def n_pw(self):
        return len(self.basis)

    @property
    def kpt_weights(self):
        return np.array([kp.weight for kp in self.kpoints])

    @property
    def spin_factor(self):
        return 2.0 / self.nspin


def build_system(crystal: Crystal, pps: dict, ecut_ev: float, kpoints, symmetry: SymmetryInfo | None = None,
                 ecutrho_ratio: int = 4, fft_grid=None, gaussian_sigma: float = 1.0, nspin: int = 1,
                 with_initial_density: bool = True, projectors_on_device: bool = False,
                 local_on_device: bool = False) -> ScfSystem:
    """ScfContext::new (context.rs:102-231) plus the SAD start density
    (initial_density.rs:64-143).  projectors_on_device: skip the host B
    (the GPU builds it from the UPF radial data at pwgpu_create).
    local_on_device: skip the host V_loc(G), core density and start density
    (v_local_g and rho_init_r are None; the GPU builds them at pwgpu_create,
    PwGpu.initial_density() returns the start density)."""
    basis = BasisSet(crystal.lattice, ecut_ev)
    dims = grid_dims_for(basis, ecutrho_ratio, fft_grid)
    omega = crystal.lattice.volume()
    nel = float(sum(pps[a.symbol].z_valence for a in crystal.atoms))
    g_to_fft = miller_to_idx(dims, basis.miller[:, 0].astype(np.int64), basis.miller[:, 1].astype(np.int64),
                             basis.miller[:, 2].astype(np.int64))
    recip = crystal.lattice.reciprocal()
    gv = grid_g_vectors(dims, recip)
    g2 = (gv[:, 0] * gv[:, 0] + gv[:, 1] * gv[:, 1]) + gv[:, 2] * gv[:, 2]
    gn = np.sqrt(g2)
    n = gv.shape[0]
    taus = [a.cart(crystal.lattice) for a in crystal.atoms]

    v_loc, rho_core_r = None, np.zeros(0)
    if not local_on_device:
        # per-species structure factors S_s(G) = sum over its atoms of e^{-iG.tau},
        # shared by the V_loc, core and start-density sums
        sfac = {}
        for at, tau in zip(crystal.atoms, taus):
            ph = -((gv[:, 0] * tau[0] + gv[:, 1] * tau[1]) + gv[:, 2] * tau[2])
            term = np.cos(ph) + 1j * np.sin(ph)
            if at.symbol in sfac:
                sfac[at.symbol] += term
            else:
                sfac[at.symbol] = term

        def structure_sum(radial_of_species):
            acc = np.zeros(n, dtype=np.complex128)
            for sp in sfac:
                rad = radial_of_species(sp)
                if rad is not None:
                    acc += sfac[sp] * rad
            return acc

        v_loc = structure_sum(lambda sp: _per_unique(gn, lambda u: v_local_of_g(pps[sp], u, omega)))

        if any(pps[s].has_nlcc() for s in crystal.species()):
            four_pi = 4.0 * math.pi

            def core_rad(sp):
                pp = pps[sp]
                if not pp.has_nlcc():
                    return None
                return _per_unique(gn, lambda u: four_pi * sinc_transform(pp, pp.core_charge, True, u) / omega)

            rho_core_g = structure_sum(core_rad)
            rho_core_r = inverse_fft_unnormalized(rho_core_g, dims).real.copy()
        else:
            rho_core_r = np.zeros(0)

    tables = {sp: upf_radial_table(pps[sp]) for sp in crystal.species()}
    kin = [basis.kinetic(kp.k) for kp in kpoints]
    if projectors_on_device:
        layout = projector_layout(crystal, tables)
        projs = [layout for _ in kpoints]
    else:
        projs = [build_projectors(crystal, basis, kp.k, tables) for kp in kpoints]
    e_ew = ewald_energy(crystal, [pps[a.symbol].z_valence for a in crystal.atoms])
    sym = symmetry if symmetry is not None else SymmetryInfo.identity_only()

    rho0 = None if local_on_device else np.zeros(0)
    if with_initial_density and not local_on_device:
        def sad_rad(sp):
            pp = pps[sp]
            if pp.has_rho_atom():
                return _per_unique(gn, lambda u: sinc_transform(pp, pp.rho_atom, False, u) / omega)
            return pp.z_valence * np.exp(-0.5 * g2 * gaussian_sigma * gaussian_sigma) / omega

        rho_g = structure_sum(sad_rad)
        rho0 = inverse_fft_unnormalized(rho_g, dims).real.copy()
        rho0[rho0 < 0.0] = 0.0
        dv = omega / n
        integ = rho0.sum() * dv
        if integ > 1e-15:
            rho0 *= nel / integ

    out = ScfSystem(crystal, basis, dims, g_to_fft, list(kpoints), kin, projs, v_loc, g2, rho_core_r, nel, omega,
                    e_ew, sym, rho0, nspin)
    out.extra["pps"] = pps
    out.extra["gaussian_sigma"] = float(gaussian_sigma)
    return out

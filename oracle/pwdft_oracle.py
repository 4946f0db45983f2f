"""ORACLE -- test infrastructure only.

CPU FP64 restatement (numpy/scipy) of the reference's per-iteration SCF
algorithm, used by tests/, __graft_entry__.smoke() and bench.py's CPU
baseline leg as the checker.  It is never part of the product path.

Each function cites the reference file:line it restates (paths relative to
pwdft/pwdft-core/src/ of Ron-Leizrowice/pwdft-rs).  The reference's own
Rust crate cannot be built here (no Rust toolchain, and the snapshot does
not compile), so parity is pinned through the reference's golden numbers:
  * SCF golden  -- tests/cpu_scf_baseline.rs:43-44 (E=-213.028339 eV,
                   E_F=8.052064 eV, Si prim, 100 eV, 16^3, Γ, 4 bands)
  * QE pins        -- tests/qe_validation.rs (Si 4x4x4 15 Ry: -231.6544 eV,
                      E_F, QE energy and one-electron sum; C diamond E_F;
                      Al FCC energy, E_F and one-electron sum; Fe Ewald)
  * component CSVs -- data/csv/{vloc_g,beta_q,dij,rho_core_g}_si_reference.csv,
                      the heavy-atom data/csv/vgch_{beta_l,vloc}_heavy.csv
  * per-component energies -- tests/vgc5_per_component_si.rs
  * basis counts   -- basis.rs:139-148 (259 G at 200 eV)
Third-party numerics: rustfft 6.4.1 (restated by numpy.fft, same sign and
normalisation conventions), faer 0.24 self_adjoint_eigen (restated by
LAPACK zheevr via scipy.linalg.eigh), puruspe 0.4.4 erf/erfc (scipy.special).
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np
import scipy.fft as sfft
import scipy.linalg as sla
from scipy.special import erfc

HA_TO_EV = 27.211386245988
BOHR_TO_ANG = 0.529177210903
BOHR3_TO_ANG3 = BOHR_TO_ANG ** 3
E2_COULOMB = 14.399645351950548
G2_ZERO_THRESHOLD = 1e-12
RHO_FLOOR = 1e-30

_WORKERS = -1


def set_workers(n: int):
    """Thread count for the oracle's FFTs (-1 = all cores)."""
    global _WORKERS
    _WORKERS = n


# ---------------------------------------------------------------------------
# FFT conventions (fft.rs:19-114): both directions unnormalised.
# ---------------------------------------------------------------------------

def ifft3(x, dims):
    return sfft.ifftn(x.reshape(dims), norm="forward", workers=_WORKERS).ravel()


def fft3(x, dims):
    return sfft.fftn(x.reshape(dims), workers=_WORKERS).ravel()


def density_r_to_g(rho_r, dims):
    """ρ(G) = (1/N) Σ_r ρ(r) e^{-iG·r} (energy.rs:250-259)."""
    return fft3(rho_r.astype(np.complex128), dims) / rho_r.size


# ---------------------------------------------------------------------------
# Hamiltonian (potentials.rs:163-190, nonlocal.rs:432-450)
# ---------------------------------------------------------------------------

def miller_to_idx(dims, m):
    d0, d1, d2 = dims
    return (np.mod(m[..., 0], d0) * d1 + np.mod(m[..., 1], d1)) * d2 + np.mod(m[..., 2], d2)


def dense_hamiltonian(miller, kinetic, veff_g, dims, b, d_dense):
    """H[i,j] = V_eff(G_i−G_j) + δ_ij T_i, then H += B·(D·B^H).

    fill_hamiltonian_with_v_eff (potentials.rs:163-190) followed by
    NonlocalPotential::add_to_hamiltonian (nonlocal.rs:432-450)."""
    m = miller.astype(np.int64)
    dm = m[:, None, :] - m[None, :, :]
    h = veff_g[miller_to_idx(dims, dm)].astype(np.complex128)
    h[np.diag_indices_from(h)] += kinetic
    if b.shape[1]:
        h += b @ (d_dense @ b.conj().T)
    return h


def apply_h_fft(g_to_fft, kinetic, veff_g, dims, b, d_dense, psi):
    """H·ψ by the FFT form, identical to the dense form of potentials.rs:163-190:
    (Vψ)(G_i) = (1/N) Σ_r e^{-iG_i·r} V(r) ψ(r), V(r) and ψ(r) unnormalised
    inverse transforms; plus the nonlocal B·(D·(B^H ψ))."""
    n = int(np.prod(dims))
    vr = ifft3(veff_g, dims)
    out = np.empty_like(psi)
    for j in range(psi.shape[1]):
        grid = np.zeros(n, dtype=np.complex128)
        grid[g_to_fft] = psi[:, j]
        pr = ifft3(grid, dims)
        hg = fft3(pr * vr, dims) / n
        out[:, j] = hg[g_to_fft] + kinetic * psi[:, j]
    if b.shape[1]:
        out += b @ (d_dense @ (b.conj().T @ psi))
    return out


def lowest_eigenpairs(h, n_bands):
    """Lowest n_bands eigenpairs, ascending (eigensolver/dense.rs:50-98: the
    full self_adjoint_eigen, then the first n_bands columns).  LAPACK's
    subset driver (zheevr) returns the same pairs to rounding at a fifth of
    the cost of the full decomposition."""
    n_bands = min(n_bands, h.shape[0])
    w, v = sla.eigh(h, subset_by_index=[0, n_bands - 1], driver="evr", check_finite=False)
    return w.copy(), v.copy()


# ---------------------------------------------------------------------------
# Occupations (smearing.rs:38-252)
# ---------------------------------------------------------------------------

def _step(e, ef):
    return np.where(e < ef, 1.0, np.where(np.abs(e - ef) < 1e-12, 0.5, 0.0))


def occupation01(scheme, e, ef, sigma):
    e = np.asarray(e, dtype=np.float64)
    if sigma < 1e-15:
        return _step(e, ef)
    x = (e - ef) / sigma
    if scheme in ("fermi_dirac", "fixed"):
        with np.errstate(over="ignore"):
            v = 1.0 / (1.0 + np.exp(np.clip(x, -40.0, 40.0)))
        return np.where(x > 40.0, 0.0, np.where(x < -40.0, 1.0, v))
    if scheme == "gaussian":
        return erfc(x) / 2.0
    if scheme == "methfessel_paxton":
        return erfc(x) / 2.0 - 0.5 * x * np.exp(-x * x) / math.sqrt(math.pi)
    if scheme == "cold":
        a = x + 1.0 / math.sqrt(2.0)
        return 0.5 * erfc(a) + np.exp(-a * a) / math.sqrt(2.0 * math.pi)
    raise ValueError(scheme)


def find_fermi_energy(evals, weights, n_el, sigma, scheme, spin_factor):
    """Bisection, ≤200 steps, stop at 1e-14 (smearing.rs:49-90)."""
    flat = np.concatenate([np.asarray(e) for e in evals])
    wk = np.concatenate([np.full(len(e), w) for e, w in zip(evals, weights)])
    lo = flat.min() - 10.0 * max(sigma, 0.1)
    hi = flat.max() + 10.0 * max(sigma, 0.1)
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        n = float(np.sum(wk * occupation01(scheme, flat, mid, sigma) * spin_factor))
        if n < n_el:
            lo = mid
        else:
            hi = mid
        if abs(hi - lo) < 1e-14:
            break
    return 0.5 * (lo + hi)


def entropy_ts(evals, weights, ef, sigma, scheme, spin_factor):
    """T·S (smearing.rs:202-252)."""
    if sigma < 1e-15:
        return 0.0
    s = 0.0
    for e, w in zip(evals, weights):
        x = (np.asarray(e) - ef) / sigma
        if scheme in ("fermi_dirac", "fixed"):
            f = 1.0 / (1.0 + np.exp(np.clip(x, -700, 700)))
            f = np.clip(f, 1e-30, 1.0 - 1e-30)
            with np.errstate(divide="ignore", invalid="ignore"):
                sw = np.where(np.abs(x) > 30.0, 0.0, -(f * np.log(f) + (1.0 - f) * np.log(1.0 - f)))
        elif scheme == "gaussian":
            sw = np.exp(-x * x) / math.sqrt(math.pi)
        elif scheme == "methfessel_paxton":
            sw = (0.5 - x * x) * np.exp(-x * x) / math.sqrt(math.pi)
        else:
            a = x + 1.0 / math.sqrt(2.0)
            sw = a * np.exp(-a * a) / math.sqrt(math.pi)
        s += w * float(np.sum(sw))
    return s * sigma * spin_factor


# ---------------------------------------------------------------------------
# Density (density.rs:41-111)
# ---------------------------------------------------------------------------

def compute_density(g_to_fft, dims, psis, occs, weights, n_el, omega):
    n = int(np.prod(dims))
    rho = np.zeros(n)
    for psi, occ, w in zip(psis, occs, weights):
        for ib in range(len(occ)):
            f = occ[ib] * w
            if f < 1e-15:
                continue
            grid = np.zeros(n, dtype=np.complex128)
            grid[g_to_fft] = psi[:, ib]
            pr = ifft3(grid, dims)
            rho += f * (pr.real * pr.real + pr.imag * pr.imag)
    integ = rho.sum() * (omega / n)
    if abs(integ) > 1e-15:
        rho *= n_el / integ
    return rho


def gather_map(dims, ops):
    """Source index ρ(R^T n mod N) and phase argument 2π n·τ per op and grid
    point (g_space.rs:21-91 rotate_miller/miller_to_flat/flat_to_miller)."""
    d0, d1, d2 = dims
    ax = [np.where(np.arange(d) > d // 2, np.arange(d) - d, np.arange(d)) for d in dims]
    n1, n2, n3 = [a.ravel() for a in np.meshgrid(*ax, indexing="ij")]
    srcs, args = [], []
    for rot, tau in ops:
        s = [rot[0][i] * n1 + rot[1][i] * n2 + rot[2][i] * n3 for i in range(3)]
        srcs.append(((np.mod(s[0], d0) * d1 + np.mod(s[1], d1)) * d2 + np.mod(s[2], d2)).astype(np.int32))
        args.append(2.0 * math.pi * ((n1 * tau[0] + n2 * tau[1]) + n3 * tau[2]))
    return np.stack(srcs), np.stack(args)


def symmetrize_density(rho_r, dims, src, arg):
    """G-space symmetrisation (symmetry/density/g_space.rs:147-252).

    src/arg: gather map [n_ops, N] (source flat index, 2π n·τ)."""
    n_ops = src.shape[0]
    if n_ops <= 1:
        return rho_r.copy()
    rg = fft3(rho_r.astype(np.complex128), dims)
    acc = np.zeros(rg.size, dtype=np.complex128)
    for s in range(n_ops):
        acc += (np.cos(arg[s]) - 1j * np.sin(arg[s])) * rg[src[s]]
    acc *= 1.0 / n_ops
    return (ifft3(acc, dims) / rg.size).real.copy()


def symmetrize_real_space(rho_r, dims, symmetry):
    """Real-space symmetrisation on the grid points, the reference's test
    helper `symmetrize_real_ref` (symmetry/density/g_space.rs:278-323):
    rho_sym(r) = (1/N_ops) sum_S rho(S^-1 r), S^-1 = (R^-1, -R^-1 tau) on
    fractional coordinates, each image rounded to its nearest grid point.
    Equal to the G-space form only where every image lands on a grid point
    (Si Fd-3m: grid sizes divisible by 4)."""
    d = np.array(dims, dtype=np.int64)
    idx = np.indices(tuple(dims)).reshape(3, -1).T.astype(np.float64)
    f = idx / d
    out = np.zeros(rho_r.size)
    for op in symmetry.operations:
        rinv = np.rint(np.linalg.inv(np.array(op.rotation, dtype=np.float64)))
        tinv = -rinv @ np.array(op.translation, dtype=np.float64)
        j = np.rint((f @ rinv.T + tinv) * d).astype(np.int64) % d
        out += rho_r[(j[:, 0] * d[1] + j[:, 1]) * d[2] + j[:, 2]]
    return out / symmetry.n_ops


# ---------------------------------------------------------------------------
# Potentials and XC (energy.rs:293-358, xc.rs:129-596)
# ---------------------------------------------------------------------------

def hartree(rho_g, g2):
    fpe = 4.0 * math.pi * E2_COULOMB
    out = np.zeros_like(rho_g)
    m = g2 > G2_ZERO_THRESHOLD
    out[m] = rho_g[m] * fpe / g2[m]
    return out


def hartree_energy(rho_g, g2, omega):
    fpe = 4.0 * math.pi * E2_COULOMB
    m = g2 > G2_ZERO_THRESHOLD
    return float(np.sum((rho_g[m].real ** 2 + rho_g[m].imag ** 2) * fpe / g2[m])) * 0.5 * omega


def _pz_rs(rs, polarized):
    if polarized:
        g, b1, b2 = -0.0843, 1.3981, 0.2611
        a, b, c, d = 0.01555, -0.0269, 0.0007, -0.0048
    else:
        g, b1, b2 = -0.1423, 1.0529, 0.3334
        a, b, c, d = 0.0311, -0.048, 0.0020, -0.0116
    rs = np.asarray(rs)
    hi = rs >= 1.0
    sq = np.sqrt(np.where(hi, rs, 1.0))
    den = 1.0 + b1 * sq + b2 * rs
    ec_h = g / den
    dec_h = -g * (b1 / (2.0 * sq) + b2) / (den * den)
    vc_h = ec_h - rs / 3.0 * dec_h
    lr = np.log(np.where(hi, 1.0, rs))
    ec_l = a * lr + b + c * rs * lr + d * rs
    dec_l = a / np.where(hi, 1.0, rs) + c * (lr + 1.0) + d
    vc_l = ec_l - rs / 3.0 * dec_l
    return np.where(hi, ec_h, ec_l), np.where(hi, vc_h, vc_l)


def lda_xc(rho):
    """PZ81 LDA: (ε_xc, v_xc) in eV for ρ in e/Å³ (xc.rs:129-288)."""
    rho = np.asarray(rho, dtype=np.float64)
    ok = rho >= RHO_FLOOR
    rb = np.where(ok, rho, 1.0) * BOHR3_TO_ANG3
    ex = -0.75 * np.cbrt(3.0 * rb / math.pi)
    vx = (4.0 / 3.0) * ex
    rs = np.cbrt(3.0 / (4.0 * math.pi * rb))
    ec, vc = _pz_rs(rs, False)
    exc = np.where(ok, (ex + ec) * HA_TO_EV, 0.0)
    vxc = np.where(ok, (vx + vc) * HA_TO_EV, 0.0)
    return exc, vxc


def lsda_xc(rho_up, rho_dn):
    """LSDA: Slater spin scaling + PZ von Barth-Hedin interpolation (xc.rs:374-596)."""
    ru = np.asarray(rho_up, dtype=np.float64)
    rd = np.asarray(rho_dn, dtype=np.float64)
    rho = ru + rd
    ok = rho >= RHO_FLOOR
    rhs = np.where(ok, rho, 1.0)
    rub, rdb = ru * BOHR3_TO_ANG3, rd * BOHR3_TO_ANG3
    exu = np.where(rub > RHO_FLOOR, -0.75 * np.cbrt(6.0 * np.maximum(rub, 0) / math.pi), 0.0)
    exd = np.where(rdb > RHO_FLOOR, -0.75 * np.cbrt(6.0 * np.maximum(rdb, 0) / math.pi), 0.0)
    rb = rhs * BOHR3_TO_ANG3
    ex = (rub * exu + rdb * exd) / rb
    vxu, vxd = (4.0 / 3.0) * exu, (4.0 / 3.0) * exd
    rs = np.cbrt(3.0 / (4.0 * math.pi * rb))
    zeta = np.clip((ru - rd) / rhs, -1.0, 1.0)
    ecu, vcu = _pz_rs(rs, False)
    ecp, vcp = _pz_rs(rs, True)
    fden = 2.0 * np.cbrt(2.0) - 2.0
    op, om = np.maximum(1.0 + zeta, 0.0), np.maximum(1.0 - zeta, 0.0)
    cop, com = np.cbrt(op), np.cbrt(om)
    fz = (cop * op + com * om - 2.0) / fden
    dfz = (4.0 / 3.0) * (cop - com) / fden
    ec = ecu + fz * (ecp - ecu)
    vrs = vcu + fz * (vcp - vcu)
    dz = dfz * (ecp - ecu)
    vcu_ = vrs + (1.0 - zeta) * dz
    vcd_ = vrs - (1.0 + zeta) * dz
    z = lambda x: np.where(ok, x * HA_TO_EV, 0.0)
    return z(ex + ec), z(vxu + vcu_), z(vxd + vcd_)


def add_core(rho, rho_core):
    if rho_core.size == 0:
        return rho.copy()
    return np.maximum(rho + rho_core, 0.0)


def xc_energy_corrected(rho_xc, rho_val, exc, vxc, omega):
    dv = omega / rho_xc.size
    return float(np.sum(rho_xc * exc * dv)) - float(np.sum(rho_val * vxc * dv))


def kinetic_expectation(kinetic, psis, occs, weights):
    """Σ_k w_k Σ_b f_b Σ_G |c_b(G)|² (ħ²/2m)|k+G|² (kinetic_expectation, energy.rs:382-421)."""
    e = 0.0
    for kin, v, o, w in zip(kinetic, psis, occs, weights):
        t = np.sum(np.abs(v) ** 2 * kin[:, None], axis=0)
        e += w * float(np.sum(np.where(o == 0.0, 0.0, o * t)))
    return e


def nonlocal_expectation(bs, d_dense, psis, occs, weights):
    """Σ_k w_k Σ_b f_b Re ψ_b^H H_NL ψ_b with the dense H_NL = B D B^H of each k
    (nonlocal_expectation, energy.rs:467-516)."""
    e = 0.0
    for b, d, v, o, w in zip(bs, d_dense, psis, occs, weights):
        if b.shape[1] == 0:
            continue
        h_nl = b @ (d @ b.conj().T)
        t = np.real(np.sum(v.conj() * (h_nl @ v), axis=0))
        e += w * float(np.sum(np.where(o == 0.0, 0.0, o * t)))
    return e


def local_pp_energy(rho_r, v_local_g, dims, omega):
    """∫ρ V_loc dV with V_loc(r) the unnormalised inverse FFT of V_loc(G), G = 0
    kept (driver.rs:664-668, local_pp_energy_grid energy.rs:439-445)."""
    v_r = ifft3(v_local_g, dims).real
    return float(np.sum(rho_r * v_r)) * omega / rho_r.size


def density_diff(a, b, omega):
    n = a.size
    dv = omega / n
    return math.sqrt(float(np.sum((a - b) ** 2 * dv)) / omega)


# ---------------------------------------------------------------------------
# Mixing (mixing/anderson.rs:170-266, kerker.rs:18-49, linalg.rs:24-50)
# ---------------------------------------------------------------------------

def auto_q_tf_squared(n_el, omega):
    rho_b = n_el / omega * BOHR_TO_ANG ** 3
    q2 = 4.0 * np.cbrt(3.0 * math.pi * math.pi * rho_b) / math.pi
    return q2 / (BOHR_TO_ANG * BOHR_TO_ANG)


class AndersonMixer:
    def __init__(self, beta, ndim, dims, kerker_weights=None):
        self.beta, self.ndim, self.dims = beta, ndim, dims
        self.kw = kerker_weights
        self.hin, self.hres = [], []

    def mix(self, rho_in, rho_out):
        res = rho_out - rho_in
        if self.kw is not None:
            rg = fft3(res.astype(np.complex128), self.dims) * self.kw
            res = (ifft3(rg, self.dims) / res.size).real.copy()
        self.hin.append(rho_in.copy())
        self.hres.append(res)
        if len(self.hin) > self.ndim:
            self.hin.pop(0)
            self.hres.pop(0)
        m = len(self.hin)
        if m < 2:
            return self.hin[-1] + self.beta * self.hres[-1]
        rl = self.hres[-1]
        dr = [self.hres[i] - rl for i in range(m - 1)]
        mm = m - 1
        a = np.array([[float(dr[i] @ dr[j]) for j in range(mm)] for i in range(mm)])
        b = np.array([-float(dr[i] @ rl) for i in range(mm)])
        alpha = solve_small(a, b)
        al = 1.0 - alpha.sum()
        out = al * (self.hin[-1] + self.beta * rl)
        for i in range(mm):
            out = out + alpha[i] * (self.hin[i] + self.beta * self.hres[i])
        return out


class BroydenMixer:
    """Modified Broyden (mixing/broyden.rs:26-258): history of input and
    residual differences, gamma = <df_i|df_j>^-1 <df_i|R>,
    rho_new = (rho_in - sum gamma dv) + beta (R - sum gamma df)."""

    def __init__(self, beta, ndim, dims, kerker_weights=None):
        self.beta, self.ndim, self.dims = beta, ndim, dims
        self.kw = kerker_weights
        self.dv, self.df = [], []
        self.prev_in = self.prev_res = None

    def mix(self, rho_in, rho_out):
        res = rho_out - rho_in
        if self.kw is not None:
            rg = fft3(res.astype(np.complex128), self.dims) * self.kw
            res = (ifft3(rg, self.dims) / res.size).real.copy()
        if self.prev_in is not None:
            self.dv.append(rho_in - self.prev_in)
            self.df.append(res - self.prev_res)
            if len(self.dv) > self.ndim:
                self.dv.pop(0)
                self.df.pop(0)
        self.prev_in, self.prev_res = rho_in.copy(), res.copy()
        m = len(self.df)
        if m == 0:
            return rho_in + self.beta * res
        a = np.array([[float(self.df[i] @ self.df[j]) for j in range(m)] for i in range(m)])
        w = np.array([float(self.df[i] @ res) for i in range(m)])
        g = solve_small(a, w)
        cdv = sum(g[i] * self.dv[i] for i in range(m))
        cdf = sum(g[i] * self.df[i] for i in range(m))
        return (rho_in - cdv) + self.beta * (res - cdf)


class PeriodicPulayMixer(AndersonMixer):
    """Periodic Pulay (mixing/anderson.rs:294-386): Anderson history every
    step, a DIIS step every `period`-th step (history >= 2), linear mixing
    of the last entry otherwise."""

    def __init__(self, beta, ndim, dims, period=3, kerker_weights=None):
        super().__init__(beta, ndim, dims, kerker_weights)
        self.period, self.iteration = period, 0

    def mix(self, rho_in, rho_out):
        self.iteration += 1
        if self.iteration % self.period == 0:
            return super().mix(rho_in, rho_out)  # linear while the history is shorter than 2
        res = rho_out - rho_in
        if self.kw is not None:
            rg = fft3(res.astype(np.complex128), self.dims) * self.kw
            res = (ifft3(rg, self.dims) / res.size).real.copy()
        self.hin.append(rho_in.copy())
        self.hres.append(res)
        if len(self.hin) > self.ndim:
            self.hin.pop(0)
            self.hres.pop(0)
        return self.hin[-1] + self.beta * self.hres[-1]


def make_mixer(kind, beta, ndim, dims, kerker_weights=None, period=3):
    """Mixer::new (mixing/mod.rs:245-276): 'anderson' (Plain / Kerker),
    'broyden', 'periodic_pulay'."""
    if kind == "anderson":
        return AndersonMixer(beta, ndim, dims, kerker_weights)
    if kind == "broyden":
        return BroydenMixer(beta, ndim, dims, kerker_weights)
    if kind == "periodic_pulay":
        return PeriodicPulayMixer(beta, ndim, dims, period, kerker_weights)
    raise ValueError(kind)


def solve_small(a, b):
    """Partial-pivot LU with the 1e-15 singular-pivot fallback (linalg.rs:24-50)."""
    import scipy.linalg as sl
    n = b.size
    if n == 0:
        return b
    lu, piv = sl.lu_factor(a, check_finite=False)
    if np.any(np.abs(np.diag(lu)) < 1e-15):
        return np.full(n, 1.0 / (n + 1))
    return sl.lu_solve((lu, piv), b, check_finite=False)


# ---------------------------------------------------------------------------
# SCF driver (driver.rs:266-742)
# ---------------------------------------------------------------------------

@dataclass
class OracleResult:
    total_energy: float
    harris_foulkes_energy: float
    fermi_energy: float
    eigenvalues: list
    n_iterations: int
    final_delta: float
    rho_r: np.ndarray
    entropy_ts: float = 0.0
    history: list = field(default_factory=list)
    components: dict = None    # EnergyComponents (energy.rs:597-670) of the final iteration


def diag_k_task(args):
    """Dense H of one k-point and its lowest eigenpairs (the per-k body of
    driver.rs:459-472); a top-level function so that a process pool can run
    the k-points in parallel, as the reference's rayon loop does."""
    miller, kinetic, veff, dims, b, d_dense, n_bands = args
    return lowest_eigenpairs(dense_hamiltonian(miller, kinetic, veff, dims, b, d_dense), n_bands)


def run_scf_unpolarized(sys, n_bands, max_iter=100, conv_threshold=1e-6, energy_threshold=1e-5,
                        mixing_beta=0.3, mixing_ndim=8, smearing="fermi_dirac", sigma=0.01,
                        kerker=False, q_tf=None, verbose=False, mixer="anderson", mixing_period=3, kmap=map):
    """Dense-H SCF loop of driver.rs:353-735 on an ScfSystem (pwgpu.context).
    kmap: map over the per-k diagonalisations (e.g. a process pool's map)."""
    dims = sys.dims
    n = sys.n_grid
    omega = sys.omega
    weights = sys.kpt_weights
    spin_factor = 2.0
    if sys.symmetry.n_ops > 1:
        src, arg = gather_map(dims, [(op.rotation, op.translation) for op in sys.symmetry.operations])
    else:
        src = arg = np.zeros((1, 0))
    kw = None
    if kerker:
        # Broyden and Periodic Pulay always estimate q_TF (mixing/mod.rs:254-275)
        user_q = q_tf is not None and mixer == "anderson"
        q2 = q_tf * q_tf if user_q else auto_q_tf_squared(sys.n_electrons, omega)
        kw = np.where(sys.g_squared < G2_ZERO_THRESHOLD, 0.0, sys.g_squared / (sys.g_squared + q2))
    mixer = make_mixer(mixer, mixing_beta, mixing_ndim, dims, kw, mixing_period)
    d_dense = [p.d_dense() for p in sys.projectors]
    rho = sys.rho_init_r.copy()
    rho_g = density_r_to_g(rho, dims)
    e_prev = None
    hist = []
    for it in range(max_iter):
        vh = hartree(rho_g, sys.g_squared)
        rxc = add_core(rho, sys.rho_core_r)
        exc_in, vxc_in = lda_xc(rxc)
        veff = sys.v_local_g + vh + density_r_to_g(vxc_in, dims)
        evals, psis = [], []
        tasks = [(sys.basis.miller, sys.kinetic[ik], veff, dims, sys.projectors[ik].b, d_dense[ik], n_bands)
                 for ik in range(len(sys.kpoints))]
        for w, v in kmap(diag_k_task, tasks):
            evals.append(w)
            psis.append(v)
        ef = find_fermi_energy(evals, weights, sys.n_electrons, sigma, smearing, spin_factor)
        occs = [spin_factor * occupation01(smearing, e, ef, sigma) for e in evals]
        rho_new = compute_density(sys.g_to_fft, dims, psis, occs, weights, sys.n_electrons, omega)
        if src.shape[0] > 1:
            rho_new = symmetrize_density(rho_new, dims, src, arg)
        delta = density_diff(rho, rho_new, omega)
        rho_g_new = density_r_to_g(rho_new, dims)
        rxc_new = add_core(rho_new, sys.rho_core_r)
        exc_o, vxc_o = lda_xc(rxc_new)
        e_band = float(sum(np.sum(o * w * e) for o, w, e in zip(occs, weights, evals)))
        ts = entropy_ts(evals, weights, ef, sigma, smearing, spin_factor)
        e_tot = (e_band - hartree_energy(rho_g_new, sys.g_squared, omega)
                 + xc_energy_corrected(rxc_new, rho_new, exc_o, vxc_o, omega) + sys.e_ewald - ts)
        e_hf = (e_band - hartree_energy(rho_g, sys.g_squared, omega)
                + xc_energy_corrected(rxc, rho, exc_in, vxc_in, omega) + sys.e_ewald - ts)
        de = None if e_prev is None else abs(e_tot - e_prev)
        e_prev = e_tot
        hist.append((it, e_tot, delta))
        if verbose:
            print(f"iter {it:3d} E={e_tot:.10f} dE={de} drho={delta:.3e}")
        if delta < conv_threshold and de is not None and de < energy_threshold:
            dv = omega / n
            comp = dict(e_band=e_band,
                        e_kinetic=kinetic_expectation(sys.kinetic, psis, occs, weights),
                        e_local=local_pp_energy(rho_new, sys.v_local_g, dims, omega),
                        e_nonlocal=nonlocal_expectation([p.b for p in sys.projectors], d_dense, psis, occs, weights),
                        e_hartree=hartree_energy(rho_g_new, sys.g_squared, omega),
                        e_xc=float(np.sum(rxc_new * exc_o * dv)), e_vxc=float(np.sum(rho_new * vxc_o * dv)),
                        e_ewald=sys.e_ewald, e_smearing=-ts)
            return OracleResult(e_tot, e_hf, ef, evals, it + 1, delta, rho_new, ts, hist, comp)
        rho = mixer.mix(rho, rho_new)
        rho_g = density_r_to_g(rho, dims)
    raise RuntimeError(f"SCF did not converge in {max_iter} iterations (delta={delta})")


def fixed_point_check(sys, rho_r, psi, smearing, sigma, ik=0):
    """The oracle's view of a converged unpolarised single-k state computed
    elsewhere (a checker for cells too large for the dense loop):
    V_eff = V_loc + V_H + V_xc from rho_r (energy.rs:293-358), the
    FFT-form H of the reference's operator applied to the bands psi
    (n_pw x nb, potentials.rs:163-190 + nonlocal.rs:432-450), their
    Rayleigh quotients and residual norms, occupations and Fermi level from
    the quotients (smearing.rs:38-252), the density of the bands
    (density.rs:41-111) and the total energy of driver.rs:637-700 built
    from those oracle quantities alone.  Returns a dict of arrays and
    scalars (eV, e/Å³)."""
    dims = sys.dims
    p = sys.projectors[ik]
    rho_g = density_r_to_g(rho_r, dims)
    rxc = add_core(rho_r, sys.rho_core_r)
    _, vxc = lda_xc(rxc)
    veff = sys.v_local_g + hartree(rho_g, sys.g_squared) + density_r_to_g(vxc, dims)
    psi = np.asarray(psi, dtype=np.complex128)
    norms = np.linalg.norm(psi, axis=0)
    hpsi = apply_h_fft(sys.g_to_fft, sys.kinetic[ik], veff, dims, p.b, p.d_dense(), psi)
    rq = np.real(np.einsum("ij,ij->j", psi.conj(), hpsi)) / norms ** 2
    res = np.linalg.norm(hpsi - psi * rq, axis=0) / norms
    ef = find_fermi_energy([rq], [1.0], sys.n_electrons, sigma, smearing, 2.0)
    occ = 2.0 * occupation01(smearing, rq, ef, sigma)
    rho_out = compute_density(sys.g_to_fft, dims, [psi / norms], [occ], [1.0], sys.n_electrons, sys.omega)
    rho_out_g = density_r_to_g(rho_out, dims)
    rxc_o = add_core(rho_out, sys.rho_core_r)
    exc_o, vxc_o = lda_xc(rxc_o)
    ts = entropy_ts([rq], [1.0], ef, sigma, smearing, 2.0)
    e_band = float(np.sum(occ * rq))
    e_tot = (e_band - hartree_energy(rho_out_g, sys.g_squared, sys.omega)
             + xc_energy_corrected(rxc_o, rho_out, exc_o, vxc_o, sys.omega) + sys.e_ewald - ts)
    return {"rayleigh": rq, "residual": res, "fermi_energy": ef, "rho_out": rho_out, "total_energy": e_tot,
            "drho_in_out": density_diff(rho_r, rho_out, sys.omega)}


@dataclass
class OracleIter1Result:
    total_energy: float
    harris_foulkes_energy: float
    fermi_energy: float
    entropy_ts: float
    eigenvalues: list
    components: dict
    rho_r_out: np.ndarray
    rho_g_out: np.ndarray
    rho_r_in: np.ndarray
    delta_rho: float


def run_scf_iter1_from_rho_g(sys, n_bands, rho_g_fft, smearing="fermi_dirac", sigma=0.01):
    """One SCF iteration from a transplanted full-grid rho(G)
    (run_scf_iter1_from_rho_g_fft, scf/transplant.rs:114-376): rho_in(r) =
    Re N·IFFT(rho_g), rho(G) re-derived from it, then the first iteration of
    the unpolarised driver with cold dense diagonalisation; energies and
    components on the output density."""
    dims = sys.dims
    n = sys.n_grid
    omega = sys.omega
    weights = sys.kpt_weights
    spin_factor = 2.0
    if len(rho_g_fft) != n:
        raise ValueError(f"transplanted rho_g_fft has {len(rho_g_fft)} entries; expected n_grid={n}")
    rho = ifft3(np.asarray(rho_g_fft, dtype=np.complex128), dims).real.copy()
    rho_g = density_r_to_g(rho, dims)
    vh = hartree(rho_g, sys.g_squared)
    rxc = add_core(rho, sys.rho_core_r)
    exc_in, vxc_in = lda_xc(rxc)
    veff = sys.v_local_g + vh + density_r_to_g(vxc_in, dims)
    d_dense = [p.d_dense() for p in sys.projectors]
    evals, psis = [], []
    for ik in range(len(sys.kpoints)):
        h = dense_hamiltonian(sys.basis.miller, sys.kinetic[ik], veff, dims, sys.projectors[ik].b, d_dense[ik])
        w, v = lowest_eigenpairs(h, n_bands)
        evals.append(w)
        psis.append(v)
    ef = find_fermi_energy(evals, weights, sys.n_electrons, sigma, smearing, spin_factor)
    occs = [spin_factor * occupation01(smearing, e, ef, sigma) for e in evals]
    rho_new = compute_density(sys.g_to_fft, dims, psis, occs, weights, sys.n_electrons, omega)
    if sys.symmetry.n_ops > 1:
        src, arg = gather_map(dims, [(op.rotation, op.translation) for op in sys.symmetry.operations])
        rho_new = symmetrize_density(rho_new, dims, src, arg)
    delta = density_diff(rho, rho_new, omega)
    rho_g_new = density_r_to_g(rho_new, dims)
    rxc_new = add_core(rho_new, sys.rho_core_r)
    exc_o, vxc_o = lda_xc(rxc_new)
    e_band = float(sum(np.sum(o * w * e) for o, w, e in zip(occs, weights, evals)))
    ts = entropy_ts(evals, weights, ef, sigma, smearing, spin_factor)
    e_tot = (e_band - hartree_energy(rho_g_new, sys.g_squared, omega)
             + xc_energy_corrected(rxc_new, rho_new, exc_o, vxc_o, omega) + sys.e_ewald - ts)
    e_hf = (e_band - hartree_energy(rho_g, sys.g_squared, omega)
            + xc_energy_corrected(rxc, rho, exc_in, vxc_in, omega) + sys.e_ewald - ts)
    dv = omega / n
    comp = dict(e_band=e_band,
                e_kinetic=kinetic_expectation(sys.kinetic, psis, occs, weights),
                e_local=local_pp_energy(rho_new, sys.v_local_g, dims, omega),
                e_nonlocal=nonlocal_expectation([p.b for p in sys.projectors], d_dense, psis, occs, weights),
                e_hartree=hartree_energy(rho_g_new, sys.g_squared, omega),
                e_xc=float(np.sum(rxc_new * exc_o * dv)), e_vxc=float(np.sum(rho_new * vxc_o * dv)),
                e_ewald=sys.e_ewald, e_smearing=-ts)
    return OracleIter1Result(e_tot, e_hf, ef, ts, evals, comp, rho_new, rho_g_new, rho, delta)


# ---------------------------------------------------------------------------
# Spin-polarised SCF driver (driver_spin.rs:114-839)
# ---------------------------------------------------------------------------

@dataclass
class OracleSpinResult:
    total_energy: float
    harris_foulkes_energy: float
    fermi_energy: float
    eigenvalues: list          # [up k0..k_{n-1}, down k0..k_{n-1}]
    n_iterations: int
    final_delta: float
    rho_up: np.ndarray
    rho_down: np.ndarray
    magnetization: float
    entropy_ts: float = 0.0
    history: list = field(default_factory=list)
    components: dict = None    # EnergyComponents (driver_spin.rs:715-780) of the final iteration


def run_scf_spin(sys, n_bands, max_iter=100, conv_threshold=1e-6, energy_threshold=1e-5, mixing_beta=0.3,
                 mixing_ndim=8, smearing="fermi_dirac", sigma=0.01, kerker=False, q_tf=None,
                 starting_magnetization=0.0, tot_magnetization=None, verbose=False, mixer="anderson",
                 mixing_period=3):
    """LSDA SCF of driver_spin.rs:114-839 with dense diagonalisation.

    starting_magnetization: the atom average of the per-species fractions
    (driver_spin.rs:125-167); the start density splits as (1 +- m)/2.
    Mixing is CCMX: Anderson (+ Kerker when asked) on rho_up + rho_down and
    plain Anderson on rho_up - rho_down (driver_spin.rs:792-826)."""
    dims = sys.dims
    omega = sys.omega
    weights = list(sys.kpt_weights)
    n = sys.n_grid
    dv = omega / n
    spin_factor = 1.0
    if sys.symmetry.n_ops > 1:
        src, arg = gather_map(dims, [(op.rotation, op.translation) for op in sys.symmetry.operations])
    else:
        src = arg = np.zeros((1, 0))
    kw = None
    if kerker:
        # Broyden and Periodic Pulay always estimate q_TF (mixing/mod.rs:254-275)
        user_q = q_tf is not None and mixer == "anderson"
        q2 = q_tf * q_tf if user_q else auto_q_tf_squared(sys.n_electrons, omega)
        kw = np.where(sys.g_squared < G2_ZERO_THRESHOLD, 0.0, sys.g_squared / (sys.g_squared + q2))
    mix_tot = make_mixer(mixer, mixing_beta, mixing_ndim, dims, kw, mixing_period)
    mix_mag = make_mixer(mixer, mixing_beta, mixing_ndim, dims, None, mixing_period)
    d_dense = [p.d_dense() for p in sys.projectors]
    core = sys.rho_core_r
    core_half = core / 2.0 if core.size else core
    up = sys.rho_init_r * (1.0 + starting_magnetization) / 2.0
    dn = sys.rho_init_r * (1.0 - starting_magnetization) / 2.0
    e_prev = None
    hist = []
    nk = len(sys.kpoints)

    def diag(veff):
        ev, ps = [], []
        for ik in range(nk):
            h = dense_hamiltonian(sys.basis.miller, sys.kinetic[ik], veff, dims, sys.projectors[ik].b, d_dense[ik])
            w, v = lowest_eigenpairs(h, n_bands)
            ev.append(w)
            ps.append(v)
        return ev, ps

    for it in range(max_iter):
        tot = up + dn
        tot_g = density_r_to_g(tot, dims)
        vh = hartree(tot_g, sys.g_squared)
        rxu, rxd = add_core(up, core_half), add_core(dn, core_half)
        exc_in, vxu_in, vxd_in = lsda_xc(rxu, rxd)
        v_up = sys.v_local_g + vh + density_r_to_g(vxu_in, dims)
        v_dn = sys.v_local_g + vh + density_r_to_g(vxd_in, dims)
        ev_up, ps_up = diag(v_up)
        # equal potentials (an unmagnetised state) give the same eigenpairs: reuse them
        ev_dn, ps_dn = (ev_up, ps_up) if np.array_equal(v_up, v_dn) else diag(v_dn)
        ev_all = ev_up + ev_dn
        w_all = weights + weights
        if tot_magnetization is None:
            ef = find_fermi_energy(ev_all, w_all, sys.n_electrons, sigma, smearing, spin_factor)
            ef_up = ef_dn = ef
        else:
            n_up_t = 0.5 * (sys.n_electrons + tot_magnetization)
            n_dn_t = (sys.n_electrons - tot_magnetization) / 2.0
            ef_up = find_fermi_energy(ev_up, weights, n_up_t, sigma, smearing, spin_factor)
            ef_dn = find_fermi_energy(ev_dn, weights, n_dn_t, sigma, smearing, spin_factor)
            ef = 0.5 * (ef_up + ef_dn)
        occ_up = [spin_factor * occupation01(smearing, e, ef_up, sigma) for e in ev_up]
        occ_dn = [spin_factor * occupation01(smearing, e, ef_dn, sigma) for e in ev_dn]
        n_up = float(sum(np.sum(o) * w for o, w in zip(occ_up, weights)))
        n_dn = float(sum(np.sum(o) * w for o, w in zip(occ_dn, weights)))
        up_new = compute_density(sys.g_to_fft, dims, ps_up, occ_up, weights, n_up, omega)
        dn_new = compute_density(sys.g_to_fft, dims, ps_dn, occ_dn, weights, n_dn, omega)
        if src.shape[0] > 1:
            up_new = symmetrize_density(up_new, dims, src, arg)
            dn_new = symmetrize_density(dn_new, dims, src, arg)
        delta = max(density_diff(up, up_new, omega), density_diff(dn, dn_new, omega))
        tot_new = up_new + dn_new
        tot_new_g = density_r_to_g(tot_new, dims)
        exc_o, vxu_o, vxd_o = lsda_xc(add_core(up_new, core_half), add_core(dn_new, core_half))
        e_vxc_o = float(np.sum((up_new * vxu_o + dn_new * vxd_o) * dv))
        e_xc_o = float(np.sum(add_core(tot_new, core) * exc_o * dv))
        e_band = float(sum(np.sum(o * w * e) for o, w, e in zip(occ_up + occ_dn, w_all, ev_all)))
        ts = entropy_ts(ev_all, w_all, ef, sigma, smearing, spin_factor)
        e_tot = e_band - hartree_energy(tot_new_g, sys.g_squared, omega) + (e_xc_o - e_vxc_o) + sys.e_ewald - ts
        e_xc_i = float(np.sum(add_core(tot, core) * exc_in * dv))
        e_vxc_i = float(np.sum((up * vxu_in + dn * vxd_in) * dv))
        e_hf = e_band - hartree_energy(tot_g, sys.g_squared, omega) + (e_xc_i - e_vxc_i) + sys.e_ewald - ts
        de = None if e_prev is None else abs(e_tot - e_prev)
        e_prev = e_tot
        mag = abs(n_up - n_dn)
        hist.append((it, e_tot, delta, mag))
        if verbose:
            print(f"iter {it:3d} E={e_tot:.10f} dE={de} drho={delta:.3e} M={mag:.6f}")
        if delta < conv_threshold and de is not None and de < energy_threshold:
            bs = [p.b for p in sys.projectors]
            comp = dict(e_band=e_band,
                        e_kinetic=(kinetic_expectation(sys.kinetic, ps_up, occ_up, weights)
                                   + kinetic_expectation(sys.kinetic, ps_dn, occ_dn, weights)),
                        e_local=local_pp_energy(tot_new, sys.v_local_g, dims, omega),
                        e_nonlocal=(nonlocal_expectation(bs, d_dense, ps_up, occ_up, weights)
                                    + nonlocal_expectation(bs, d_dense, ps_dn, occ_dn, weights)),
                        e_hartree=hartree_energy(tot_new_g, sys.g_squared, omega), e_xc=e_xc_o, e_vxc=e_vxc_o,
                        e_ewald=sys.e_ewald, e_smearing=-ts)
            return OracleSpinResult(e_tot, e_hf, ef, ev_all, it + 1, delta, up_new, dn_new, mag, ts, hist, comp)
        t_mix = mix_tot.mix(tot, tot_new)
        m_mix = mix_mag.mix(up - dn, up_new - dn_new)
        up = 0.5 * (t_mix + m_mix)
        dn = 0.5 * (t_mix - m_mix)
    raise RuntimeError(f"spin SCF did not converge in {max_iter} iterations (delta={delta})")

"""UPF v2 norm-conserving pseudopotential reader and radial transforms.

Mirrors pwdft/pwdft-core/src/pseudopotential/upf/parse.rs:20-135 (field
extraction by first textual occurrence, Ry/Bohr -> eV/Å conversion),
upf/xml.rs (attribute and data-block scanning) and upf/mod.rs:166-213
(V_loc(|G|) with the erf split of the Coulomb tail).  Simpson quadrature
follows numerics.rs:24-53 (QE even-mesh boundary correction).
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np
from scipy.special import erf as _erf

from .consts import BOHR_TO_ANG, BOHR3_TO_ANG3, E2_COULOMB, G_ZERO_THRESHOLD, RY_TO_EV


class UpfError(ValueError):
    """Malformed or unsupported pseudopotential file (PwdftError::Parse)."""


def _extract_attr(content: str, name: str):
    pat = f'{name}="'
    s = content.find(pat)
    if s < 0:
        return None
    s += len(pat)
    e = content.find('"', s)
    if e < 0:
        return None
    return content[s:e]


def _extract_block(content: str, tag: str, expected: int) -> np.ndarray:
    p = content.find(f"<{tag}")
    if p < 0:
        raise UpfError(f"missing tag <{tag}>")
    gt = content.find(">", p)
    if gt < 0:
        raise UpfError(f"malformed tag <{tag}>")
    start = gt + 1
    end = content.find(f"</{tag}>", start)
    if end < 0:
        raise UpfError(f"missing closing tag </{tag}>")
    toks = content[start:end].split()
    try:
        vals = np.array([float(t) for t in toks], dtype=np.float64)
    except ValueError as exc:
        raise UpfError(f"float parse error in {tag}: {exc}") from exc
    if vals.size != expected:
        raise UpfError(f"{tag}: expected {expected} values, got {vals.size}")
    return vals


def _beta_l(content: str, tag: str) -> int:
    p = content.find(f"<{tag}")
    if p < 0:
        raise UpfError(f"missing tag <{tag}>")
    gt = content.find(">", p)
    if gt < 0:
        raise UpfError(f"malformed tag <{tag}>")
    am = _extract_attr(content[p:gt], "angular_momentum")
    if am is None:
        raise UpfError(f"missing angular_momentum attribute in {tag}")
    l = int(am.strip())
    if l < 0:
        raise UpfError(f"{tag}: angular_momentum must be non-negative (got {l})")
    return l


@dataclass
class Upf:
    element: str
    z_valence: float
    l_max: int
    r: np.ndarray          # Å
    rab: np.ndarray        # Å
    v_local: np.ndarray    # eV
    beta_l: list           # angular momentum per projector
    beta: list             # r·β(r) per projector, UPF value / sqrt(BOHR_TO_ANG)
    dij: np.ndarray        # eV, n_proj x n_proj row-major
    rho_atom: np.ndarray   # UPF value / BOHR_TO_ANG
    core_charge: np.ndarray = field(default_factory=lambda: np.zeros(0))  # e/Å³, empty if no NLCC

    @property
    def n_proj(self) -> int:
        return len(self.beta)

    def has_nlcc(self) -> bool:
        return self.core_charge.size > 0

    def has_rho_atom(self) -> bool:
        return bool(np.any(np.abs(self.rho_atom) > 1e-20))


def parse_upf(content: str) -> Upf:
    """parse_upf_body (upf/parse.rs:20-135)."""
    if "<UPF" not in content and "<PP_HEADER" not in content:
        raise UpfError("unrecognized pseudopotential format (only UPF v2 is supported)")
    el = _extract_attr(content, "element")
    if el is None:
        raise UpfError("missing element in PP_HEADER")

    def num(name, conv):
        v = _extract_attr(content, name)
        if v is None:
            raise UpfError(f"missing {name}")
        try:
            return conv(v.strip())
        except ValueError as exc:
            raise UpfError(f"{name} parse error: {exc}") from exc

    zv = num("z_valence", float)
    lmax = num("l_max", int)
    nproj = num("number_of_proj", int)
    mesh = num("mesh_size", int)
    r = _extract_block(content, "PP_R", mesh) * BOHR_TO_ANG
    rab = _extract_block(content, "PP_RAB", mesh) * BOHR_TO_ANG
    vloc = _extract_block(content, "PP_LOCAL", mesh) * RY_TO_EV
    sq = math.sqrt(BOHR_TO_ANG)
    betas, ls = [], []
    for i in range(1, nproj + 1):
        tag = f"PP_BETA.{i}"
        ls.append(_beta_l(content, tag))
        betas.append(_extract_block(content, tag, mesh) / sq)
    dij = _extract_block(content, "PP_DIJ", nproj * nproj) * RY_TO_EV
    try:
        rho_atom = _extract_block(content, "PP_RHOATOM", mesh) / BOHR_TO_ANG
    except UpfError:
        rho_atom = np.zeros(mesh)
    nlcc = ('core_correction="T"' in content or 'core_correction="t"' in content
            or "nlcc=.true." in content)
    if nlcc:
        try:
            core = _extract_block(content, "PP_NLCC", mesh) / BOHR3_TO_ANG3
        except UpfError:
            core = np.zeros(mesh)
    else:
        core = np.zeros(0)
    return Upf(el.strip(), zv, lmax, r, rab, vloc, ls, betas, dij, rho_atom, core)


def load_upf(path) -> Upf:
    with open(path, "r", encoding="utf-8", errors="replace") as f:
        return parse_upf(f.read())


def simpson(f: np.ndarray, rab: np.ndarray) -> float:
    """Scalar Simpson with the reference's summation order (numerics.rs:24-53)."""
    n = f.size
    if n < 3:
        return float(np.sum(f * rab))
    s = 0.0
    fr = f * rab
    for i in range(1, n - 1):
        s += (4.0 if i % 2 == 1 else 2.0) * fr[i]
    if n % 2 == 1:
        return (fr[0] + s + fr[n - 1]) / 3.0
    acc = fr[0] + s
    acc = acc - 0.25 * fr[n - 3]
    acc += fr[n - 2]
    acc = acc + 1.25 * fr[n - 1]
    return acc / 3.0


def simpson_rows(f: np.ndarray, rab: np.ndarray) -> np.ndarray:
    """Vectorised Simpson over the last axis of f (many integrands at once).

    Same weights as `simpson`; the summation order differs, so results agree
    to a few ulps rather than bit for bit.
    """
    n = f.shape[-1]
    fr = f * rab
    if n < 3:
        return fr.sum(axis=-1)
    w = np.where(np.arange(n) % 2 == 1, 4.0, 2.0)
    w[0] = 1.0
    if n % 2 == 1:
        w[-1] = 1.0
    else:
        # interior weights up to n-2, then -1/4 at n-3, +1 at n-2, 5/4 at n-1
        w[n - 1] = 1.25
        w[n - 2] = w[n - 2] + 1.0
        w[n - 3] = w[n - 3] - 0.25
    return (fr @ w) / 3.0


def v_local_of_g(pp: Upf, g_norm: np.ndarray, omega: float) -> np.ndarray:
    """V_loc(|G|) in eV for an array of |G| (upf/mod.rs:166-213).

    Short-range part by Simpson with sinc(Gr); the erf(r)/r Coulomb tail is
    added analytically as −4πZe² e^{−G²/4}/(ΩG²).  At G=0 the full Coulomb
    term Ze²/r is removed instead (the finite "α Z" piece).
    """
    g = np.asarray(g_norm, dtype=np.float64)
    out = np.empty_like(g)
    four_pi = 4.0 * math.pi
    r = pp.r
    zero = g < G_ZERO_THRESHOLD
    if np.any(zero):
        vs = pp.v_local + pp.z_valence * E2_COULOMB / np.maximum(r, 1e-20)
        out[zero] = four_pi / omega * simpson_rows(r * r * vs, pp.rab)
    nz = ~zero
    if np.any(nz):
        tsp = 2.0 / math.sqrt(math.pi)
        with np.errstate(divide="ignore", invalid="ignore"):
            eor = np.where(r < 1e-20, tsp, _erf(r) / np.where(r < 1e-20, 1.0, r))
        vs = pp.v_local + pp.z_valence * E2_COULOMB * eor
        base = r * r * vs
        gz = g[nz]
        res = np.empty(gz.size)
        for s in range(0, gz.size, 512):
            gg = gz[s:s + 512, None]
            gr = gg * r[None, :]
            with np.errstate(divide="ignore", invalid="ignore"):
                sinc = np.where(gr < 1e-10, 1.0 - gr * gr / 6.0, np.sin(gr) / np.where(gr < 1e-10, 1.0, gr))
            res[s:s + 512] = simpson_rows(base[None, :] * sinc, pp.rab)
        g2 = gz * gz
        out[nz] = four_pi / omega * res - four_pi * pp.z_valence * E2_COULOMB * np.exp(-g2 / 4.0) / (omega * g2)
    return out


def spherical_bessel(l: int, x: np.ndarray) -> np.ndarray:
    """j_l(x) by explicit l=0,1 forms and upward recurrence (nonlocal.rs:592-612)."""
    x = np.asarray(x, dtype=np.float64)
    small = np.abs(x) < 1e-10
    xs = np.where(small, 1.0, x)
    s, c = np.sin(xs), np.cos(xs)
    j0 = s / xs
    if l == 0:
        return np.where(small, 1.0, j0)
    j1 = s / (xs * xs) - c / xs
    if l == 1:
        return np.where(small, 0.0, j1)
    jm1, jl = j0, j1
    for n in range(1, l):
        jp1 = (2 * n + 1) / xs * jl - jm1
        jm1, jl = jl, jp1
    return np.where(small, 0.0, jl)


def beta_form_factor(pp: Upf, iproj: int, q: np.ndarray) -> np.ndarray:
    """F_i(q) = 4π ∫ [rβ_i(r)] j_l(qr) r dr (nonlocal.rs:566-583), q in Å⁻¹."""
    q = np.asarray(q, dtype=np.float64)
    l = pp.beta_l[iproj]
    rb = pp.beta[iproj] * pp.r
    out = np.empty(q.size)
    for s in range(0, q.size, 512):
        qq = q[s:s + 512, None]
        out[s:s + 512] = 4.0 * math.pi * simpson_rows(rb[None, :] * spherical_bessel(l, qq * pp.r[None, :]), pp.rab)
    return out


def sinc_transform(pp: Upf, radial: np.ndarray, weight_r2: bool, g: np.ndarray) -> np.ndarray:
    """∫ f(r) j0(|G| r) [r²] dr by Simpson for an array of |G| (potentials.rs:99-115,
    initial_density.rs:149-166)."""
    g = np.asarray(g, dtype=np.float64)
    base = radial * (pp.r * pp.r if weight_r2 else 1.0)
    out = np.empty(g.size)
    for s in range(0, g.size, 512):
        gr = g[s:s + 512, None] * pp.r[None, :]
        with np.errstate(divide="ignore", invalid="ignore"):
            j0 = np.where(gr < 1e-10, 1.0 - gr * gr / 6.0, np.sin(gr) / np.where(gr < 1e-10, 1.0, gr))
        out[s:s + 512] = simpson_rows(base[None, :] * j0, pp.rab)
    return out

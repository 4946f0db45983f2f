"""Crystal geometry, plane-wave basis, FFT grid index maps and k-point sets.

Host-side mirror of the reference's setup layer:
  * Lattice / Crystal          -- pwdft/pwdft-core/src/crystal.rs:77-120
  * BasisSet                   -- pwdft/pwdft-core/src/basis.rs:36-63
  * fft_grid_size, FftGrid     -- pwdft/pwdft-core/src/fft.rs:257-279, scf/grid.rs:44-147
  * monkhorst_pack             -- pwdft/pwdft-core/src/kpoints.rs:226-288

Floating-point expressions keep the reference's operation order so that the
integer maps (Miller lists, flat FFT indices) are bit-identical: the basis
filter compares |G|^2 computed as ((gx*gx + gy*gy) + gz*gz) with
G = (n1*b1 + n2*b2) + n3*b3, exactly as nalgebra evaluates it.
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from .consts import HBAR2_OVER_2M


def _cross(a, b):
    return np.array([a[1] * b[2] - a[2] * b[1],
                     a[2] * b[0] - a[0] * b[2],
                     a[0] * b[1] - a[1] * b[0]], dtype=np.float64)


def _dot(a, b):
    return (a[0] * b[0] + a[1] * b[1]) + a[2] * b[2]


@dataclass
class Lattice:
    """Real-space lattice vectors a, b, c (Å), rows of a 3x3 array."""
    a: np.ndarray
    b: np.ndarray
    c: np.ndarray

    @staticmethod
    def from_rows(rows) -> "Lattice":
        r = np.asarray(rows, dtype=np.float64)
        return Lattice(r[0].copy(), r[1].copy(), r[2].copy())

    def volume(self) -> float:
        """Ω = |a·(b×c)| (crystal.rs:108)."""
        return abs(_dot(_cross(self.a, self.b), self.c))

    def reciprocal(self) -> "Lattice":
        """b_i = 2π (a_j × a_k) / (a·(b×c)) (crystal.rs:112-120)."""
        triple = _dot(_cross(self.a, self.b), self.c)
        factor = 2.0 * math.pi / triple
        return Lattice(_cross(self.b, self.c) * factor,
                       _cross(self.c, self.a) * factor,
                       _cross(self.a, self.b) * factor)

    def rows(self) -> np.ndarray:
        return np.stack([self.a, self.b, self.c])

    def matrix(self) -> np.ndarray:
        """Columns a, b, c (crystal.rs:124)."""
        return self.rows().T.copy()


@dataclass
class Atom:
    symbol: str
    frac: tuple  # fractional coordinates

    def cart(self, lat: Lattice) -> np.ndarray:
        """τ = f1 a + f2 b + f3 c (crystal.rs:77-80)."""
        f1, f2, f3 = self.frac
        return (f1 * lat.a + f2 * lat.b) + f3 * lat.c


@dataclass
class Crystal:
    lattice: Lattice
    atoms: list = field(default_factory=list)

    def species(self) -> list:
        out = []
        for a in self.atoms:
            if a.symbol not in out:
                out.append(a.symbol)
        return out


def fcc_primitive(a_ang: float) -> Lattice:
    """a/2·{(0,1,1),(1,0,1),(1,1,0)} -- the reference's Si test cell."""
    return Lattice(a_ang / 2.0 * np.array([0.0, 1.0, 1.0]),
                   a_ang / 2.0 * np.array([1.0, 0.0, 1.0]),
                   a_ang / 2.0 * np.array([1.0, 1.0, 0.0]))


def diamond_primitive(symbol: str, a_ang: float) -> Crystal:
    return Crystal(fcc_primitive(a_ang), [Atom(symbol, (0.0, 0.0, 0.0)),
                                         Atom(symbol, (0.25, 0.25, 0.25))])


DIAMOND_CONVENTIONAL_SITES = [
    (0.0, 0.0, 0.0), (0.0, 0.5, 0.5), (0.5, 0.0, 0.5), (0.5, 0.5, 0.0),
    (0.25, 0.25, 0.25), (0.25, 0.75, 0.75), (0.75, 0.25, 0.75), (0.75, 0.75, 0.25),
]


def diamond_supercell(symbol: str, a_ang: float, reps=(1, 1, 1),
                      displacement_ang: float = 0.0, rng=None) -> Crystal:
    """Conventional cubic diamond cell repeated reps times, with optional
    seeded uniform Cartesian displacements in [-d, d] per component."""
    n1, n2, n3 = reps
    lat = Lattice(np.array([a_ang * n1, 0.0, 0.0]), np.array([0.0, a_ang * n2, 0.0]),
                  np.array([0.0, 0.0, a_ang * n3]))
    atoms = []
    for i in range(n1):
        for j in range(n2):
            for k in range(n3):
                for s in DIAMOND_CONVENTIONAL_SITES:
                    f = ((s[0] + i) / n1, (s[1] + j) / n2, (s[2] + k) / n3)
                    atoms.append(Atom(symbol, f))
    if displacement_ang > 0.0:
        rng = rng if rng is not None else np.random.default_rng(0)
        lens = np.array([a_ang * n1, a_ang * n2, a_ang * n3])
        for at in atoms:
            d = rng.uniform(-displacement_ang, displacement_ang, 3)
            at.frac = tuple(float(x) for x in (np.array(at.frac) + d / lens))
    return Crystal(lat, atoms)


class BasisSet:
    """G-sphere (ħ²/2m)|G|² ≤ ecut, enumerated n1 → n2 → n3 (basis.rs:36-63).

    The sphere is k-independent: the same Miller list serves every k-point.
    Because the outermost loop is n1, the points of one x-plane (fixed n1)
    are contiguous in basis order; the GPU plane kernels rely on this.
    """

    def __init__(self, lattice: Lattice, ecut_ev: float):
        recip = lattice.reciprocal()
        g_max_sq = ecut_ev / HBAR2_OVER_2M
        g_max = math.sqrt(g_max_sq)
        b1, b2, b3 = recip.a, recip.b, recip.c
        nmax = [int(math.ceil(g_max / math.sqrt(_dot(b, b)))) for b in (b1, b2, b3)]
        r1 = np.arange(-nmax[0], nmax[0] + 1, dtype=np.int32)
        r2 = np.arange(-nmax[1], nmax[1] + 1, dtype=np.int32)
        r3 = np.arange(-nmax[2], nmax[2] + 1, dtype=np.int32)
        m1, m2, m3 = np.meshgrid(r1, r2, r3, indexing="ij")
        m1 = m1.ravel(); m2 = m2.ravel(); m3 = m3.ravel()
        f1 = m1.astype(np.float64); f2 = m2.astype(np.float64); f3 = m3.astype(np.float64)
        g = np.empty((m1.size, 3))
        for c in range(3):
            g[:, c] = (f1 * b1[c] + f2 * b2[c]) + f3 * b3[c]
        n2 = (g[:, 0] * g[:, 0] + g[:, 1] * g[:, 1]) + g[:, 2] * g[:, 2]
        keep = n2 <= g_max_sq
        self.miller = np.stack([m1[keep], m2[keep], m3[keep]], axis=1).astype(np.int32)
        self.g = g[keep].copy()
        self.ecut = ecut_ev
        self.recip = recip

    def __len__(self):
        return self.miller.shape[0]

    def index_of(self, n1, n2, n3):
        hit = np.nonzero((self.miller[:, 0] == n1) & (self.miller[:, 1] == n2) & (self.miller[:, 2] == n3))[0]
        return int(hit[0]) if hit.size else None

    def kinetic(self, k=(0.0, 0.0, 0.0)) -> np.ndarray:
        """(ħ²/2m)|k+G|² in eV (potentials.rs:179)."""
        q = np.asarray(k, dtype=np.float64)[None, :] + self.g
        return HBAR2_OVER_2M * ((q[:, 0] * q[:, 0] + q[:, 1] * q[:, 1]) + q[:, 2] * q[:, 2])


def is_fft_friendly(n: int) -> bool:
    if n == 0:
        return False
    for p in (2, 3, 5):
        while n % p == 0:
            n //= p
    return n == 1


def fft_grid_size(n_max: int) -> int:
    """Smallest 2,3,5-smooth n ≥ 2·n_max+1 (fft.rs:257-266)."""
    n = 2 * n_max + 1
    while not is_fft_friendly(n):
        n += 1
    return n


MAX_FFT_DIM = 1024


def grid_dims_for(basis: BasisSet, ecutrho_ratio: int = 4, explicit=None):
    """FftGrid::new sizing rule (scf/grid.rs:44-87)."""
    if explicit is not None:
        dims = tuple(int(d) for d in explicit)
    else:
        nmax = np.abs(basis.miller).max(axis=0) if len(basis) else np.zeros(3, dtype=np.int64)
        s = math.isqrt(ecutrho_ratio)
        scale = s if s * s == ecutrho_ratio else s + 1
        dims = tuple(fft_grid_size(int(scale * m)) for m in nmax)
    if max(dims) > MAX_FFT_DIM:
        raise ValueError(f"FFT grid too large: {dims} exceeds MAX_FFT_DIM={MAX_FFT_DIM}")
    return dims


def miller_to_idx(dims, n1, n2, n3):
    """Flat index of wrapped Miller triple, x slowest (scf/grid.rs:142-147)."""
    d0, d1, d2 = dims
    i1 = np.mod(n1, d0)
    i2 = np.mod(n2, d1)
    i3 = np.mod(n3, d2)
    return (i1 * d1 + i2) * d2 + i3


def grid_miller(dims):
    """Signed Miller triple of every flat grid index (scf/grid.rs:120-129):
    i > n/2 maps to i - n."""
    out = []
    for d in dims:
        i = np.arange(d)
        out.append(np.where(i > d // 2, i - d, i).astype(np.int64))
    return out


def grid_g_vectors(dims, recip: Lattice) -> np.ndarray:
    """G-vector of every flat grid index, shape (N, 3), Å⁻¹."""
    m0, m1, m2 = grid_miller(dims)
    n1, n2, n3 = np.meshgrid(m0, m1, m2, indexing="ij")
    f1 = n1.ravel().astype(np.float64); f2 = n2.ravel().astype(np.float64); f3 = n3.ravel().astype(np.float64)
    g = np.empty((f1.size, 3))
    for c in range(3):
        g[:, c] = (f1 * recip.a[c] + f2 * recip.b[c]) + f3 * recip.c[c]
    return g


# --------------------------------------------------------------------------
# k-points (kpoints.rs:226-288)
# --------------------------------------------------------------------------

SHIFT_FLAGS = {"gamma": (0, 0, 0), "gamma_centered": (0, 0, 0), "mp1976": (1, 1, 1), "shifted": (1, 1, 1)}


@dataclass
class KPoint:
    k: np.ndarray  # Cartesian Å⁻¹
    weight: float


def mp_fractional_coord(i1, i2, i3, grid, flags):
    raw = [i1 / grid[0] + flags[0] / (2.0 * grid[0]),
           i2 / grid[1] + flags[1] / (2.0 * grid[1]),
           i3 / grid[2] + flags[2] / (2.0 * grid[2])]
    return [r - math.floor(r + 0.5) for r in raw]


def monkhorst_pack(grid, shift, lattice: Lattice):
    flags = SHIFT_FLAGS[shift] if isinstance(shift, str) else tuple(shift)
    recip = lattice.reciprocal()
    w = 1.0 / float(grid[0] * grid[1] * grid[2])
    out = []
    for i1 in range(grid[0]):
        for i2 in range(grid[1]):
            for i3 in range(grid[2]):
                f = mp_fractional_coord(i1, i2, i3, grid, flags)
                k = (f[0] * recip.a + f[1] * recip.b) + f[2] * recip.c
                out.append(KPoint(k, w))
    return out


def gamma_only():
    return [KPoint(np.zeros(3), 1.0)]

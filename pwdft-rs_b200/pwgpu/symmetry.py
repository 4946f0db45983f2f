"""Space-group detection, IBZ k-point reduction, and the G-space
symmetrisation gather map.

Mirrors pwdft/pwdft-core/src/symmetry/detect.rs:22-186 (metric-preserving
integer rotations + fractional translations), symmetry/operations.rs
(rotation algebra, wrap_to_unit_cell, frac_distance), symmetry/mod.rs:32-45
(SymmetryInfo) and symmetry/kpoints.rs:31-143 (orbit-based IBZ reduction).
The gather map of symmetry/density/g_space.rs:147-252 is produced here as
integer source indices + phase arguments so that the device kernel only
gathers; the map is bit-identical to the reference's index arithmetic.
"""

from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from .crystal import Crystal, KPoint, SHIFT_FLAGS, grid_miller, mp_fractional_coord


def _wrap(f):
    return [x - math.floor(x) for x in f]


def _frac_distance(a, b):
    d2 = 0.0
    for i in range(3):
        dx = a[i] - b[i]
        dx -= _round_half_away(dx)
        d2 += dx * dx
    return math.sqrt(d2)


def _round_half_away(x):
    """Rust f64::round: half away from zero."""
    return math.floor(x + 0.5) if x >= 0 else -math.floor(-x + 0.5)


def _apply(rot, f):
    return [(rot[i][0] * f[0] + rot[i][1] * f[1]) + rot[i][2] * f[2] for i in range(3)]


@dataclass
class SpaceGroupOp:
    rotation: list      # 3x3 int, acts on fractional coordinates
    translation: list   # fractional, wrapped to [0,1)

    def is_identity(self, tol):
        return (self.rotation == [[1, 0, 0], [0, 1, 0], [0, 0, 1]]
                and all(min(abs(t), abs(1.0 - t)) < tol for t in self.translation))


@dataclass
class SymmetryInfo:
    operations: list
    has_inversion: bool
    has_time_reversal: bool
    tolerance: float

    @property
    def n_ops(self):
        return len(self.operations)

    @staticmethod
    def identity_only():
        return SymmetryInfo([SpaceGroupOp([[1, 0, 0], [0, 1, 0], [0, 0, 1]], [0.0, 0.0, 0.0])],
                            False, False, 1e-5)

    @staticmethod
    def from_crystal(crystal: Crystal, tolerance: float = 1e-5):
        ops = find_symmetry_operations(crystal, tolerance)
        inv = any(op.rotation == [[-1, 0, 0], [0, -1, 0], [0, 0, -1]] for op in ops)
        return SymmetryInfo(ops, inv, True, tolerance)


def _metric(crystal: Crystal):
    m = crystal.lattice.matrix()  # columns a, b, c
    g = np.zeros((3, 3))
    for i in range(3):
        for j in range(3):
            g[i, j] = (m[0, i] * m[0, j] + m[1, i] * m[1, j]) + m[2, i] * m[2, j]
    return g


def _dot_metric(c, d, g):
    s = 0.0
    for i in range(3):
        for j in range(3):
            s += float(c[i]) * g[i, j] * float(d[j])
    return s


def _candidates(g, target, tol):
    rng = [int(math.sqrt(target / g[i, i]) + 1.5) for i in range(3)]
    out = []
    for n0 in range(-rng[0], rng[0] + 1):
        for n1 in range(-rng[1], rng[1] + 1):
            for n2 in range(-rng[2], rng[2] + 1):
                c = (n0, n1, n2)
                if abs(_dot_metric(c, c, g) - target) < tol:
                    out.append(c)
    return out


def find_symmetry_operations(crystal: Crystal, tol: float):
    """detect.rs:22-49."""
    g = _metric(crystal)
    cands = [_candidates(g, g[j, j], tol) for j in range(3)]
    rots = []
    for c0 in cands[0]:
        for c1 in cands[1]:
            if abs(_dot_metric(c0, c1, g) - g[0, 1]) > tol:
                continue
            for c2 in cands[2]:
                det = (c0[0] * (c1[1] * c2[2] - c1[2] * c2[1]) - c0[1] * (c1[0] * c2[2] - c1[2] * c2[0])
                       + c0[2] * (c1[0] * c2[1] - c1[1] * c2[0]))
                if det not in (1, -1):
                    continue
                if abs(_dot_metric(c0, c2, g) - g[0, 2]) > tol:
                    continue
                if abs(_dot_metric(c1, c2, g) - g[1, 2]) > tol:
                    continue
                rots.append([[c0[0], c1[0], c2[0]], [c0[1], c1[1], c2[1]], [c0[2], c1[2], c2[2]]])
    ops = []
    for rot in rots:
        tau = _find_translation(crystal, rot, tol)
        if tau is not None:
            ops.append(SpaceGroupOp(rot, _wrap(tau)))
    if not any(op.is_identity(tol) for op in ops):
        raise RuntimeError("identity operation not found -- bug in symmetry detection")
    return ops


def _find_translation(crystal, rot, tol):
    if not crystal.atoms:
        return [0.0, 0.0, 0.0]
    ref = crystal.atoms[0]
    rp = _apply(rot, ref.frac)
    for tgt in crystal.atoms:
        if tgt.symbol != ref.symbol:
            continue
        tau = _wrap([tgt.frac[i] - rp[i] for i in range(3)])
        if _all_atoms_map(crystal, rot, tau, tol):
            return tau
    return None


def _all_atoms_map(crystal, rot, tau, tol):
    for at in crystal.atoms:
        rp = _apply(rot, at.frac)
        mapped = _wrap([rp[i] + tau[i] for i in range(3)])
        if not any(o.symbol == at.symbol and _frac_distance(mapped, o.frac) < tol for o in crystal.atoms):
            return False
    return True


def _inverse_transpose(rot):
    r = rot
    d = (r[0][0] * (r[1][1] * r[2][2] - r[1][2] * r[2][1]) - r[0][1] * (r[1][0] * r[2][2] - r[1][2] * r[2][0])
         + r[0][2] * (r[1][0] * r[2][1] - r[1][1] * r[2][0]))
    adj = [[(r[1][1] * r[2][2] - r[1][2] * r[2][1]) * d, (r[0][2] * r[2][1] - r[0][1] * r[2][2]) * d,
            (r[0][1] * r[1][2] - r[0][2] * r[1][1]) * d],
           [(r[1][2] * r[2][0] - r[1][0] * r[2][2]) * d, (r[0][0] * r[2][2] - r[0][2] * r[2][0]) * d,
            (r[0][2] * r[1][0] - r[0][0] * r[1][2]) * d],
           [(r[1][0] * r[2][1] - r[1][1] * r[2][0]) * d, (r[0][1] * r[2][0] - r[0][0] * r[2][1]) * d,
            (r[0][0] * r[1][1] - r[0][1] * r[1][0]) * d]]
    return [[adj[j][i] for j in range(3)] for i in range(3)]


def _frac_to_grid_index(f, grid, flags):
    idx = []
    for j in range(3):
        n = float(grid[j])
        x = f[j] - math.floor(f[j])
        i_f = x * n - 0.5 * flags[j]
        i_r = _round_half_away(i_f)
        if abs(i_f - i_r) > 1e-6:
            return None
        i = int(i_r)
        idx.append(((i % grid[j]) + grid[j]) % grid[j])
    return (idx[0] * grid[1] + idx[1]) * grid[2] + idx[2]


def reduce_kpoints(grid, shift, symmetry: SymmetryInfo, lattice):
    """Orbit reduction of a Monkhorst-Pack mesh (symmetry/kpoints.rs:31-95).

    Weight of each representative = orbit size / N_total; representatives
    keep the first-visited grid point's coordinates."""
    flags = SHIFT_FLAGS[shift] if isinstance(shift, str) else tuple(shift)
    recip = lattice.reciprocal()
    n_total = grid[0] * grid[1] * grid[2]
    fracs = [mp_fractional_coord(i1, i2, i3, grid, flags)
             for i1 in range(grid[0]) for i2 in range(grid[1]) for i3 in range(grid[2])]
    rits = [_inverse_transpose(op.rotation) for op in symmetry.operations]
    visited = [False] * n_total
    out = []
    for idx in range(n_total):
        if visited[idx]:
            continue
        f = fracs[idx]
        orbit = 0
        for rit in rits:
            kr = _apply(rit, f)
            ri = _frac_to_grid_index(kr, grid, flags)
            if ri is not None and not visited[ri]:
                visited[ri] = True
                orbit += 1
            if symmetry.has_time_reversal:
                ni = _frac_to_grid_index([-kr[0], -kr[1], -kr[2]], grid, flags)
                if ni is not None and not visited[ni]:
                    visited[ni] = True
                    orbit += 1
        k = (f[0] * recip.a + f[1] * recip.b) + f[2] * recip.c
        out.append(KPoint(k, orbit / n_total))
    return out


def g_space_gather_map(dims, symmetry: SymmetryInfo):
    """Per destination grid point and op: flat source index of ρ(R^T n) and
    the phase argument 2π n·τ (symmetry/density/g_space.rs:176-243).

    Returns (src int32 [n_ops, N], arg float64 [n_ops, N]).  The device
    kernel computes ρ_sym(n) = (1/N_ops) Σ_S e^{-i arg_S(n)} ρ(src_S(n)).
    """
    m0, m1, m2 = grid_miller(dims)
    n1, n2, n3 = np.meshgrid(m0, m1, m2, indexing="ij")
    n1 = n1.ravel(); n2 = n2.ravel(); n3 = n3.ravel()
    d0, d1, d2 = dims
    srcs, args = [], []
    two_pi = 2.0 * math.pi
    for op in symmetry.operations:
        r = op.rotation
        rt = [[r[j][i] for j in range(3)] for i in range(3)]
        s1 = rt[0][0] * n1 + rt[0][1] * n2 + rt[0][2] * n3
        s2 = rt[1][0] * n1 + rt[1][1] * n2 + rt[1][2] * n3
        s3 = rt[2][0] * n1 + rt[2][1] * n2 + rt[2][2] * n3
        src = (np.mod(s1, d0) * d1 + np.mod(s2, d1)) * d2 + np.mod(s3, d2)
        t = op.translation
        arg = two_pi * ((n1.astype(np.float64) * t[0] + n2.astype(np.float64) * t[1]) + n3.astype(np.float64) * t[2])
        srcs.append(src.astype(np.int32))
        args.append(arg)
    return np.stack(srcs), np.stack(args)

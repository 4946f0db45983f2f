"""Symmetry detection and IBZ reduction of the host setup against the
reference's own unit tests (symmetry/detect.rs:246-335,
symmetry/kpoints.rs:170-270): operation counts of Fd-3m Si, BCC Fe, P1 and
P-1 cells, identity, inversion, closure and determinants, and the IBZ sizes
of the Si meshes."""

import numpy as np

from pwgpu.crystal import Atom, Crystal, Lattice, diamond_primitive, monkhorst_pack
from pwgpu.symmetry import SymmetryInfo, reduce_kpoints

TOL = 1e-5


def si_fcc():
    return diamond_primitive("Si", 5.431)


def fe_bcc():
    a = 2.87
    return Crystal(Lattice(a / 2 * np.array([-1.0, 1.0, 1.0]), a / 2 * np.array([1.0, -1.0, 1.0]),
                           a / 2 * np.array([1.0, 1.0, -1.0])), [Atom("Fe", (0.0, 0.0, 0.0))])


def triclinic(atoms):
    return Crystal(Lattice(np.array([3.1, 0.2, 0.1]), np.array([0.3, 4.2, -0.1]), np.array([-0.1, 0.15, 5.3])),
                   atoms)


def ops_of(cr):
    return SymmetryInfo.from_crystal(cr, TOL).operations


def closed(ops):
    """Every product S1 S2 = (R1 R2, R1 t2 + t1) is in the set (t mod 1)."""
    table = [(np.array(o.rotation), np.array(o.translation, dtype=float)) for o in ops]
    for r1, t1 in table:
        for r2, t2 in table:
            r, t = r1 @ r2, r1 @ t2 + t1
            hit = False
            for r3, t3 in table:
                d = t - t3
                if np.array_equal(r, r3) and np.all(np.abs(d - np.round(d)) < TOL):
                    hit = True
                    break
            if not hit:
                return False
    return True


def test_si_fd3m():
    ops = ops_of(si_fcc())
    assert len(ops) == 48
    assert any(o.is_identity(TOL) for o in ops)
    assert any(np.array_equal(np.array(o.rotation), -np.eye(3, dtype=int)) for o in ops)
    assert SymmetryInfo.from_crystal(si_fcc(), TOL).has_inversion
    dets = [round(np.linalg.det(np.array(o.rotation, dtype=float))) for o in ops]
    assert set(dets) <= {1, -1} and dets.count(1) == 24 and dets.count(-1) == 24
    assert closed(ops)


def test_bcc_fe():
    ops = ops_of(fe_bcc())
    assert len(ops) == 48
    assert closed(ops)


def test_triclinic_cells():
    assert len(ops_of(triclinic([Atom("C", (0.13, 0.27, 0.41)), Atom("N", (0.6, 0.3, 0.1))]))) == 1
    assert len(ops_of(triclinic([Atom("C", (0.13, 0.27, 0.41)), Atom("C", (0.87, 0.73, 0.59))]))) == 2


def test_si_ibz_sizes():
    cr = si_fcc()
    sym = SymmetryInfo.from_crystal(cr, TOL)
    for grid, shift, n in (((4, 4, 4), "gamma", 8), ((4, 4, 4), "mp1976", 10), ((3, 3, 3), "gamma", 4)):
        kp = reduce_kpoints(grid, shift, sym, cr.lattice)
        assert len(kp) == n, (grid, shift, len(kp))
        assert abs(sum(k.weight for k in kp) - 1.0) < 1e-12
    kp = reduce_kpoints((4, 4, 4), "gamma", SymmetryInfo.identity_only(), cr.lattice)
    assert len(kp) == 64 == len(monkhorst_pack((4, 4, 4), "gamma", cr.lattice))


def test_monkhorst_pack_meshes():
    """kpoints.rs:398-470: 64 points, weights sum to 1, Gamma in the
    Gamma-centred 4x4x4 and 3x3x3 meshes and not in the shifted 4x4x4, and
    per-axis flags (0,0,0) / (1,1,1) equal to the named shifts."""
    lat = si_fcc().lattice
    g4 = monkhorst_pack((4, 4, 4), "gamma", lat)
    assert len(g4) == 64 and abs(sum(k.weight for k in g4) - 1.0) < 1e-12
    has_gamma = lambda kp: any(np.linalg.norm(k.k) < 1e-12 for k in kp)
    assert has_gamma(g4) and has_gamma(monkhorst_pack((3, 3, 3), "gamma", lat))
    s4 = monkhorst_pack((4, 4, 4), "mp1976", lat)
    assert not has_gamma(s4)
    for named, flags in ((g4, (0, 0, 0)), (s4, (1, 1, 1))):
        custom = monkhorst_pack((4, 4, 4), flags, lat)
        assert len(custom) == len(named)
        assert all(np.linalg.norm(a.k - b.k) < 1e-14 for a, b in zip(named, custom))


def test_basis_properties():
    """basis.rs:122-180 at 200 eV: 259 plane waves, G = 0 present, every
    kinetic energy within the cutoff, Miller indices unique."""
    from pwgpu.consts import HBAR2_OVER_2M
    from pwgpu.crystal import BasisSet
    b = BasisSet(si_fcc().lattice, 200.0)
    assert len(b) == 259
    ke = HBAR2_OVER_2M * np.einsum("ij,ij->i", b.g, b.g)
    assert np.min(ke) < 1e-12 and np.max(ke) <= 200.0 + 1e-10
    assert (b.miller == 0).all(axis=1).sum() == 1
    assert len({tuple(m) for m in b.miller.tolist()}) == len(b)

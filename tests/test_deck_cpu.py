"""The YAML deck front door (pwgpu.deck) against the reference's deck
contract (settings.rs:27-613, scf/mod.rs:166-225, main.rs:32-114):
defaults, rejections, and a deck-built system equal to the one built by
hand for the same calculation.  CPU only."""

import numpy as np
import pytest

from conftest import GOLDEN
from pwgpu.consts import BOHR_TO_ANG, RY_TO_EV
from pwgpu.deck import DeckError, deck_system, load_pseudopotentials, parse_deck, to_symmetry_info
from pwgpu.upf import load_upf

UPF = GOLDEN + "/upf"

SI2 = """
system:
  lattice:
    - [0.0, {h}, {h}]
    - [{h}, 0.0, {h}]
    - [{h}, {h}, 0.0]
  atoms:
    - {{symbol: Si, position: [0.0, 0.0, 0.0]}}
    - {{symbol: Si, position: [0.25, 0.25, 0.25]}}
kpoints:
  type: monkhorst_pack
  grid: [4, 4, 4]
"""


def si2_deck(extra="", a_ang=10.26 * BOHR_TO_ANG):
    return SI2.format(h=a_ang / 2.0) + extra


def test_defaults_match_the_reference():
    d = parse_deck(si2_deck())
    assert d.basis == {"ecutwfc": 300.0, "ecutrho_ratio": 4, "fft_grid": None}
    assert d.kpoints["shift"] == (0, 0, 0)
    assert d.scf == {"max_iter": 50, "conv_threshold": 1e-6, "energy_threshold": 1e-5, "n_bands": None,
                     "eigensolver": "dense", "wfrx_subspace": False, "mixing_beta": 0.3, "mixing_ndim": 8,
                     "mixing_mode": "plain", "pulay_period": 3, "adaptive_beta": False, "smearing": "fermi_dirac",
                     "smearing_width": 0.05}
    assert d.electrons == {"spin_polarized": False, "starting_magnetization": {}, "tot_magnetization": None,
                           "occupations": "smearing"}
    assert d.xc == {"functional": "pz"}
    assert d.symmetry == {"enabled": True, "time_reversal": True, "tolerance": 1e-5}
    assert d.output == {"verbosity": "normal", "write_density": False, "write_bands": True}
    assert d.initial_density == {"gaussian_sigma": 1.0}


@pytest.mark.parametrize("shift,flags", [("gamma_centered", (0, 0, 0)), ("mp1976", (1, 1, 1)),
                                         ("shifted", (1, 1, 1)), ("mp_1976", (1, 1, 1)),
                                         ("{custom: [1, 0, 1]}", (1, 0, 1))])
def test_kgrid_shift_spellings(shift, flags):
    d = parse_deck(si2_deck().replace("grid: [4, 4, 4]", f"grid: [4, 4, 4]\n  shift: {shift}"))
    assert d.kpoints["shift"] == flags


@pytest.mark.parametrize("bad", [
    "scf:\n  mixing_beta: 0.3\n  mixin_ndim: 4\n",          # unknown field
    "xcc:\n  functional: pz\n",                              # unknown block
    "scf:\n  max_iter: many\n",                              # wrong type
    "scf:\n  smearing: triangle\n",                          # unknown variant
    "electrons:\n  starting_magnetization: {Xx: 0.5}\n",     # unknown element
])
def test_parse_errors(bad):
    with pytest.raises(DeckError) as e:
        parse_deck(si2_deck(bad))
    assert e.value.kind == "parse"


def test_missing_required_blocks():
    with pytest.raises(DeckError):
        parse_deck("basis:\n  ecutwfc: 100.0\n")
    with pytest.raises(DeckError):
        parse_deck(si2_deck().split("kpoints:")[0])


@pytest.mark.parametrize("extra,name", [
    ("scf:\n  mixing_beta: 0.0\n", "mixing_beta"),
    ("scf:\n  mixing_beta: 1.5\n", "mixing_beta"),
    ("scf:\n  conv_threshold: 0.0\n", "conv_threshold"),
    ("scf:\n  n_bands: 0\n", "n_bands"),
    ("scf:\n  smearing_width: -0.1\n", "smearing_sigma"),
    ("scf:\n  mixing_mode: periodic_pulay\n  pulay_period: 0\n", "pulay_period"),
    ("basis:\n  ecutwfc: 100.0\n  ecutrho_ratio: 0\n", "ecutrho_ratio"),
    ("initial_density:\n  gaussian_sigma: -1.0\n", "gaussian_sigma"),
])
def test_invalid_params(si_pp, extra, name):
    d = parse_deck(si2_deck("basis:\n  ecutwfc: 100.0\n" + extra if not extra.startswith("basis") else extra))
    with pytest.raises(DeckError) as e:
        deck_system(d, {"Si": si_pp})
    assert e.value.kind == "invalid_param" and e.value.name == name


@pytest.mark.parametrize("extra", ["xc:\n  functional: pbe\n", "scf:\n  adaptive_beta: true\n",
                                   ])
def test_not_implemented(si_pp, extra):
    d = parse_deck(si2_deck("basis:\n  ecutwfc: 100.0\n" + extra))
    with pytest.raises(DeckError) as e:
        deck_system(d, {"Si": si_pp})
    assert e.value.kind == "not_implemented"


def test_band_path_parses_and_is_refused(si_pp):
    d = parse_deck(si2_deck().replace("type: monkhorst_pack\n  grid: [4, 4, 4]",
                                      "type: band_path\n  path:\n    - {label: G, frac: [0, 0, 0]}\n"
                                      "    - {label: X, frac: [0.5, 0, 0.5]}"))
    assert d.kpoints["npoints"] == 50 and [p[0] for p in d.kpoints["path"]] == ["G", "X"]
    with pytest.raises(DeckError) as e:
        deck_system(d, {"Si": si_pp})
    assert e.value.kind == "not_implemented"


def test_deck_system_equals_the_hand_built_case(si_pp):
    """The plain-method case written as a deck builds the same system as
    pwgpu.config1 (10 IBZ k-points, n_pw 411, 24^3)."""
    from pwgpu.config1 import SCF_KW, config1_system
    extra = ("basis:\n  ecutwfc: {e}\nscf:\n  n_bands: 8\n  mixing_beta: 0.7\n  smearing: fixed\n"
             "  max_iter: 120\n").format(e=20.0 * RY_TO_EV)
    d = parse_deck(si2_deck(extra).replace("grid: [4, 4, 4]", "grid: [4, 4, 4]\n  shift: mp1976"))
    pps = load_pseudopotentials([a for a, _ in d.atoms], UPF)
    s, kw = deck_system(d, pps)
    ref = config1_system(load_upf(UPF + "/Si.upf"))
    assert (s.n_pw, s.dims, len(s.kpoints)) == (ref.n_pw, ref.dims, len(ref.kpoints)) == (411, (24, 24, 24), 10)
    assert np.allclose([k.weight for k in s.kpoints], [k.weight for k in ref.kpoints])
    assert np.array_equal(s.rho_init_r, ref.rho_init_r)
    assert np.array_equal(s.v_local_g, ref.v_local_g)
    assert kw["n_bands"] == SCF_KW["n_bands"] and kw["mixing_beta"] == SCF_KW["mixing_beta"]
    assert kw["smearing"] == "fixed" and kw["mixer"] == "anderson" and kw["kerker"] is False


def test_spin_and_symmetry_switches(si_pp):
    d = parse_deck(si2_deck("basis:\n  ecutwfc: 100.0\nelectrons:\n  spin_polarized: true\n"
                            "  starting_magnetization: {Si: 0.4}\n  tot_magnetization: 2.0\n"
                            "symmetry:\n  enabled: false\n"))
    s, kw = deck_system(d, {"Si": si_pp})
    assert s.nspin == 2 and kw["starting_magnetization"] == pytest.approx(0.4) and kw["tot_magnetization"] == 2.0
    assert to_symmetry_info(d, None).n_ops == 1
    assert len(s.kpoints) == 64  # identity only, no time reversal: the full 4x4x4 mesh
    d2 = parse_deck(si2_deck("basis:\n  ecutwfc: 100.0\nsymmetry:\n  time_reversal: false\n"))
    s2, _ = deck_system(d2, {"Si": si_pp})
    d3 = parse_deck(si2_deck("basis:\n  ecutwfc: 100.0\n"))
    s3, kw3 = deck_system(d3, {"Si": si_pp})
    assert len(s2.kpoints) >= len(s3.kpoints) and kw3["n_bands"] == min(s3.n_pw, 20)


CUBE = "system:\n  lattice: [[1,0,0],[0,1,0],[0,0,1]]\nkpoints:\n  type: monkhorst_pack\n  grid: [2, 2, 2]\n"


@pytest.mark.parametrize("field", ["nspin: 2", "mixing_beta: 0.25"])
def test_pre_rename_electrons_fields_rejected_by_name(field):
    """settings.rs:854-897: `electrons.nspin` and `electrons.mixing_beta`
    (moved to `spin_polarized` and `scf.*`) are parse errors naming the field."""
    with pytest.raises(DeckError) as e:
        parse_deck(CUBE + "electrons:\n  " + field + "\n")
    assert e.value.kind == "parse" and field.split(":")[0] in str(e.value)


@pytest.mark.parametrize("mode,mixer,kerker", [
    ("plain", "anderson", False), ("kerker", "anderson", True), ("broyden", "broyden", False),
    ("broyden_kerker", "broyden", True), ("periodic_pulay", "periodic_pulay", False),
    ("periodic_pulay_kerker", "periodic_pulay", True)])
@pytest.mark.parametrize("period", [None, 5])
def test_mixing_modes_convert_to_the_mixer(si_pp, mode, mixer, kerker, period):
    """settings.rs:1078-1175, 1389-1418: every MixingModeType parses and
    converts to its mixer (Kerker with q_TF estimated at run time); Periodic
    Pulay takes scf.pulay_period, default 3."""
    extra = f"basis:\n  ecutwfc: 100.0\nscf:\n  mixing_mode: {mode}\n"
    if period is not None:
        extra += f"  pulay_period: {period}\n"
    d = parse_deck(si2_deck(extra))
    assert d.scf["mixing_mode"] == mode
    _, kw = deck_system(d, {"Si": si_pp})
    assert (kw["mixer"], kw["kerker"]) == (mixer, kerker)
    assert kw["mixing_period"] == (3 if period is None else period)


def test_fixed_occupations_with_fixed_smearing():
    """settings.rs:1468-1483."""
    d = parse_deck(CUBE + "scf:\n  smearing: fixed\nelectrons:\n  occupations: fixed\n")
    assert d.scf["smearing"] == "fixed" and d.electrons["occupations"] == "fixed" and d.atoms == []


@pytest.mark.parametrize("smearing", ["fermi_dirac", "gaussian", "methfessel_paxton", "cold", "fixed"])
def test_smearing_names_parse(smearing):
    """settings.rs:1031-1044, 1419-1434."""
    assert parse_deck(CUBE + f"scf:\n  smearing: {smearing}\n").scf["smearing"] == smearing


@pytest.mark.parametrize("verbosity", ["low", "normal", "high"])
def test_verbosity_names_parse(verbosity):
    """settings.rs:428-433, 1060-1067."""
    assert parse_deck(CUBE + f"output:\n  verbosity: {verbosity}\n").output["verbosity"] == verbosity


def test_to_crystal_structure():
    """settings.rs:968-981: lattice rows as given (Å), fractional positions."""
    from pwgpu.deck import to_crystal
    d = parse_deck(si2_deck(a_ang=5.431))
    c = to_crystal(d)
    assert [a.symbol for a in c.atoms] == ["Si", "Si"] and tuple(c.atoms[1].frac) == (0.25, 0.25, 0.25)
    assert abs(c.lattice.a[0]) < 1e-12 and abs(c.lattice.a[1] - 2.7155) < 1e-12


def test_deck_contract_follows_the_reference_code_not_its_stale_tests():
    """Two of the reference's settings tests expect what its own types
    refuse: settings.rs:829 parses a deck with a `pseudopotentials:` block,
    but InputSettings (settings.rs:27-68) denies unknown fields and has no
    such field; settings.rs:1486 expects an unknown element symbol to parse
    and fail in to_crystal, but AtomInput.symbol is the Element enum
    (settings.rs:89-92), so the symbol fails at parse time. The deck here
    follows the types: both are parse errors naming the offending value."""
    with pytest.raises(DeckError) as e:
        parse_deck(si2_deck('pseudopotentials:\n  Si: "../pseudopotentials/nc/lda/Si.upf"\n'))
    assert e.value.kind == "parse" and "pseudopotentials" in str(e.value)
    with pytest.raises(DeckError) as e:
        parse_deck(si2_deck().replace("symbol: Si, position: [0.0, 0.0, 0.0]", "symbol: Xz, position: [0.0, 0.0, 0.0]"))
    assert e.value.kind == "parse" and "Xz" in str(e.value)


@pytest.mark.parametrize("text,field,value", [
    ("scf:\n  conv_threshold: 1e-8\n", ("scf", "conv_threshold"), 1e-8),
    ("scf:\n  energy_threshold: 1E-7\n", ("scf", "energy_threshold"), 1e-7),
    ("scf:\n  mixing_beta: .5\n", ("scf", "mixing_beta"), 0.5),
    ("scf:\n  max_iter: 0x40\n", ("scf", "max_iter"), 64),
    ("scf:\n  n_bands: ~\n", ("scf", "n_bands"), None),
    ("symmetry:\n  enabled: False\n", ("symmetry", "enabled"), False),
    ("electrons:\n  tot_magnetization: null\n", ("electrons", "tot_magnetization"), None),
])
def test_plain_scalars_typed_as_the_reference_reader_types_them(text, field, value):
    """The reference reads decks with serde_yaml_ng 0.10 (settings.rs:509-511),
    which types plain scalars by the YAML 1.2 core rules: an exponent without
    a dot is a float (PyYAML's YAML 1.1 rules would make `1e-8` a string and
    refuse the deck), 0x/0o/0b prefixes are integers, ~ and null are null."""
    d = parse_deck(CUBE + text)
    assert getattr(d, field[0])[field[1]] == value


@pytest.mark.parametrize("text", [
    "symmetry:\n  enabled: yes\n",        # YAML 1.1 boolean words are strings
    "output:\n  write_bands: on\n",
    "scf:\n  max_iter: 010\n",            # leading zero: a string, not octal 8
    "scf:\n  mixing_beta: '0.5'\n",       # a quoted number stays a string
    "scf:\n  conv_threshold: 1_0\n",
])
def test_yaml_1_1_forms_are_not_numbers_or_booleans(text):
    with pytest.raises(DeckError) as e:
        parse_deck(CUBE + text)
    assert e.value.kind == "parse"

"""The library's deck reader (pwgpu_deck_parse, csrc/deck.cu) against the
Python front door (pwgpu.deck.parse_deck), which the reference's settings
tests pin: the same settings, defaults filled in, from every deck of the
corpus below, and the same refusals (kind 'parse', or 'invalid_param' for a
custom k-grid shift flag above 1). CPU only."""

import pytest

from pwgpu.deck import DeckError, parse_deck, parse_deck_native
from test_deck_cpu import CUBE, si2_deck

FULL = """---
# every block given
system:
  lattice:
    - [0.0, 2.7155, 2.7155]
    - [2.7155, 0.0, 2.7155]
    - [2.7155, 2.7155, 0.0]
  atoms:
    - symbol: Si
      position: [0.0, 0.0, 0.0]
    - symbol: "Si"   # quoted
      position: [0.25, 0.25, 0.25]
basis:
  ecutwfc: 200.0
  ecutrho_ratio: 4
  fft_grid: [24, 24, 24]
kpoints:
  type: monkhorst_pack
  grid: [4, 4, 4]
  shift: mp1976
scf:
  max_iter: 100
  conv_threshold: 1.0e-6
  energy_threshold: 1e-5
  n_bands: 8
  eigensolver: iterative
  wfrx_subspace: true
  mixing_beta: 0.3
  mixing_ndim: 8
  mixing_mode: periodic_pulay_kerker
  pulay_period: 4
  adaptive_beta: false
  smearing: gaussian
  smearing_width: 0.1
electrons:
  occupations: smearing
  spin_polarized: true
  starting_magnetization: {Si: 0.5}
  tot_magnetization: 2
xc:
  functional: pbe
symmetry:
  enabled: false
  time_reversal: false
  tolerance: 1.0e-4
output:
  verbosity: high
  write_density: true
  write_bands: false
initial_density:
  gaussian_sigma: 0.8
"""

FLOW = ("{system: {lattice: [[1, 0, 0], [0, 1, 0], [0, 0, 1]], atoms: [{symbol: C, position: [0, 0, 0]}]},\n"
        " kpoints: {type: monkhorst_pack, grid: [2, 2, 2], shift: {custom: [1, 0, 1]}}}\n")

BAND = CUBE.replace("type: monkhorst_pack\n  grid: [2, 2, 2]",
                    "type: band_path\n  path:\n    - {label: G, frac: [0, 0, 0]}\n"
                    "    - {label: 'X', frac: [0.5, 0, 0.5]}\n    - {label: 1, frac: [0.5, 0.5, 0.5]}\n  npoints: 20")

VALID = {
    "si2": si2_deck(),
    "full": FULL,
    "flow": FLOW,
    "band_path": BAND,
    "cube_no_atoms": CUBE,
    "comments_and_blank_lines": "# deck\n\n" + CUBE.replace("grid: [2, 2, 2]", "grid: [2, 2, 2]  # mesh") + "\n# end\n",
    "nested_lattice_lines": CUBE.replace("[[1,0,0],[0,1,0],[0,0,1]]", "[[1, 0, 0],\n    [0, 1, 0],\n    [0, 0, 1]]"),
    "shift_shifted": si2_deck().replace("grid: [4, 4, 4]", "grid: [4, 4, 4]\n  shift: shifted"),
    "shift_mp_1976": si2_deck().replace("grid: [4, 4, 4]", "grid: [4, 4, 4]\n  shift: mp_1976"),
    "yaml12_numbers": CUBE + "scf:\n  conv_threshold: 1e-8\n  max_iter: 0x40\n  mixing_beta: .5\n  n_bands: ~\n",
    "nulls": CUBE + "basis:\nscf:\n  n_bands: null\nelectrons:\n  tot_magnetization: ~\n  starting_magnetization:\n",
    "dash_at_key_indent": CUBE.replace("system:\n  lattice: [[1,0,0],[0,1,0],[0,0,1]]\n",
                                       "system:\n  lattice:\n  - [1, 0, 0]\n  - [0, 1, 0]\n  - [0, 0, 1]\n"),
    "fixed_occupations": CUBE + "scf:\n  smearing: fixed\nelectrons:\n  occupations: fixed\n",
    "magnetization_two_species": CUBE + "electrons:\n  spin_polarized: true\n  starting_magnetization:\n"
                                        "    Fe: 0.4\n    O: -0.1\n",
}

INVALID = {
    "unknown_field": si2_deck("scf:\n  mixing_beta: 0.3\n  mixin_ndim: 4\n"),
    "unknown_block": si2_deck("xcc:\n  functional: pz\n"),
    "wrong_type": si2_deck("scf:\n  max_iter: many\n"),
    "unknown_variant": si2_deck("scf:\n  smearing: triangle\n"),
    "unknown_element_magnetization": si2_deck("electrons:\n  starting_magnetization: {Xx: 0.5}\n"),
    "unknown_element_atom": si2_deck().replace("symbol: Si, position: [0.0, 0.0, 0.0]", "symbol: Xz, position: [0.0, 0.0, 0.0]"),
    "no_kpoints": si2_deck().split("kpoints:")[0],
    "no_system": "basis:\n  ecutwfc: 100.0\n",
    "empty": "",
    "not_a_mapping": "just text\n",
    "pre_rename_nspin": CUBE + "electrons:\n  nspin: 2\n",
    "pseudopotentials_block": si2_deck('pseudopotentials:\n  Si: "../Si.upf"\n'),
    "yes_bool": CUBE + "symmetry:\n  enabled: yes\n",
    "leading_zero": CUBE + "scf:\n  max_iter: 010\n",
    "quoted_number": CUBE + "scf:\n  mixing_beta: '0.5'\n",
    "lattice_two_rows": CUBE.replace("[[1,0,0],[0,1,0],[0,0,1]]", "[[1,0,0],[0,1,0]]"),
    "grid_two_values": CUBE.replace("grid: [2, 2, 2]", "grid: [2, 2]"),
    "negative_uint": CUBE + "scf:\n  mixing_ndim: -1\n",
    "float_for_uint": CUBE + "scf:\n  max_iter: 5.0\n",
    "null_variant": CUBE + "scf:\n  eigensolver: null\n",
    "missing_grid": CUBE.replace("  grid: [2, 2, 2]\n", ""),
    "missing_type": CUBE.replace("  type: monkhorst_pack\n", ""),
    "custom_without_flags": CUBE.replace("grid: [2, 2, 2]", "grid: [2, 2, 2]\n  shift: {custom: }"),
    "atom_without_position": CUBE.replace("kpoints", "  atoms:\n    - {symbol: Si}\nkpoints"),
    "duplicate_key": CUBE + "scf:\n  max_iter: 5\n  max_iter: 6\n",
    "bad_indent": CUBE + "scf:\n  max_iter: 5\n   mixing_ndim: 4\n",
    "unclosed_bracket": CUBE.replace("grid: [2, 2, 2]", "grid: [2, 2, 2"),
    "tab_indent": CUBE + "scf:\n\tmax_iter: 5\n",
}


@pytest.mark.parametrize("name", sorted(VALID))
def test_valid_decks_give_the_same_settings(name):
    assert parse_deck_native(VALID[name]) == parse_deck(VALID[name])


@pytest.mark.parametrize("name", sorted(INVALID))
def test_invalid_decks_refused_by_both(name):
    with pytest.raises(DeckError) as want:
        parse_deck(INVALID[name])
    with pytest.raises(DeckError) as got:
        parse_deck_native(INVALID[name])
    assert got.value.kind == want.value.kind == "parse", (name, str(got.value))


def test_custom_shift_flag_above_one_is_an_invalid_parameter():
    text = CUBE.replace("grid: [2, 2, 2]", "grid: [2, 2, 2]\n  shift: {custom: [2, 0, 0]}")
    for reader in (parse_deck, parse_deck_native):
        with pytest.raises(DeckError) as e:
            reader(text)
        assert e.value.kind == "invalid_param"


def _damaged(text, n, seed):
    """Seeded random damage: cut a few characters, insert or swap one
    character from the deck's own alphabet of indicators and digits."""
    import numpy as np
    rng = np.random.default_rng(seed)
    alphabet = list("0123456789.-+eE [],{}:\n #\"'xyz_")
    for _ in range(n):
        t = text
        for _ in range(int(rng.integers(1, 3))):
            kind, i = int(rng.integers(3)), int(rng.integers(len(t)))
            c = alphabet[int(rng.integers(len(alphabet)))]
            t = (t[:i] + t[i + int(rng.integers(1, 8)):] if kind == 0 else
                 t[:i] + c + t[i:] if kind == 1 else t[:i] + c + t[i + 1:])
        yield t


@pytest.mark.parametrize("name", ["full", "si2", "band_path", "magnetization_two_species"])
def test_damaged_decks_same_verdict_in_both_readers(name):
    """On 300 seeded damaged copies of a deck the two readers accept the same
    decks with the same settings and refuse the rest with the same kind."""
    accepted = 0
    for t in _damaged(VALID[name], 300, seed=sum(map(ord, name))):
        try:
            want, wk = parse_deck(t), "ok"
        except DeckError as e:
            want, wk = None, e.kind
        try:
            got, gk = parse_deck_native(t), "ok"
        except DeckError as e:
            got, gk = None, e.kind
        assert (gk, got) == (wk, want), t
        accepted += want is not None
    assert 0 < accepted < 300

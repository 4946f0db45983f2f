"""YAML deck front door: the reference's input deck (InputSettings,
settings.rs:27-454) read with the same field names, defaults and
rejections, turned into an ScfSystem plus the SCF keyword arguments of
pwgpu, and run on the device.

What follows the reference:
  * schema: top-level blocks system / basis / kpoints / scf / electrons /
    xc / symmetry / output / initial_density; unknown keys are rejected at
    every level (serde deny_unknown_fields); `system` and `kpoints` are
    required, every other block and field has the reference's default;
  * conversion: InputSettings::to_crystal, to_scf_params (settings.rs:
    520-577), to_symmetry_info (identity only when symmetry is disabled;
    time reversal as configured, :606-613); the Monkhorst-Pack grid is
    always reduced by the symmetry group (main.rs:70-103); n_bands
    defaults to min(n_pw, 20) (main.rs:44); pseudopotentials are
    <Symbol>.upf of a norm-conserving LDA library (upf/mod.rs:114-128);
  * validation: ScfParams::validate (scf/mod.rs:166-225) -- n_bands > 0,
    conv_threshold > 0, mixing_beta in (0, 1], smearing width >= 0,
    ecutrho_ratio >= 1, pulay_period >= 1 for Periodic Pulay, gaussian_sigma
    positive and finite -- and the functional check at SCF entry (only
    "pz" runs; pbe / pbe0 / hse06 parse and are refused as not
    implemented);
  * spin: `spin_polarized` selects two channels; the start density splits
    by the atom average of the per-species starting_magnetization
    (driver_spin.rs:125-167); tot_magnetization fixes the moment.

What differs: both `eigensolver` values (dense, iterative) name the lowest
n_bands eigenpairs, which the device's LOBPCG computes; `wfrx_subspace` (a
warm start of the dense solver) has no counterpart and is accepted.
`adaptive_beta: true` is refused (the device mixers keep beta fixed), and a
`band_path` deck (the reference's band-structure tool, no SCF) is parsed
and refused by run_deck.
"""

from __future__ import annotations

import math
import os
import re
from dataclasses import dataclass

import numpy as np
import yaml

from .context import build_system
from .crystal import Atom, BasisSet, Crystal, Lattice
from .lib import PRECISION_FP64, PwGpu
from .output import write_bands, write_density
from .symmetry import SymmetryInfo, reduce_kpoints
from .upf import load_upf

# IUPAC symbols Z = 1..118 (the set the reference's Element type accepts)
ELEMENTS = (
    "H He Li Be B C N O F Ne Na Mg Al Si P S Cl Ar K Ca Sc Ti V Cr Mn Fe Co Ni Cu Zn Ga Ge As Se Br Kr "
    "Rb Sr Y Zr Nb Mo Tc Ru Rh Pd Ag Cd In Sn Sb Te I Xe Cs Ba La Ce Pr Nd Pm Sm Eu Gd Tb Dy Ho Er Tm "
    "Yb Lu Hf Ta W Re Os Ir Pt Au Hg Tl Pb Bi Po At Rn Fr Ra Ac Th Pa U Np Pu Am Cm Bk Cf Es Fm Md No "
    "Lr Rf Db Sg Bh Hs Mt Ds Rg Cn Nh Fl Mc Lv Ts Og").split()

SMEARINGS = ("fermi_dirac", "gaussian", "methfessel_paxton", "cold", "fixed")
MIXING_MODES = {  # MixingModeType -> (mixer, kerker), settings.rs:355-377
    "plain": ("anderson", False), "kerker": ("anderson", True),
    "broyden": ("broyden", False), "broyden_kerker": ("broyden", True),
    "periodic_pulay": ("periodic_pulay", False), "periodic_pulay_kerker": ("periodic_pulay", True),
}
FUNCTIONALS = ("pz", "pbe", "pbe0", "hse06")


# Plain-scalar typing of the reference's YAML reader (serde_yaml_ng 0.10, the
# YAML 1.2 core schema as that crate applies it), restated here because
# PyYAML types plain scalars by YAML 1.1 (`1e-8` a string, `yes`/`on`
# booleans, `010` octal):
#   null  ~ null Null NULL and the empty scalar;
#   bool  true True TRUE false False FALSE only;
#   int   decimal digits with an optional sign, or 0x / 0o / 0b with digits
#         of that base; digits with a leading zero (`010`) stay a string;
#   float a decimal number with a fraction and/or exponent (`1e-8`, `1.`,
#         `.5`), or .inf / -.inf / .nan in their three spellings; anything
#         else that is not finite stays a string;
# everything else, and every quoted scalar, is a string.
_INT_DEC = re.compile(r"[-+]?[0-9]+\Z")
_FLOAT_DEC = re.compile(r"[-+]?(?:[0-9]+\.?[0-9]*|\.[0-9]+)(?:[eE][-+]?[0-9]+)?\Z")
_RADIX = {"0x": 16, "0o": 8, "0b": 2}


def _core_scalar(v: str):
    if v in ("", "~", "null", "Null", "NULL"):
        return None
    if v in ("true", "True", "TRUE"):
        return True
    if v in ("false", "False", "FALSE"):
        return False
    unsigned = v[1:] if v.startswith("+") else v
    if unsigned[:1] in "+-" and v.startswith("+"):
        return v
    for prefix, base in _RADIX.items():
        if unsigned.startswith(prefix):
            try:
                return int(unsigned[2:], base)
            except ValueError:
                return v
    digits = unsigned.lstrip("-")
    if len(digits) > 1 and digits[0] == "0" and digits.isdigit():
        return v
    if _INT_DEC.match(v):
        return int(v)
    if unsigned in (".inf", ".Inf", ".INF"):
        return math.inf
    if v in ("-.inf", "-.Inf", "-.INF"):
        return -math.inf
    if v in (".nan", ".NaN", ".NAN"):
        return math.nan
    if _FLOAT_DEC.match(v):
        f = float(v)
        return f if math.isfinite(f) else v
    return v


class _DeckLoader(yaml.SafeLoader):
    """SafeLoader with no implicit typing: every plain scalar arrives as a
    string node and is typed by _core_scalar."""


_DeckLoader.yaml_implicit_resolvers = {}


def _construct_str(loader, node):
    value = loader.construct_scalar(node)
    return _core_scalar(value) if node.style is None else value


_DeckLoader.add_constructor("tag:yaml.org,2002:str", _construct_str)


def _construct_map(loader, node):
    """A mapping; a key given twice is an error (serde refuses duplicate
    fields, PyYAML would keep the last)."""
    loader.flatten_mapping(node)
    out = {}
    for k_node, v_node in node.value:
        k = loader.construct_object(k_node, deep=True)
        if isinstance(k, (list, dict)):
            raise yaml.constructor.ConstructorError(None, None, "a collection as a mapping key", k_node.start_mark)
        if k in out:
            raise yaml.constructor.ConstructorError(None, None, f"duplicate field `{k}`", k_node.start_mark)
        out[k] = loader.construct_object(v_node, deep=True)
    return out


_DeckLoader.add_constructor("tag:yaml.org,2002:map", _construct_map)


class DeckError(ValueError):
    """A deck the reference would refuse: kind is 'parse' (PwdftError::Parse),
    'invalid_param' (InvalidParam, with the parameter's name) or
    'not_implemented' (NotImplemented)."""

    def __init__(self, kind: str, message: str, name: str | None = None):
        super().__init__(message)
        self.kind = kind
        self.name = name


def _parse_err(msg):
    return DeckError("parse", f"YAML parse error: {msg}")


def _block(d, where, fields):
    """Check a mapping against its allowed fields (deny_unknown_fields)."""
    if d is None:
        return {}
    if not isinstance(d, dict):
        raise _parse_err(f"{where}: expected a mapping")
    unknown = [k for k in d if k not in fields]
    if unknown:
        raise _parse_err(f"{where}: unknown field `{unknown[0]}`, expected one of {', '.join(fields)}")
    return d


def _num(v, where):
    if isinstance(v, bool) or not isinstance(v, (int, float)):
        raise _parse_err(f"{where}: expected a number, got {v!r}")
    return float(v)


def _uint(v, where):
    if isinstance(v, bool) or not isinstance(v, int) or v < 0:
        raise _parse_err(f"{where}: expected a non-negative integer, got {v!r}")
    return int(v)


def _bool(v, where):
    if not isinstance(v, bool):
        raise _parse_err(f"{where}: expected true or false, got {v!r}")
    return v


def _vec3(v, where, conv):
    if not isinstance(v, (list, tuple)) or len(v) != 3:
        raise _parse_err(f"{where}: expected a list of 3 values")
    return [conv(x, where) for x in v]


def _choice(v, where, options):
    if v not in options:
        raise _parse_err(f"{where}: unknown variant `{v}`, expected one of {', '.join(options)}")
    return v


def _element(v, where):
    if v not in ELEMENTS:
        raise _parse_err(f"{where}: unknown element `{v}`")
    return v


@dataclass
class Deck:
    """The resolved settings (defaults filled in, names as in the YAML)."""
    lattice: list
    atoms: list                 # [(symbol, [f1, f2, f3])]
    basis: dict
    kpoints: dict
    scf: dict
    electrons: dict
    xc: dict
    symmetry: dict
    output: dict
    initial_density: dict


def parse_deck(text: str) -> Deck:
    """InputSettings::from_yaml_str: parse and check a deck; defaults filled in."""
    try:
        raw = yaml.load(text, Loader=_DeckLoader)
    except yaml.YAMLError as e:
        raise _parse_err(str(e)) from None
    top = _block(raw, "settings", ("system", "basis", "kpoints", "scf", "electrons", "xc", "symmetry", "output",
                                   "initial_density"))
    for req in ("system", "kpoints"):
        if req not in top:
            raise _parse_err(f"missing field `{req}`")
    sysb = _block(top["system"], "system", ("lattice", "atoms"))
    if "lattice" not in sysb:
        raise _parse_err("system: missing field `lattice`")
    lat = sysb["lattice"]
    if not isinstance(lat, list) or len(lat) != 3:
        raise _parse_err("system.lattice: expected 3 vectors")
    lattice = [_vec3(row, "system.lattice", _num) for row in lat]
    atoms = []
    for i, a in enumerate(sysb.get("atoms") or []):
        ab = _block(a, f"system.atoms[{i}]", ("symbol", "position"))
        for req in ("symbol", "position"):
            if req not in ab:
                raise _parse_err(f"system.atoms[{i}]: missing field `{req}`")
        atoms.append((_element(ab["symbol"], f"system.atoms[{i}].symbol"),
                      _vec3(ab["position"], f"system.atoms[{i}].position", _num)))

    bb = _block(top.get("basis"), "basis", ("ecutwfc", "ecutrho_ratio", "fft_grid"))
    basis = {"ecutwfc": _num(bb.get("ecutwfc", 300.0), "basis.ecutwfc"),
             "ecutrho_ratio": _uint(bb.get("ecutrho_ratio", 4), "basis.ecutrho_ratio"),
             "fft_grid": (None if bb.get("fft_grid") is None
                          else _vec3(bb["fft_grid"], "basis.fft_grid", _uint))}

    kb = top["kpoints"]
    if not isinstance(kb, dict) or "type" not in kb:
        raise _parse_err("kpoints: missing field `type`")
    ktype = _choice(kb["type"], "kpoints.type", ("monkhorst_pack", "band_path"))
    if ktype == "monkhorst_pack":
        kb = _block(kb, "kpoints", ("type", "grid", "shift"))
        if "grid" not in kb:
            raise _parse_err("kpoints: missing field `grid`")
        shift = kb.get("shift", "gamma_centered")
        if isinstance(shift, dict):
            sb = _block(shift, "kpoints.shift", ("custom",))
            flags = _vec3(sb.get("custom"), "kpoints.shift.custom", _uint)
            if any(f > 1 for f in flags):
                raise DeckError("invalid_param", "kpoints.shift.custom: half-shift flags must be 0 or 1", "shift")
            shift_flags = tuple(flags)
        else:
            s = _choice(shift, "kpoints.shift", ("gamma_centered", "mp1976", "mp_1976", "shifted"))
            shift_flags = (0, 0, 0) if s == "gamma_centered" else (1, 1, 1)
        kpoints = {"type": ktype, "grid": _vec3(kb["grid"], "kpoints.grid", _uint), "shift": shift_flags}
    else:
        kb = _block(kb, "kpoints", ("type", "path", "npoints"))
        path = []
        for i, p in enumerate(kb.get("path") or []):
            pb = _block(p, f"kpoints.path[{i}]", ("label", "frac"))
            path.append((str(pb.get("label")), _vec3(pb.get("frac"), f"kpoints.path[{i}].frac", _num)))
        kpoints = {"type": ktype, "path": path, "npoints": _uint(kb.get("npoints", 50), "kpoints.npoints")}

    sb = _block(top.get("scf"), "scf", ("max_iter", "conv_threshold", "energy_threshold", "n_bands", "eigensolver",
                                        "wfrx_subspace", "mixing_beta", "mixing_ndim", "mixing_mode", "pulay_period",
                                        "adaptive_beta", "smearing", "smearing_width"))
    scf = {"max_iter": _uint(sb.get("max_iter", 50), "scf.max_iter"),
           "conv_threshold": _num(sb.get("conv_threshold", 1e-6), "scf.conv_threshold"),
           "energy_threshold": _num(sb.get("energy_threshold", 1e-5), "scf.energy_threshold"),
           "n_bands": None if sb.get("n_bands") is None else _uint(sb["n_bands"], "scf.n_bands"),
           "eigensolver": _choice(sb.get("eigensolver", "dense"), "scf.eigensolver", ("dense", "iterative")),
           "wfrx_subspace": _bool(sb.get("wfrx_subspace", False), "scf.wfrx_subspace"),
           "mixing_beta": _num(sb.get("mixing_beta", 0.3), "scf.mixing_beta"),
           "mixing_ndim": _uint(sb.get("mixing_ndim", 8), "scf.mixing_ndim"),
           "mixing_mode": _choice(sb.get("mixing_mode", "plain"), "scf.mixing_mode", tuple(MIXING_MODES)),
           "pulay_period": _uint(sb.get("pulay_period", 3), "scf.pulay_period"),
           "adaptive_beta": _bool(sb.get("adaptive_beta", False), "scf.adaptive_beta"),
           "smearing": _choice(sb.get("smearing", "fermi_dirac"), "scf.smearing", SMEARINGS),
           "smearing_width": _num(sb.get("smearing_width", 0.05), "scf.smearing_width")}

    eb = _block(top.get("electrons"), "electrons", ("spin_polarized", "starting_magnetization", "tot_magnetization",
                                                    "occupations"))
    sm = eb.get("starting_magnetization") or {}
    if not isinstance(sm, dict):
        raise _parse_err("electrons.starting_magnetization: expected a mapping")
    electrons = {"spin_polarized": _bool(eb.get("spin_polarized", False), "electrons.spin_polarized"),
                 "starting_magnetization": {_element(k, "electrons.starting_magnetization"):
                                            _num(v, f"electrons.starting_magnetization.{k}") for k, v in sm.items()},
                 "tot_magnetization": (None if eb.get("tot_magnetization") is None
                                       else _num(eb["tot_magnetization"], "electrons.tot_magnetization")),
                 "occupations": _choice(eb.get("occupations", "smearing"), "electrons.occupations",
                                        ("smearing", "fixed"))}

    xb = _block(top.get("xc"), "xc", ("functional",))
    xc = {"functional": _choice(xb.get("functional", "pz"), "xc.functional", FUNCTIONALS)}
    yb = _block(top.get("symmetry"), "symmetry", ("enabled", "time_reversal", "tolerance"))
    symmetry = {"enabled": _bool(yb.get("enabled", True), "symmetry.enabled"),
                "time_reversal": _bool(yb.get("time_reversal", True), "symmetry.time_reversal"),
                "tolerance": _num(yb.get("tolerance", 1e-5), "symmetry.tolerance")}
    ob = _block(top.get("output"), "output", ("verbosity", "write_density", "write_bands"))
    output = {"verbosity": _choice(ob.get("verbosity", "normal"), "output.verbosity", ("low", "normal", "high")),
              "write_density": _bool(ob.get("write_density", False), "output.write_density"),
              "write_bands": _bool(ob.get("write_bands", True), "output.write_bands")}
    ib = _block(top.get("initial_density"), "initial_density", ("gaussian_sigma",))
    initial = {"gaussian_sigma": _num(ib.get("gaussian_sigma", 1.0), "initial_density.gaussian_sigma")}
    return Deck(lattice, atoms, basis, kpoints, scf, electrons, xc, symmetry, output, initial)


def parse_deck_native(text: str) -> Deck:
    """The same deck read by the library's own reader (pwgpu_deck_parse,
    csrc/deck.cu), returned as the Deck parse_deck gives; raises DeckError
    with the same kinds ('parse' for PWGPU_E_PARSE, 'invalid_param' for
    PWGPU_E_INVALID)."""
    import ctypes as ct

    from .lib import PwgpuDeckSettings, load_library
    lib = load_library()
    raw = text.encode()
    h = ct.c_void_p()
    rc = lib.pwgpu_deck_parse(raw, len(raw), ct.byref(h))
    if rc != 0:
        msg = lib.pwgpu_last_error().decode(errors="replace")
        raise DeckError("invalid_param" if rc == -1 else "parse", msg, "shift" if rc == -1 else None)
    try:
        st = PwgpuDeckSettings()
        lib.pwgpu_deck_get_settings(h, ct.byref(st))

        def names(n, width, getter):
            buf = ct.create_string_buffer(max(n, 1) * width)
            vals = np.zeros(max(n, 1) * 3)
            getter(h, buf, vals.ctypes.data_as(ct.POINTER(ct.c_double)))
            return [buf.raw[k * width:(k + 1) * width].split(b"\0")[0].decode() for k in range(n)], vals

        syms, pos = names(st.n_atoms, 8, lib.pwgpu_deck_get_atoms)
        msyms, mvals = names(st.n_starting_magnetization, 8, lib.pwgpu_deck_get_starting_magnetization)
        labels, frac = names(st.n_path, 16, lib.pwgpu_deck_get_band_path)
    finally:
        lib.pwgpu_deck_free(h)
    modes = list(MIXING_MODES)
    if st.kpoints_type == 0:
        kpoints = {"type": "monkhorst_pack", "grid": list(st.mp_grid), "shift": tuple(st.mp_shift)}
    else:
        kpoints = {"type": "band_path", "npoints": st.band_npoints,
                   "path": [(labels[k], [float(x) for x in frac[3 * k:3 * k + 3]]) for k in range(st.n_path)]}
    return Deck(
        lattice=[[st.lattice[3 * r + c] for c in range(3)] for r in range(3)],
        atoms=[(syms[a], [float(x) for x in pos[3 * a:3 * a + 3]]) for a in range(st.n_atoms)],
        basis={"ecutwfc": st.ecutwfc, "ecutrho_ratio": st.ecutrho_ratio,
               "fft_grid": None if not any(st.fft_grid) else list(st.fft_grid)},
        kpoints=kpoints,
        scf={"max_iter": st.max_iter, "conv_threshold": st.conv_threshold, "energy_threshold": st.energy_threshold,
             "n_bands": None if st.n_bands < 0 else st.n_bands,
             "eigensolver": ("dense", "iterative")[st.eigensolver], "wfrx_subspace": bool(st.wfrx_subspace),
             "mixing_beta": st.mixing_beta, "mixing_ndim": st.mixing_ndim, "mixing_mode": modes[st.mixing_mode],
             "pulay_period": st.pulay_period, "adaptive_beta": bool(st.adaptive_beta),
             "smearing": SMEARINGS[st.smearing], "smearing_width": st.smearing_width},
        electrons={"spin_polarized": bool(st.spin_polarized),
                   "starting_magnetization": {k: float(v) for k, v in zip(msyms, mvals)},
                   "tot_magnetization": st.tot_magnetization if st.has_tot_magnetization else None,
                   "occupations": ("smearing", "fixed")[st.occupations]},
        xc={"functional": FUNCTIONALS[st.functional]},
        symmetry={"enabled": bool(st.symmetry_enabled), "time_reversal": bool(st.time_reversal),
                  "tolerance": st.symmetry_tolerance},
        output={"verbosity": ("low", "normal", "high")[st.verbosity], "write_density": bool(st.write_density),
                "write_bands": bool(st.write_bands)},
        initial_density={"gaussian_sigma": st.gaussian_sigma})


def load_deck(path: str) -> Deck:
    """InputSettings::from_yaml_file."""
    with open(path) as f:
        return parse_deck(f.read())


def validate(deck: Deck, n_bands: int) -> None:
    """ScfParams::validate (scf/mod.rs:166-225) on the converted parameters."""
    s = deck.scf

    def bad(name, reason):
        raise DeckError("invalid_param", f"invalid parameter `{name}`: {reason}", name)

    if n_bands == 0:
        bad("n_bands", "must be > 0")
    if s["conv_threshold"] <= 0.0:
        bad("conv_threshold", "must be positive")
    if s["mixing_beta"] <= 0.0 or s["mixing_beta"] > 1.0:
        bad("mixing_beta", f"must be in (0, 1], got {s['mixing_beta']}")
    if s["smearing_width"] < 0.0:
        bad("smearing_sigma", "must be non-negative")
    if deck.basis["ecutrho_ratio"] < 1:
        bad("ecutrho_ratio", f"must be >= 1, got {deck.basis['ecutrho_ratio']}")
    if s["mixing_mode"].startswith("periodic_pulay") and s["pulay_period"] == 0:
        bad("pulay_period", "must be >= 1 for PeriodicPulay mixing")
    g = deck.initial_density["gaussian_sigma"]
    if not math.isfinite(g) or g <= 0.0:
        bad("gaussian_sigma", f"must be positive and finite, got {g}")


def to_crystal(deck: Deck) -> Crystal:
    """InputSettings::to_crystal (settings.rs:520-539)."""
    rows = np.array(deck.lattice, dtype=np.float64)
    return Crystal(Lattice(rows[0], rows[1], rows[2]), [Atom(sym, tuple(pos)) for sym, pos in deck.atoms])


def to_symmetry_info(deck: Deck, crystal: Crystal) -> SymmetryInfo:
    """InputSettings::to_symmetry_info (settings.rs:606-613)."""
    if not deck.symmetry["enabled"]:
        return SymmetryInfo.identity_only()
    info = SymmetryInfo.from_crystal(crystal, deck.symmetry["tolerance"])
    info.has_time_reversal = deck.symmetry["time_reversal"]
    return info


def load_pseudopotentials(symbols, pp_dir: str) -> dict:
    """<Symbol>.upf from pp_dir (or pp_dir/nc/lda, the reference's library
    layout, upf/mod.rs:123-125) for every species of the deck."""
    out = {}
    for sym in dict.fromkeys(symbols):
        for cand in (os.path.join(pp_dir, f"{sym}.upf"), os.path.join(pp_dir, "nc", "lda", f"{sym}.upf")):
            if os.path.exists(cand):
                out[sym] = load_upf(cand)
                break
        else:
            raise DeckError("parse", f"no pseudopotential {sym}.upf under {pp_dir}")
    return out


def deck_system(deck: Deck, pps: dict, projectors_on_device: bool = False):
    """(ScfSystem, SCF keyword arguments of PwGpu.scf_run) of a
    Monkhorst-Pack deck: main.rs:32-114 up to run_scf."""
    if deck.kpoints["type"] != "monkhorst_pack":
        raise DeckError("not_implemented", "band_path decks run the band-structure tool, not an SCF")
    if deck.xc["functional"] != "pz":
        raise DeckError("not_implemented", f"functional `{deck.xc['functional']}` is not implemented (pz only)")
    if deck.scf["adaptive_beta"]:
        raise DeckError("not_implemented", "adaptive_beta: the device mixers keep beta fixed")
    crystal = to_crystal(deck)
    sym = to_symmetry_info(deck, crystal)
    kpts = reduce_kpoints(tuple(deck.kpoints["grid"]), deck.kpoints["shift"], sym, crystal.lattice)
    n_pw = len(BasisSet(crystal.lattice, deck.basis["ecutwfc"]).miller)
    nb = deck.scf["n_bands"] if deck.scf["n_bands"] is not None else min(n_pw, 20)
    validate(deck, nb)
    nspin = 2 if deck.electrons["spin_polarized"] else 1
    fft = None if deck.basis["fft_grid"] is None else tuple(deck.basis["fft_grid"])
    s = build_system(crystal, pps, deck.basis["ecutwfc"], kpts, sym, ecutrho_ratio=deck.basis["ecutrho_ratio"],
                     fft_grid=fft, gaussian_sigma=deck.initial_density["gaussian_sigma"], nspin=nspin,
                     projectors_on_device=projectors_on_device)
    mixer, kerker = MIXING_MODES[deck.scf["mixing_mode"]]
    per_atom = [deck.electrons["starting_magnetization"].get(sym_, 0.0) for sym_, _ in deck.atoms]
    kw = dict(n_bands=nb, max_iter=deck.scf["max_iter"], conv_threshold=deck.scf["conv_threshold"],
              energy_threshold=deck.scf["energy_threshold"], mixing_beta=deck.scf["mixing_beta"],
              mixing_ndim=deck.scf["mixing_ndim"], mixer=mixer, kerker=kerker,
              mixing_period=deck.scf["pulay_period"], smearing=deck.scf["smearing"],
              sigma=deck.scf["smearing_width"])
    if nspin == 2:
        kw["starting_magnetization"] = sum(per_atom) / max(len(per_atom), 1)
        kw["tot_magnetization"] = deck.electrons["tot_magnetization"]
    return s, kw


def run_deck(path: str, pp_dir: str, output_dir: str | None = None, precision: int = PRECISION_FP64,
             device: int = 0, lanes: int = 0):
    """Read a deck, run its SCF on the device, write the output files the
    deck asks for (bands.txt / density.npz in output_dir); returns
    (result dict, eigenvalues [nspin * n_k, n_bands], rho_r, system)."""
    deck = load_deck(path)
    pps = load_pseudopotentials([a for a, _ in deck.atoms], pp_dir)
    s, kw = deck_system(deck, pps, projectors_on_device=True)
    nb = kw.pop("n_bands")
    with PwGpu(s, device=device, lanes=lanes) as dev:
        res, ev, rho, rg = dev.scf_run(s.rho_init_r, nb, precision=precision, **kw)
    if output_dir is not None:
        os.makedirs(output_dir, exist_ok=True)
        if deck.output["write_bands"]:
            write_bands(os.path.join(output_dir, "bands.txt"), s, ev, res["fermi_energy"])
        if deck.output["write_density"]:
            write_density(os.path.join(output_dir, "density.npz"), s, rho, rg)
    return res, ev, rho, s

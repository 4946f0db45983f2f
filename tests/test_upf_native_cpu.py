"""The library's UPF reader (pwgpu_upf_load / pwgpu_upf_parse, host C++)
against the Python reader that the host setup uses and that the parity
pins check (parse_upf_body, pseudopotential/upf/parse.rs:20-135): every
array bit for bit on the twelve UPFs of the fixtures, and the same
acceptance on malformed files (each refused by both, PWGPU_E_PARSE here,
with the reason). CPU only."""

import os
import re

import numpy as np
import pytest

from conftest import UPF_DIR
from pwgpu.lib import PWGPU_E_PARSE, PwGpuError, load_upf_native
from pwgpu.upf import UpfError, load_upf, parse_upf

UPFS = sorted(f for f in os.listdir(UPF_DIR) if f.endswith(".upf"))


def _same(a, b):
    assert a.element == b.element
    assert a.z_valence == b.z_valence and a.l_max == b.l_max
    for name in ("r", "rab", "v_local", "dij", "rho_atom", "core_charge"):
        x, y = getattr(a, name), getattr(b, name)
        assert x.shape == y.shape and np.array_equal(x, y), name
    assert a.beta_l == b.beta_l and len(a.beta) == len(b.beta)
    for x, y in zip(a.beta, b.beta):
        assert np.array_equal(x, y)
    assert a.has_nlcc() == b.has_nlcc() and a.has_rho_atom() == b.has_rho_atom()


@pytest.mark.parametrize("name", UPFS)
def test_native_reader_equals_python_reader(name):
    path = os.path.join(UPF_DIR, name)
    _same(load_upf_native(path), load_upf(path))
    with open(path) as f:
        _same(load_upf_native(text=f.read()), load_upf(path))


def _si_text():
    with open(os.path.join(UPF_DIR, "Si.upf")) as f:
        return f.read()


def _drop_first_value(text, tag):
    """Remove the first number inside <tag ...> ... </tag>."""
    p = text.index("<" + tag)
    gt = text.index(">", p)
    m = re.compile(r"\S+").search(text, gt + 1)
    return text[:m.start()] + text[m.end():]


def _replace_first_value(text, tag, tok):
    p = text.index("<" + tag)
    gt = text.index(">", p)
    m = re.compile(r"\S+").search(text, gt + 1)
    return text[:m.start()] + tok + text[m.end():]


MALFORMED = {
    "not_upf": lambda t: "just some text\n",
    "no_element": lambda t: t.replace('element="', 'elemnt="', 1),
    "no_z_valence": lambda t: t.replace('z_valence="', 'z_val="', 1),
    "bad_mesh_size": lambda t: re.sub(r'mesh_size="\s*(\d+)"', r'mesh_size="\1.5"', t, count=1),
    "short_local": lambda t: _drop_first_value(t, "PP_LOCAL"),
    "bad_float_dij": lambda t: _replace_first_value(t, "PP_DIJ", "1.0q0"),
    "hex_float_r": lambda t: _replace_first_value(t, "PP_R ", "0x1p-3"),
    "unclosed_rab": lambda t: t.replace("</PP_RAB>", "</PP_RAB_X>", 1),
    "negative_l": lambda t: re.sub(r'angular_momentum="\s*\d+"', 'angular_momentum="-1"', t, count=1),
    "missing_beta": lambda t: t.replace("<PP_BETA.2", "<PP_BETA_2", 1).replace("</PP_BETA.2>", "</PP_BETA_2>", 1),
}


@pytest.mark.parametrize("case", sorted(MALFORMED))
def test_malformed_files_refused_by_both_readers(case):
    text = MALFORMED[case](_si_text())
    with pytest.raises(UpfError):
        parse_upf(text)
    with pytest.raises(PwGpuError) as e:
        load_upf_native(text=text)
    assert e.value.code == PWGPU_E_PARSE and str(e.value)


def test_unreadable_optional_blocks_read_as_zero_by_both():
    """PP_RHOATOM and PP_NLCC that do not parse read as zeros (parse.rs
    treats them as optional), in both readers."""
    text = _drop_first_value(_drop_first_value(_si_text(), "PP_RHOATOM"), "PP_NLCC")
    a, b = load_upf_native(text=text), parse_upf(text)
    _same(a, b)
    assert not a.has_rho_atom() and a.has_nlcc() and not np.any(a.core_charge)


def test_accessors_refuse_bad_requests():
    import ctypes as ct

    from pwgpu.lib import UPF_BETA, UPF_R, _f64, load_library
    lib = load_library()
    h = ct.c_void_p()
    assert lib.pwgpu_upf_load(os.fsencode(os.path.join(UPF_DIR, "Si.upf")), ct.byref(h)) == 0
    try:
        small = np.zeros(3)
        assert lib.pwgpu_upf_get_array(h, UPF_R, 0, _f64(small), 3) == -1
        assert b"need" in lib.pwgpu_last_error()
        big = np.zeros(100000)
        assert lib.pwgpu_upf_get_array(h, UPF_BETA, 99, _f64(big), big.size) == -1
        assert lib.pwgpu_upf_get_array(h, 42, 0, _f64(big), big.size) == -1
    finally:
        assert lib.pwgpu_upf_free(h) == 0
    assert lib.pwgpu_upf_load(b"/nonexistent/X.upf", ct.byref(h)) == -1


def _mutations(text, n, seed=20261203):
    """Seeded random damage to a UPF: cut a span, duplicate a span, swap a
    character for another, or cut the file short."""
    rng = np.random.default_rng(seed)
    alphabet = list('0123456789.-+eE <>/="\n PQRSTUVWXYZ_abc')
    for _ in range(n):
        t = text
        for _ in range(int(rng.integers(1, 4))):
            kind = int(rng.integers(4))
            i = int(rng.integers(len(t)))
            if kind == 0:
                t = t[:i] + t[i + int(rng.integers(1, 200)):]
            elif kind == 1:
                j = i + int(rng.integers(1, 200))
                t = t[:j] + t[i:j] + t[j:]
            elif kind == 2:
                t = t[:i] + alphabet[int(rng.integers(len(alphabet)))] + t[i + 1:]
            else:
                t = t[:i]
        yield t


@pytest.mark.parametrize("name", ["Si.upf", "C.upf", "Si_hgh.upf"])
def test_damaged_files_same_verdict_in_both_readers(name):
    """On 150 seeded damaged copies of a UPF, the library's reader and the
    Python reader accept and refuse the same files, and read the same
    arrays from the files they accept; nothing crashes."""
    with open(os.path.join(UPF_DIR, name)) as f:
        text = f.read()
    accepted = 0
    for t in _mutations(text, 150):
        try:
            want = parse_upf(t)
        except (UpfError, ValueError):
            want = None
        try:
            got = load_upf_native(text=t)
        except PwGpuError as e:
            assert e.code == PWGPU_E_PARSE
            got = None
        assert (want is None) == (got is None)
        if want is not None:
            _same(got, want)
            accepted += 1
    assert 0 < accepted < 150

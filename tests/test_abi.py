"""The C-ABI library loads and exports every entry point include/*.h declares.
CPU only: symbols are resolved, nothing is computed."""

import ctypes
import glob
import os
import re

from conftest import ROOT
from pwgpu import lib as L


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b(pwgpu_\w+)\s*\(", text):
            names.add(m.group(1))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_functions()
    for n in ("pwgpu_create", "pwgpu_destroy", "pwgpu_apply_h", "pwgpu_set_veff_g", "pwgpu_last_error"):
        assert n in names


def test_library_exports_every_declared_symbol():
    lib = L.load_library()
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, f"symbols declared in include/ but not exported: {missing}"


def test_version_and_error_strings_callable_without_gpu():
    lib = L.load_library()
    assert lib.pwgpu_version().startswith(b"pwgpu")
    assert isinstance(lib.pwgpu_last_error(), bytes)


def test_create_rejects_null_system_without_touching_device():
    lib = L.load_library()
    h = ctypes.c_void_p()
    rc = lib.pwgpu_create(None, None, ctypes.byref(h))
    assert rc == -1
    assert b"NULL" in lib.pwgpu_last_error()


def test_header_compiles_as_c99_and_cxx(tmp_path):
    """A C caller's view: include/pwgpu.h alone compiles as strict C99 and
    as C++17 (no C++ or torch types cross the boundary)."""
    import shutil
    import subprocess
    import pytest
    if shutil.which("gcc") is None or shutil.which("g++") is None:
        pytest.skip("no host C compiler")
    src = tmp_path / "use_header.c"
    src.write_text('#include "pwgpu.h"\n#include "pwgpu_deck.h"\nint main(void) { return pwgpu_version() == 0; }\n')
    inc = os.path.join(ROOT, "include")
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Wextra", "-pedantic", "-Werror", "-fsyntax-only", "-I", inc,
                    str(src)], check=True)
    subprocess.run(["g++", "-std=c++17", "-Wall", "-Werror", "-fsyntax-only", "-I", inc, "-x", "c++", str(src)],
                   check=True)


def test_ctypes_structs_match_header_layout(tmp_path):
    """Every field of the ctypes mirrors of the header's PODs sits at the
    offset the C compiler gives it, and the sizes agree (a field appended to
    the header without its mirror shows up here)."""
    import shutil
    import subprocess
    if shutil.which("gcc") is None:
        import pytest
        pytest.skip("gcc not available")
    mirrors = {"pwgpu_system": L.PwgpuSystem, "pwgpu_options": L.PwgpuOptions,
               "pwgpu_scf_params": L.PwgpuScfParams, "pwgpu_scf_result": L.PwgpuScfResult,
               "pwgpu_server_options": L.PwgpuServerOptions, "pwgpu_job_info": L.PwgpuJobInfo,
               "pwgpu_server_stats": L.PwgpuServerStats, "pwgpu_upf_info": L.PwgpuUpfInfo,
               "pwgpu_deck_settings": L.PwgpuDeckSettings}
    lines = ['#include <stddef.h>', '#include <stdio.h>', '#include "pwgpu.h"', '#include "pwgpu_deck.h"',
             'int main(void) {']
    for cname, py in mirrors.items():
        lines.append(f'  printf("{cname} size %zu\\n", sizeof({cname}));')
        for fname, _ in py._fields_:
            lines.append(f'  printf("{cname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    lines += ['  return 0;', '}']
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c99", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    got = {tuple(l.split()[:2]): int(l.split()[2]) for l in out if l.strip()}
    for cname, py in mirrors.items():
        assert got[(cname, "size")] == ctypes.sizeof(py), cname
        for fname, _ in py._fields_:
            assert got[(cname, fname)] == getattr(py, fname).offset, (cname, fname)


_C_TO_RUST = {"int32_t": "i32", "int64_t": "i64", "double": "f64", "char": "c_char", "void": "c_void",
              "pwgpu_status": "i32"}


def _rust_type(ctype, array=None):
    """Rust spelling of a C type of the header: `const T*` -> `*const T`,
    `T**` -> `*mut *mut T`, `const char**` -> `*mut *const c_char`."""
    ctype = ctype.strip()
    stars = ctype.count("*")
    base = ctype.replace("*", " ").split()
    const = "const" in base
    base = [b for b in base if b != "const"]
    assert len(base) == 1, ctype
    t = _C_TO_RUST.get(base[0], base[0])
    for i in range(stars):
        t = ("*const " if (i == 0 and const) else "*mut ") + t
    if array:
        t = f"[{t}; {array}]"
    return t.replace(" ", "")


def _header_text():
    text = "".join(open(h).read() for h in sorted(glob.glob(os.path.join(ROOT, "include", "*.h"))))
    return re.sub(r"/\*.*?\*/", "", text, flags=re.S)


def _header_struct(name):
    m = re.search(r"typedef struct " + name + r"\s*\{(.*?)\}\s*" + name + ";", _header_text(), flags=re.S)
    assert m, name
    fields = []
    for decl in m.group(1).split(";"):
        decl = decl.strip()
        if not decl:
            continue
        first = re.match(r"((?:const\s+)?\w+\s*\**)\s*(.*)", decl, flags=re.S)
        ctype, rest = first.group(1), first.group(2)
        for d in rest.split(","):
            d = d.strip()
            stars = len(d) - len(d.lstrip("*"))
            d = d.lstrip("*").strip()
            arr = re.match(r"(\w+)\[(\d+)\]", d)
            if arr:
                fields.append((arr.group(1), _rust_type(ctype + "*" * stars, arr.group(2))))
            else:
                fields.append((d, _rust_type(ctype + "*" * stars)))
    return fields


def _header_function(name):
    m = re.search(r"([\w\s\*]+?)\b" + name + r"\s*\((.*?)\)\s*;", _header_text(), flags=re.S)
    assert m, name
    args = []
    for a in m.group(2).split(","):
        a = " ".join(a.split())
        if a in ("", "void"):
            continue
        t = re.match(r"(.*?[\s\*])(\w+)$", a)
        args.append(_rust_type(t.group(1)))
    return _rust_type(m.group(1).split("\n")[-1]), args


def _rust_block():
    text = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    m = re.search(r"```rust\n(.*?)```", text, flags=re.S)
    return re.sub(r"//[^\n]*", "", m.group(1))


def test_rust_binding_in_integration_matches_header():
    """The Rust FFI declarations a maintainer would add are
    the header's: every #[repr(C)] struct field by field (name and type, in
    order) and every extern fn argument by argument."""
    rust = _rust_block()
    structs = re.findall(r"#\[repr\(C\)\]\s*pub struct (\w+)\s*\{(.*?)\}", rust, flags=re.S)
    checked = set()
    for name, body in structs:
        if "_private" in body:
            assert re.search(r"typedef struct " + name + " " + name + ";", _header_text()), name
            continue
        got = []
        for f in body.split(","):
            f = f.strip()
            if f:
                fm = re.match(r"pub (\w+):\s*(.+)$", f, flags=re.S)
                got.append((fm.group(1), fm.group(2).replace(" ", "").replace("\n", "")))
        assert got == _header_struct(name), name
        checked.add(name)
    assert {"pwgpu_system", "pwgpu_options", "pwgpu_scf_params", "pwgpu_scf_result"} <= checked
    fns = re.findall(r"pub fn (\w+)\((.*?)\)\s*->\s*([^;]+);", rust, flags=re.S)
    assert len(fns) >= 10
    for name, args, ret in fns:
        want_ret, want_args = _header_function(name)
        got_args = [re.match(r"\s*\w+:\s*(.+)$", a, flags=re.S).group(1).replace(" ", "").replace("\n", "")
                    for a in args.split(",") if a.strip()]
        assert got_args == want_args, name
        assert ret.replace(" ", "") == want_ret, name


def _ctypes_argtypes(name):
    """ctypes argument types of a header declaration: pointers as void*,
    int32_t / pwgpu_status as int32, int64_t, double."""
    _, args = _header_function(name)
    out = []
    for a in args:
        if a.startswith("*"):
            out.append(ctypes.c_void_p)
        else:
            out.append({"i32": ctypes.c_int32, "i64": ctypes.c_int64, "f64": ctypes.c_double}[a])
    return out


_NULL_SWEEP = r"""
import ctypes, sys
sys.path[:0] = sys.argv[1:3]
import test_abi as T
from pwgpu import lib as L
lib = ctypes.CDLL(L.LIB_PATH)
lib.pwgpu_last_error.restype = ctypes.c_char_p
for name in T.declared_functions():
    if name in ("pwgpu_version", "pwgpu_last_error"):
        continue
    f = getattr(lib, name)
    f.argtypes = T._ctypes_argtypes(name)
    f.restype = ctypes.c_int32
    print(name, f(*[None if t is ctypes.c_void_p else 0 for t in f.argtypes]),
          (lib.pwgpu_last_error() or b"").decode(errors="replace").replace(" ", "_") or "-", flush=True)
"""


def test_every_entry_point_refuses_null_arguments(tmp_path):
    """No entry point dereferences a NULL handle, server or array: called
    with every pointer NULL and every size zero, each returns
    PWGPU_E_INVALID with a message, and the destroy / free calls accept NULL
    (a no-op, as free(NULL)); the process survives the whole sweep. Runs in
    a child process, so a crash fails this test instead of the suite."""
    import subprocess
    import sys
    script = tmp_path / "null_sweep.py"
    script.write_text(_NULL_SWEEP)
    tests_dir = os.path.join(ROOT, "tests")
    r = subprocess.run([sys.executable, str(script), tests_dir, os.path.join(ROOT, "pwdft-rs_b200")],
                       capture_output=True, text=True, timeout=300, cwd=tests_dir)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    got = {l.split()[0]: (int(l.split()[1]), l.split()[2]) for l in r.stdout.splitlines() if l.startswith("pwgpu_")}
    expected = [n for n in declared_functions() if n not in ("pwgpu_version", "pwgpu_last_error")]
    assert sorted(got) == sorted(expected)
    for name, (rc, msg) in got.items():
        if name in ("pwgpu_destroy", "pwgpu_server_destroy", "pwgpu_upf_free", "pwgpu_deck_free"):
            assert rc == 0, name
        else:
            assert rc == -1, (name, rc)  # PWGPU_E_INVALID
            assert msg != "-", name


_C_CALLER = r"""
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include "pwgpu.h"
#include "pwgpu_deck.h"

/* A C host: read a deck, then the UPF of each species it names, the way a
 * caller without Python fills pwgpu_system's radial fields. */
int main(int argc, char** argv) {
  FILE* f = fopen(argv[1], "rb");
  if (!f) return 2;
  char text[1 << 16];
  size_t n = fread(text, 1, sizeof(text), f);
  fclose(f);
  pwgpu_deck* d = NULL;
  if (pwgpu_deck_parse(text, (int64_t)n, &d) != PWGPU_OK) { printf("deck: %s\n", pwgpu_last_error()); return 3; }
  pwgpu_deck_settings s;
  pwgpu_deck_get_settings(d, &s);
  char* sym = calloc((size_t)s.n_atoms, 8);
  double* pos = calloc((size_t)s.n_atoms * 3, sizeof(double));
  pwgpu_deck_get_atoms(d, sym, pos);
  printf("atoms %d ecut %.3f grid %d %d %d shift %d %d %d nbands %d smearing %d mixing %d\n", s.n_atoms, s.ecutwfc,
         s.mp_grid[0], s.mp_grid[1], s.mp_grid[2], s.mp_shift[0], s.mp_shift[1], s.mp_shift[2], s.n_bands,
         s.smearing, s.mixing_mode);
  for (int a = 0; a < s.n_atoms; ++a) {
    char path[4096];
    snprintf(path, sizeof(path), "%s/%s.upf", argv[2], sym + 8 * a);
    pwgpu_upf* u = NULL;
    if (pwgpu_upf_load(path, &u) != PWGPU_OK) { printf("upf: %s\n", pwgpu_last_error()); return 4; }
    pwgpu_upf_info info;
    pwgpu_upf_get_info(u, &info);
    double* r = malloc(sizeof(double) * (size_t)info.mesh);
    pwgpu_upf_get_array(u, PWGPU_UPF_R, 0, r, info.mesh);
    printf("atom %d %s at %.2f %.2f %.2f: z %.1f nproj %d mesh %d r_last %.6f\n", a, sym + 8 * a, pos[3 * a],
           pos[3 * a + 1], pos[3 * a + 2], info.z_valence, info.n_proj, info.mesh, r[info.mesh - 1]);
    free(r);
    pwgpu_upf_free(u);
  }
  /* a malformed deck is refused with PWGPU_E_PARSE and a message */
  pwgpu_deck* bad = NULL;
  const char* broken = "system:\n  lattice: [[1,0,0]]\n";
  int rc = pwgpu_deck_parse(broken, (int64_t)strlen(broken), &bad);
  printf("broken %d %s\n", rc, rc == PWGPU_E_PARSE && bad == NULL && strlen(pwgpu_last_error()) > 0 ? "refused" : "?");
  free(sym);
  free(pos);
  pwgpu_deck_free(d);
  return 0;
}
"""


def test_c_caller_reads_deck_and_pseudopotentials(tmp_path):
    """A C program linked against libpwgpu.so reads a deck and the UPF of
    each of its species through the C-ABI alone (what the reference's Rust
    host would call), with the values the Python readers give."""
    import shutil
    import subprocess
    import pytest
    from pwgpu.upf import load_upf
    from conftest import UPF_DIR
    if shutil.which("gcc") is None:
        pytest.skip("gcc not available")
    deck = tmp_path / "gaas.yaml"
    deck.write_text("system:\n  lattice: [[0, 2.83, 2.83], [2.83, 0, 2.83], [2.83, 2.83, 0]]\n  atoms:\n"
                    "    - {symbol: Ga, position: [0, 0, 0]}\n    - {symbol: As, position: [0.25, 0.25, 0.25]}\n"
                    "basis:\n  ecutwfc: 272.1\nkpoints:\n  type: monkhorst_pack\n  grid: [4, 4, 4]\n  shift: mp1976\n"
                    "scf:\n  n_bands: 12\n  smearing: gaussian\n  mixing_mode: broyden_kerker\n")
    src = tmp_path / "caller.c"
    src.write_text(_C_CALLER)
    exe = tmp_path / "caller"
    libdir = os.path.dirname(L.LIB_PATH)
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe),
                    "-L", libdir, "-lpwgpu", f"-Wl,-rpath,{libdir}"], check=True)
    out = subprocess.run([str(exe), str(deck), UPF_DIR], check=True, capture_output=True, text=True, timeout=60).stdout
    lines = out.splitlines()
    assert lines[0] == "atoms 2 ecut 272.100 grid 4 4 4 shift 1 1 1 nbands 12 smearing 1 mixing 3"
    for k, el in enumerate(("Ga", "As")):
        pp = load_upf(os.path.join(UPF_DIR, f"{el}.upf"))
        assert lines[1 + k].startswith(f"atom {k} {el} at ")
        assert f"z {pp.z_valence:.1f} nproj {pp.n_proj} mesh {pp.r.size} r_last {pp.r[-1]:.6f}" in lines[1 + k]
    assert lines[3] == "broken -8 refused"

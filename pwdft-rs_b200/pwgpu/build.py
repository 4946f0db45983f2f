"""Build libpwgpu.so (sm_100a) in-tree with nvcc.

    python -m pwgpu.build        (from the pwdft-rs_b200 directory)

The shared library lands next to this file (pwgpu/_lib/libpwgpu.so) so that
it travels with the source tree; nothing is installed elsewhere.
"""

from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
PKG_ROOT = os.path.dirname(HERE)
CSRC = os.path.join(PKG_ROOT, "csrc")
INCLUDE = os.path.join(os.path.dirname(PKG_ROOT), "include")
LIBDIR = os.path.join(HERE, "_lib")
LIB = os.path.join(LIBDIR, "libpwgpu.so")

SOURCES = ["api.cu", "hpsi.cu", "linalg.cu", "lobpcg.cu", "scf.cu", "noalloc.cu", "gemm_bf16.cu", "nl_mixed.cu", "server.cu", "gamma.cu", "setup.cu", "components.cu", "eigh.cu", "chol.cu", "upf.cu", "deck.cu"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
    "--expt-relaxed-constexpr", "-diag-suppress", "20012",
]


def cutlass_root() -> str:
    """CUTLASS/CuTe header tree vendored with the installed flashinfer wheel."""
    import sysconfig
    for base in (sysconfig.get_paths()["purelib"], sysconfig.get_paths()["platlib"]):
        for rel in ("flashinfer/data/cutlass", "tilelang/3rdparty/cutlass"):
            p = os.path.join(base, rel)
            if os.path.isdir(os.path.join(p, "include", "cute")):
                return p
    raise RuntimeError("CUTLASS headers not found (flashinfer/data/cutlass)")


def nvcc_path() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    return "nvcc"


def build(verbose: bool = False, extra_flags=None) -> str:
    os.makedirs(LIBDIR, exist_ok=True)
    objs = []
    nvcc = nvcc_path()
    for src in SOURCES:
        path = os.path.join(CSRC, src)
        obj = os.path.join(LIBDIR, src.replace(".cu", ".o"))
        deps = [path] + [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".hpp"))]
        deps.append(os.path.join(INCLUDE, "pwgpu.h"))
        if not os.path.exists(obj) or os.path.getmtime(obj) < max(os.path.getmtime(d) for d in deps):
            cut = cutlass_root()
            cmd = [nvcc, *NVCC_FLAGS, *(extra_flags or []), "-I", INCLUDE, "-I", os.path.join(cut, "include"),
                   "-I", os.path.join(cut, "tools", "util", "include"), "-c", path, "-o", obj]
            if verbose:
                print(" ".join(cmd))
            subprocess.run(cmd, check=True)
        objs.append(obj)
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs):
        cmd = [nvcc, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", *objs, "-o", LIB,
               "-lcublas", "-lcusolver", "-lcudart"]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    print(build(verbose=True, extra_flags=sys.argv[1:]))

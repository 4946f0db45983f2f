"""Output files of a run: the density checkpoint and the band table.

The reference's deck carries `write_density` and `write_bands`
(OutputSettings, settings.rs:435-454) without a file format behind them;
these writers give them one.

Density checkpoint (.npz, numpy's zip of arrays):
  dims (3,), lattice (3, 3) rows a, b, c in Å, omega (Å^3), nspin,
  miller (n_pw, 3) of the basis, rho_r (nspin, N) in e/Å^3 on the FFT grid
  (x slowest, z fastest; up then down for nspin = 2), rho_g_fft (N complex,
  the total density as rho(G) = (1/N) sum_r rho(r) e^{-iG.r} on the same
  grid: the input of pwgpu_scf_iter1_from_rho_g, so a checkpoint restarts
  through one transplanted iteration), rho_g_basis (n_pw complex, the total
  rho(G) in basis order as ScfResult::rho_g, scf/mod.rs:269-322).

QE density bundle (read only): the VGCH2BIN files the reference's transplant
tests seed from (tests/vgch_transplant_c.rs:45-158): magic "VGCH2BIN",
u32 version 1, u8 gamma_only, i32 nspin, i32 ngm, the reciprocal vectors
(9 f64), ngm Miller triples (i32), nspin x ngm complex rho(G) in Bohr^-3,
all little-endian.

Band table (text): '#' header lines with the Fermi level and counts, then one
row per (spin, k-point): spin, k index, k (Å^-1, 3 numbers), weight, and
the n_bands eigenvalues in eV, ascending.
"""

from __future__ import annotations

import numpy as np

FORMAT_VERSION = 1


def density_to_g_fft(rho_r_total: np.ndarray, dims) -> np.ndarray:
    """rho(G) = (1/N) sum_r rho(r) e^{-iG.r} on the FFT grid (density_r_to_g,
    energy.rs:250-259), flattened in grid order."""
    n = int(np.prod(dims))
    return np.fft.fftn(np.asarray(rho_r_total, dtype=np.float64).reshape(dims)).ravel() / n


def write_density(path: str, sys_, rho_r: np.ndarray, rho_g_basis: np.ndarray | None = None) -> None:
    """Write the density checkpoint of system `sys_` (an ScfSystem) with its
    real-space density rho_r (nspin * N, as pwgpu_scf_run returns it)."""
    n = sys_.n_grid
    ns = sys_.nspin
    rho = np.asarray(rho_r, dtype=np.float64).reshape(ns, n)
    total = rho.sum(axis=0)
    lat = sys_.crystal.lattice
    g_fft = density_to_g_fft(total, sys_.dims)
    np.savez(path, format_version=FORMAT_VERSION, dims=np.array(sys_.dims, dtype=np.int64),
             lattice=np.array([lat.a, lat.b, lat.c], dtype=np.float64), omega=float(sys_.omega), nspin=ns,
             miller=np.asarray(sys_.basis.miller, dtype=np.int32), rho_r=rho, rho_g_fft=g_fft,
             rho_g_basis=(np.asarray(rho_g_basis, dtype=np.complex128) if rho_g_basis is not None
                          else g_fft[sys_.g_to_fft]))


def read_density(path: str) -> dict:
    """The arrays of a density checkpoint as a dict."""
    with np.load(path) as z:
        out = {k: z[k] for k in z.files}
    if int(out["format_version"]) != FORMAT_VERSION:
        raise ValueError(f"density checkpoint format {int(out['format_version'])} is not {FORMAT_VERSION}")
    out["dims"] = tuple(int(x) for x in out["dims"])
    out["omega"] = float(out["omega"])
    out["nspin"] = int(out["nspin"])
    return out


def restart_rho_g(sys_, checkpoint: dict) -> np.ndarray:
    """The checkpoint's full-grid rho(G) after checking that it belongs to a
    system with the same FFT grid and cell."""
    if tuple(checkpoint["dims"]) != tuple(sys_.dims):
        raise ValueError(f"checkpoint grid {checkpoint['dims']} differs from the system's {sys_.dims}")
    if abs(checkpoint["omega"] - sys_.omega) > 1e-9 * sys_.omega:
        raise ValueError("checkpoint cell volume differs from the system's")
    return checkpoint["rho_g_fft"]


def read_qe_density_bundle(path: str) -> dict:
    """Parse a VGCH2BIN density bundle: {"nspin", "miller" (ngm, 3) int,
    "rho_g" (nspin, ngm) complex in Bohr^-3}.  Raises ValueError on a bad
    magic, version, a Gamma-only bundle or a truncated file."""
    import struct
    with open(path, "rb") as f:
        b = f.read()
    if len(b) < 8 + 4 + 1 + 4 + 4 + 72 or b[:8] != b"VGCH2BIN":
        raise ValueError(f"{path}: not a VGCH2BIN bundle")
    off = 8
    (version,) = struct.unpack_from("<I", b, off)
    off += 4
    if version != 1:
        raise ValueError(f"{path}: unsupported VGCH2BIN version {version}")
    if b[off] != 0:
        raise ValueError(f"{path}: Gamma-only bundles are not supported")
    off += 1
    nspin, ngm = struct.unpack_from("<ii", b, off)
    off += 8 + 72
    if nspin < 1 or ngm < 1 or off + 12 * ngm + 16 * nspin * ngm > len(b):
        raise ValueError(f"{path}: truncated or inconsistent bundle")
    mill = np.frombuffer(b, dtype="<i4", count=3 * ngm, offset=off).reshape(ngm, 3).astype(np.int64)
    off += 12 * ngm
    rho = np.frombuffer(b, dtype="<c16", count=nspin * ngm, offset=off).reshape(nspin, ngm).astype(np.complex128)
    return {"nspin": nspin, "miller": mill, "rho_g": rho}


def qe_rho_g_on_grid(bundle: dict, dims, spin: int = 0) -> np.ndarray:
    """The bundle's rho(G) of one spin channel on the FFT grid in Å^-3,
    negative Miller indices wrapped (the scatter of tests/vgch_transplant_c.rs:
    125-153): the rho_g input of pwgpu_scf_iter1_from_rho_g."""
    from .consts import BOHR_TO_ANG
    d = np.asarray(dims, dtype=np.int64)
    m = bundle["miller"] % d
    idx = (m[:, 0] * d[1] + m[:, 1]) * d[2] + m[:, 2]
    out = np.zeros(int(np.prod(d)), dtype=np.complex128)
    out[idx] = bundle["rho_g"][spin] / BOHR_TO_ANG ** 3
    return out


def write_bands(path: str, sys_, eigenvalues: np.ndarray, fermi_energy: float) -> None:
    """Write the band table; eigenvalues [nspin * n_k, n_bands] as pwgpu_scf_run
    returns them (spin up k-points first)."""
    ev = np.asarray(eigenvalues, dtype=np.float64)
    nk = len(sys_.kpoints)
    ns = sys_.nspin
    if ev.ndim != 2 or ev.shape[0] != ns * nk:
        raise ValueError(f"eigenvalues have shape {ev.shape}; expected (nspin * n_k = {ns * nk}, n_bands)")
    with open(path, "w") as f:
        f.write(f"# pwgpu bands v{FORMAT_VERSION}\n")
        f.write(f"# fermi_energy_ev {fermi_energy:.12f}\n")
        f.write(f"# nspin {ns} n_k {nk} n_bands {ev.shape[1]}\n")
        f.write("# spin ik kx ky kz (1/Å) weight eigenvalues (eV)\n")
        for s in range(ns):
            for ik, kp in enumerate(sys_.kpoints):
                k = np.asarray(kp.k, dtype=np.float64)
                row = [f"{s}", f"{ik}", f"{k[0]:.12f}", f"{k[1]:.12f}", f"{k[2]:.12f}", f"{kp.weight:.12f}"]
                row += [f"{e:.10f}" for e in ev[s * nk + ik]]
                f.write(" ".join(row) + "\n")


def read_bands(path: str) -> dict:
    """Fermi level, k-points, weights and eigenvalues [nspin * n_k, n_bands] of a band table."""
    ef = None
    rows = []
    with open(path) as f:
        for line in f:
            if line.startswith("# fermi_energy_ev"):
                ef = float(line.split()[2])
            elif line.startswith("#") or not line.strip():
                continue
            else:
                rows.append([float(x) for x in line.split()])
    a = np.array(rows)
    return {"fermi_energy": ef, "spin": a[:, 0].astype(int), "ik": a[:, 1].astype(int), "k": a[:, 2:5],
            "weight": a[:, 5], "eigenvalues": a[:, 6:]}

"""Serving: the Python face of the pwgpu_server_* job queue and the seeded
request stream of the serving workload.

Stream: requests arrive as a Poisson process (seeded exponential gaps);
each samples Si or C diamond (50/50) with 2, 8, 16 or 64 atoms (weights
4:3:2:1; 2 = fcc primitive, 8 = conventional cube, 16 = conventional x
(2,1,1), 64 = x (2,2,2)), an isotropic strain U(-2 %, +2 %), seeded atomic
displacements U(-0.05, 0.05) bohr per component, ecutwfc uniform in
{20, 25, 30, 35} Ry, a Gamma-only or Gamma-centred 2x2x2 mesh (50/50,
reduced by the cell's symmetry), PZ-LDA, unpolarised, mixed precision.

The projector matrices, the local potential, the core density and the
start density of a request are built on the device from the UPF radial
data (pwgpu_create), not on the host.

SCF controls of a request: bands = N_el/2 + max(4, N_el/20); Gaussian
smearing 0.01 Ry; Anderson beta 0.4 + Kerker, 8 slots (the settings of the
64-atom benchmark solve, which converge the wide-gap C cells too); density
rms 1e-6 e/Å^3 and energy change 1e-5 eV (reference defaults).
"""

from __future__ import annotations

import ctypes as ct
import math
import threading
import time
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass

import numpy as np

from .consts import BOHR_TO_ANG, RY_TO_EV
from .context import build_system
from .crystal import Atom, Crystal, Lattice, diamond_primitive, diamond_supercell
from .lib import (PRECISION_MIXED, PWGPU_OK, PwgpuJobInfo, PwgpuScfResult, PwgpuServerOptions,
                  PwgpuServerStats, PwGpuError, _check, _f64, load_library, pack_system, scf_params)
from .symmetry import SymmetryInfo, reduce_kpoints

SEED = 20261203
LATTICE_BOHR = {"Si": 10.26, "C": 6.74}
SIZES = (2, 8, 16, 64)
SIZE_WEIGHTS = (4, 3, 2, 1)
ECUTS_RY = (20.0, 25.0, 30.0, 35.0)
SERVE_KW = dict(max_iter=100, conv_threshold=1e-6, energy_threshold=1e-5, mixing_beta=0.4, mixing_ndim=8,
                kerker=True, smearing="gaussian", sigma=0.01 * RY_TO_EV)


class Server:
    """pwgpu_server_*: submit systems, collect results (thread-safe)."""

    def __init__(self, device: int = 0, workers: int = 4, precision: int = PRECISION_MIXED, lanes_per_job: int = 2,
                 hbm_budget_bytes: int = 0):
        self.lib = load_library()
        opt = PwgpuServerOptions(device, workers, precision, lanes_per_job, hbm_budget_bytes)
        h = ct.c_void_p()
        _check(self.lib, self.lib.pwgpu_server_create(ct.byref(opt), ct.byref(h)))
        self.h = h
        self.shapes = {}
        self._lock = threading.Lock()

    def close(self):
        if self.h:
            self.lib.pwgpu_server_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def submit(self, sys_, n_bands: int, rho_init=None, **kw) -> int:
        st, keep = pack_system(sys_)
        p = scf_params(n_bands, **kw)
        rho0 = sys_.rho_init_r if rho_init is None else rho_init
        # None: the start density is built on the device with the local potential
        rho = None if rho0 is None else np.ascontiguousarray(rho0, dtype=np.float64)
        jid = ct.c_int64()
        _check(self.lib, self.lib.pwgpu_server_submit(self.h, ct.byref(st), ct.byref(p),
                                                      None if rho is None else _f64(rho), ct.byref(jid)))
        with self._lock:
            self.shapes[jid.value] = (sys_.nspin * len(sys_.kpoints), n_bands)
        return jid.value

    def poll(self, job_id: int) -> dict:
        info = PwgpuJobInfo()
        _check(self.lib, self.lib.pwgpu_server_poll(self.h, job_id, ct.byref(info)))
        return info.as_dict()

    def wait(self, job_id: int, timeout_s: float = 600.0) -> dict:
        info = PwgpuJobInfo()
        _check(self.lib, self.lib.pwgpu_server_wait(self.h, job_id, timeout_s, ct.byref(info)))
        return info.as_dict()

    def wait_any(self, timeout_s: float = 1.0):
        """Id of a finished, not yet collected job, or None on timeout."""
        jid = ct.c_int64()
        rc = self.lib.pwgpu_server_wait_any(self.h, timeout_s, ct.byref(jid))
        if rc == -5:
            return None
        _check(self.lib, rc)
        return jid.value

    def result(self, job_id: int):
        """(result dict, eigenvalues [nspin*n_k, n_bands], status, error message)."""
        with self._lock:
            nks, nb = self.shapes[job_id]
        res = PwgpuScfResult()
        ev = np.zeros((nks, nb))
        err = ct.c_char_p()
        _check(self.lib, self.lib.pwgpu_server_result(self.h, job_id, ct.byref(res), _f64(ev), ct.byref(err)))
        info = self.poll(job_id)
        return res.as_dict(), ev, info["status"], (err.value or b"").decode(errors="replace")

    def release(self, job_id: int):
        _check(self.lib, self.lib.pwgpu_server_release(self.h, job_id))
        with self._lock:
            self.shapes.pop(job_id, None)

    def stats(self) -> dict:
        st = PwgpuServerStats()
        _check(self.lib, self.lib.pwgpu_server_get_stats(self.h, ct.byref(st)))
        return st.as_dict()


@dataclass
class Request:
    index: int
    arrival_s: float
    species: str
    n_atoms: int
    strain: float
    ecut_ry: float
    kgrid: tuple
    seed: int


def request_stream(n: int, rate_per_s: float = 50.0, seed: int = SEED):
    """The first n requests of the seeded stream."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    w = np.array(SIZE_WEIGHTS, dtype=float)
    w /= w.sum()
    for i in range(n):
        t += rng.exponential(1.0 / rate_per_s)
        sp = "Si" if rng.random() < 0.5 else "C"
        na = int(rng.choice(SIZES, p=w))
        strain = float(rng.uniform(-0.02, 0.02))
        ecut = float(rng.choice(ECUTS_RY))
        kg = (1, 1, 1) if rng.random() < 0.5 else (2, 2, 2)
        out.append(Request(i, t, sp, na, strain, ecut, kg, int(rng.integers(1 << 31))))
    return out


def request_crystal(req: Request) -> Crystal:
    a = LATTICE_BOHR[req.species] * BOHR_TO_ANG * (1.0 + req.strain)
    if req.n_atoms == 2:
        cr = diamond_primitive(req.species, a)
    else:
        reps = {8: (1, 1, 1), 16: (2, 1, 1), 64: (2, 2, 2)}[req.n_atoms]
        cr = diamond_supercell(req.species, a, reps)
    rng = np.random.default_rng(req.seed)
    lat = cr.lattice
    m = np.array([lat.a, lat.b, lat.c]).T
    minv = np.linalg.inv(m)
    atoms = []
    for at in cr.atoms:
        d = rng.uniform(-0.05, 0.05, 3) * BOHR_TO_ANG
        f = np.array(at.frac) + minv @ d
        atoms.append(Atom(at.symbol, tuple(float(x) for x in f)))
    return Crystal(Lattice(lat.a, lat.b, lat.c), atoms)


def request_system(req: Request, pps: dict):
    """(ScfSystem, SCF keyword arguments) of one request."""
    cr = request_crystal(req)
    sym = SymmetryInfo.from_crystal(cr, 1e-5)
    kp = reduce_kpoints(req.kgrid, "gamma", sym, cr.lattice)
    s = build_system(cr, {req.species: pps[req.species]}, req.ecut_ry * RY_TO_EV, kp, sym, projectors_on_device=True,
                     local_on_device=True)
    nel = int(round(s.n_electrons))
    nb = nel // 2 + max(4, nel // 20)
    return s, dict(SERVE_KW, n_bands=nb)


def run_stream(server: Server, requests, pps: dict, setup_threads: int = 8, precision: int = PRECISION_MIXED,
               realtime: bool = True, keep_results: bool = True):
    """Replay requests against the server: each request's host setup starts at
    its arrival time (a setup thread pool), its job is submitted when the
    setup is done; a collector records completions.  Returns per-request
    records (arrival, submit, done times relative to the stream start, GPU
    queue/run seconds, energy, status)."""
    recs = {r.index: {"arrival_s": r.arrival_s, "species": r.species, "n_atoms": r.n_atoms, "ecut_ry": r.ecut_ry,
                      "kgrid": list(r.kgrid)} for r in requests}
    job_of = {}
    lock = threading.Lock()
    done = threading.Event()
    n_total = len(requests)
    t0 = time.perf_counter()

    def prepare(req):
        s, kw = request_system(req, pps)
        kw = dict(kw)
        nb = kw.pop("n_bands")
        jid = server.submit(s, nb, precision=precision, **kw)
        with lock:
            job_of[jid] = req.index
            recs[req.index].update(submit_s=time.perf_counter() - t0, n_pw=s.n_pw, n_k=len(s.kpoints),
                                   n_bands=nb, n_electrons=s.n_electrons)

    def collect():
        got = 0
        while got < n_total:
            jid = server.wait_any(1.0)
            if jid is None:
                continue
            now = time.perf_counter() - t0
            res, ev, status, err = server.result(jid)
            info = server.poll(jid)
            server.release(jid)
            while True:
                with lock:
                    idx = job_of.get(jid)
                if idx is not None:
                    break
                time.sleep(0.001)
            with lock:
                recs[idx].update(done_s=now, status=status, error=err, queue_s=info["queue_s"],
                                 run_s=info["run_s"], total_energy=res["total_energy"],
                                 n_iterations=res["n_iterations"], converged=res["converged"])
                if keep_results:
                    recs[idx]["eigenvalues"] = ev
            got += 1
        done.set()

    col = threading.Thread(target=collect, daemon=True)
    col.start()
    with ThreadPoolExecutor(max_workers=setup_threads) as pool:
        futs = []
        for req in requests:
            if realtime:
                delay = req.arrival_s - (time.perf_counter() - t0)
                if delay > 0:
                    time.sleep(delay)
            futs.append(pool.submit(prepare, req))
        for f in futs:
            f.result()
    done.wait()
    return [recs[r.index] for r in requests], time.perf_counter() - t0


def summarize(records, wall_s: float) -> dict:
    lat = np.array([r["done_s"] - r["arrival_s"] for r in records])
    gpu = np.array([r["queue_s"] + r["run_s"] for r in records])
    ok = [r for r in records if r.get("status") in (PWGPU_OK, -4)]
    return {"requests": len(records), "wall_s": wall_s, "solves_per_s": len(records) / wall_s,
            "latency_p50_s": float(np.percentile(lat, 50)), "latency_p99_s": float(np.percentile(lat, 99)),
            "server_latency_p50_s": float(np.percentile(gpu, 50)),
            "server_latency_p99_s": float(np.percentile(gpu, 99)),
            "converged": sum(1 for r in records if r.get("converged") == 1), "finished": len(ok)}

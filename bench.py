"""Benchmark of the SCF hot path on B200 (one JSON line on stdout).

Headline: SCF solves/s of the 64-atom Si cell (2x2x2 conventional cells of
a = 10.26 bohr, seeded ±0.05 bohr displacements, Si UPF, ecutwfc 30 Ry,
n_pw 23,847 on 72^3, Γ, 160 bands, Gaussian 0.01 Ry, Anderson beta 0.4 +
Kerker) run to convergence in the mixed batched form: four cells (four
displacement seeds) solved concurrently, each on its own handle and stream,
in the mixed precision form (FP32 FFT/V_eff product, FP64 subspace algebra
and energies, FP64 H|psi> after the density rms passes 1e-6).  Next to it
the plain FP64 form, one solve at a time, and |ΔE| per atom and the
eigenvalue deviation between the two forms on every cell.  One step = one
batch from the SAD start densities; its device time is CUDA events on a
side stream bracketing the batch (device-wide syncs on both sides), the
end-to-end time the same C-ABI calls by wall clock (they include the
host->device copies of the start densities and the device->host copies of
eigenvalues and densities).

Beside it: the plain FP64 form batched the same way (separating the gain of
the precision form from that of concurrency); the accuracy gate against the
FP64 oracle (one transplanted FP64 iteration from cell 0's converged
density handed to the oracle's H, occupations, density and energy, checker
only); end to end with pwgpu_create inside the clock; the plain-method case
(Si2, 10 k-points) as complete solves on the GPU and on the oracle over all
host cores; and the synthetic H|psi> kernel bench of the same cell (160
seeded bands, 256 Gaussian KB channels, V_eff seeded in [-1, 0] Ha) for the
per-stage device times and the roofline of the dominant own kernel.

The reference arm (--impl reference) times bounded samples of the headline
FP64 solve on the host cores (the oracle's H|psi> of 8 bands and their share
of the subspace products); its value is the solve fraction a step completes
over the step's measured time.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl pwgpu|reference]

Multi-GPU: one process per GPU (torchrun); every rank solves its own replica
(weak scaling: the solve has no cross-GPU exchange at this size), barrier,
max-over-ranks device time, aggregate solves/s.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "pwdft-rs_b200"))

import numpy as np  # noqa: E402

METRIC = "SCF solves/s (Si64 Γ 30 Ry, 160 bands; mixed vs FP64 plain GPU, |ΔE| per atom reported)"
UNIT = "solves/s"
HA_TO_EV = 27.211386245988
SI_UPF = os.path.join(ROOT, "tests", "golden", "upf", "Si.upf")
SEED = 20261203
BATCH = 4  # Si64 cells solved concurrently in one step
# k_xv<float> on the 72^3 grid, one 22-band launch in one ncu capture:
# dram__bytes_read.sum + dram__bytes_write.sum.  It is the compact input of
# each band plus one FP32 V(r) read (the output stays in L2), so it is scaled
# to a launch's band count as (capture - V) / 22 per band + V.
XV_TRAFFIC_CAPTURE = (33503744 + 3072, 22)
# the fused middle kernel (k_yxy_ct<float, 8, 9, 8, 9>) on the same grid:
# dram__bytes_read.sum + dram__bytes_write.sum of one 20-band launch from one
# ncu capture (the written planes stay in L2), scaled by a launch's bands
YXY_TRAFFIC_CAPTURE = (17050880, 20)


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), float(p["bf16_tflops"]), "measured"
    except Exception:
        return 6650.0, 1590.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.samples = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
                if out.returncode == 0:
                    self.samples.append([x.strip() for x in out.stdout.strip().split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *exc):
        self._stop.set()
        if self._t:
            self._t.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}

        def num(x):
            try:
                return float(x)
            except ValueError:
                return None
        sm = [v for v in (num(s[0]) for s in self.samples) if v is not None]
        mx = [v for v in (num(s[1]) for s in self.samples) if v is not None]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4)
                          if len(s) > 3 + i and s[3 + i].strip() == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def dist_env():
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def max_over_ranks(values, dist, device):
    """Element-wise maximum of per-rank timings (every rank gets the result);
    identity without a process group."""
    if dist is None:
        return list(values)
    import torch
    t = torch.tensor(list(values), device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.tolist()


def scf_kwargs():
    from pwgpu.config3 import FP64_SWITCH, SCF_KW, SOLVER_KW
    kw = dict(SCF_KW, **SOLVER_KW)
    nb = kw.pop("n_bands")
    return nb, kw, FP64_SWITCH


# Band applications of H in the FP64 device solve of the headline cell (the GPU
# arm measures it on every run and reports it under accuracy); the CPU arm's
# samples are fractions of a solve of this size.
HEADLINE_H_APPS = 12574
SAMPLE_BANDS = 8
SUBSPACE_ND = 180  # columns of the eigensolver block (160 bands + 20 buffer bands)


def sad_veff(sys_):
    """V_eff(G) of the start density, as the solve's first iteration builds it (for CPU sampling)."""
    from oracle import pwdft_oracle as O
    rho_g = O.density_r_to_g(sys_.rho_init_r, sys_.dims)
    _, vxc = O.lda_xc(O.add_core(sys_.rho_init_r, sys_.rho_core_r))
    return sys_.v_local_g + O.hartree(rho_g, sys_.g_squared) + O.density_r_to_g(vxc, sys_.dims)


class CpuSample:
    """One bounded sample step of the headline FP64 solve on the host cores:
    the oracle's H|psi> (FFT form + projector GEMMs) of SAMPLE_BANDS bands and
    those bands' share of the block eigensolver's subspace products (two
    projections against the 180-column block and the Rayleigh-Ritz update of
    a 540-column basis), all host threads through numpy/scipy.  A step is
    SAMPLE_BANDS band applications of a solve that needs h_apps of them."""

    def __init__(self, sys_):
        from oracle import pwdft_oracle as O
        O.set_workers(-1)
        self.O = O
        self.sys = sys_
        p = sys_.projectors[0]
        self.b, self.d = p.b, p.d_dense()
        self.veff = sad_veff(sys_)
        rng = np.random.default_rng(1)
        n = sys_.n_pw
        self.psi = rng.standard_normal((n, SAMPLE_BANDS)) + 1j * rng.standard_normal((n, SAMPLE_BANDS))
        self.x = np.linalg.qr(rng.standard_normal((n, SUBSPACE_ND)) + 0j)[0]
        self.v3 = rng.standard_normal((n, 3 * SUBSPACE_ND)) + 0j
        self.c3 = rng.standard_normal((3 * SUBSPACE_ND, SAMPLE_BANDS)) + 0j

    def step(self) -> float:
        s, O = self.sys, self.O
        t0 = time.perf_counter()
        h = O.apply_h_fft(s.g_to_fft, s.kinetic[0], self.veff, s.dims, self.b, self.d, self.psi)
        for _ in range(2):
            h = h - self.x @ (self.x.conj().T @ h)
        u = self.v3 @ self.c3
        t = time.perf_counter() - t0
        if not np.isfinite(u[0, 0]):
            raise RuntimeError("CPU sample produced non-finite values")
        return t

    def describe(self, h_apps, reps, step_s):
        return (f"one step = the oracle's FP64 H|psi> of {SAMPLE_BANDS} bands of the Si64 cell plus their share of "
                f"the eigensolver's subspace products ({reps} timed step(s), {step_s * 1e3:.1f} ms each); a solve "
                f"is {h_apps} band applications, so value = ({SAMPLE_BANDS}/{h_apps} solve) / step time; density, "
                "potentials, mixing and the dense subspace eigensolves are not counted (favours the CPU)")


def cpu_sample_baseline(sys_, h_apps, steps=3):
    smp = CpuSample(sys_)
    smp.step()  # warm
    ts = [smp.step() for _ in range(steps)]
    step_s = statistics.mean(ts)
    v = (SAMPLE_BANDS / h_apps) / step_s
    return {"value": v, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
            "sample": smp.describe(h_apps, steps, step_s), "projected_solve_s": step_s * h_apps / SAMPLE_BANDS}


def headline_config(sys_, nb, world):
    return {"workload": "si64_scf_gamma_30ry", "n_pw": sys_.n_pw, "grid": list(sys_.dims),
            "n_bands": nb, "n_ch": sys_.projectors[0].n_ch, "n_atoms": len(sys_.crystal.atoms),
            "smearing": "gaussian 0.01 Ry", "mixing": "anderson beta 0.4 + kerker",
            "batch": f"{BATCH} cells (displacement seeds {SEED}..{SEED + BATCH - 1}) solved "
                     "concurrently, one handle and stream each; a step = the batch",
            "l2": "flushed before every step (256 MB write); working set > L2",
            "parallelism": f"replicas x{world}"}


def run_reference(args, world, rank):
    """CPU arm: K bounded sample steps of the headline FP64 solve on the host
    cores (the oracle restatement of the reference's operator); value = the
    fraction of a solve each step completes / its measured time."""
    if rank != 0:
        return
    from pwgpu.config3 import config3_system
    from pwgpu.upf import load_upf
    sys_ = config3_system(load_upf(SI_UPF))
    nb = scf_kwargs()[0]
    smp = CpuSample(sys_)
    for _ in range(args.warmup):
        smp.step()
    ts = [smp.step() for _ in range(args.steps)]
    step_s = statistics.mean(ts)
    frac = SAMPLE_BANDS / HEADLINE_H_APPS
    v = frac / step_s
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": step_s * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "c128", "data": "synthetic (seeded Si64 cell)",
            "config": headline_config(sys_, nb, world),
            "solve_fraction_per_step": frac,
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
                             "sample": smp.describe(HEADLINE_H_APPS, args.steps, step_s),
                             "projected_solve_s": step_s / frac},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def config1_comparison(local):
    """The plain-method case as complete solves on both sides: the Si2 fcc cell
    (a = 10.26 bohr, 20 Ry, shifted 4x4x4 MP -> 10 IBZ k-points, 8 bands,
    Si_hgh.upf, fixed occupations, Anderson 0.7) from the SAD start density to
    convergence, FP64, through pwgpu_create + pwgpu_scf_run on the GPU and
    through the oracle's dense loop (the reference's algorithm) on every host
    core, its k-points spread over a process pool as the reference's rayon loop
    spreads them.  Both clocks are wall clocks around complete solves."""
    from pwgpu.config1 import SCF_KW, config1_system
    from pwgpu.lib import PRECISION_FP64, PwGpu
    from pwgpu.upf import load_upf
    s = config1_system(load_upf(os.path.join(ROOT, "tests", "golden", "upf", "Si_hgh.upf")))
    kw = dict(SCF_KW)
    nb = kw.pop("n_bands")
    gpu = []
    res = None
    for _ in range(3):
        t0 = time.perf_counter()
        with PwGpu(s, device=local) as dev:
            t1 = time.perf_counter()
            res, _, _, _ = dev.scf_run(s.rho_init_r, nb, precision=PRECISION_FP64, **kw)
        t2 = time.perf_counter()
        gpu.append((t2 - t0, t2 - t1))
    g_create, g_solve = min(x[0] for x in gpu[1:]), min(x[1] for x in gpu[1:])
    cpu = oracle_config1_solve(s, nb)
    if "unfinished" in cpu:
        return {"workload": "si2_fcc_20ry_mp444_10k_8bands_si_hgh", "gpu_solve_s": g_solve,
                "gpu_create_and_solve_s": g_create, "cpu_oracle_solve_s": None, "cpu_unfinished": cpu["unfinished"]}
    r, cpu_s, workers = cpu["result"], cpu["seconds"], cpu["workers"]
    return {"workload": "si2_fcc_20ry_mp444_10k_8bands_si_hgh", "n_pw": s.n_pw, "grid": list(s.dims),
            "n_k": len(s.kpoints), "gpu_solve_s": g_solve, "gpu_create_and_solve_s": g_create,
            "gpu_solves_per_s": 1.0 / g_solve, "gpu_solves_per_s_with_create": 1.0 / g_create,
            "cpu_oracle_solve_s": cpu_s, "cpu_solves_per_s": 1.0 / cpu_s, "cpu_processes": workers,
            "ratio_gpu_over_cpu": cpu_s / g_solve, "ratio_with_create": cpu_s / g_create,
            "dE_gpu_vs_oracle_ev": abs(res["total_energy"] - r.total_energy),
            "iterations_gpu": res["n_iterations"], "iterations_oracle": r.n_iterations,
            "note": "complete solves on both sides, measured (no projection); the CPU side is the oracle's "
                    "dense-H loop with one single-threaded process per k-point"}


_BLAS_ENV = ("OPENBLAS_NUM_THREADS", "OMP_NUM_THREADS", "MKL_NUM_THREADS")
CPU_SOLVE_LIMIT_S = 240.0


def stage(msg):
    """Progress of the bench's legs on stderr (the JSON line alone goes to stdout)."""
    print(f"[bench {time.strftime('%H:%M:%S')}] {msg}", file=sys.stderr, flush=True)


def oracle_config1_solve(s, nb):
    """The oracle's dense loop on the plain-method case over all host cores:
    one single-threaded process per k-point (spawned), bounded by
    CPU_SOLVE_LIMIT_S.  Returns {"result", "seconds", "workers"} or
    {"unfinished": why}."""
    import concurrent.futures
    import multiprocessing

    from oracle import pwdft_oracle as O
    from pwgpu.config1 import SCF_KW
    workers = min(len(s.kpoints), os.cpu_count() or 1)
    ctx = multiprocessing.get_context("spawn")
    # one BLAS thread per worker process: set in the environment the workers start with, before any
    # of them loads a BLAS library
    saved = {k: os.environ.get(k) for k in _BLAS_ENV}
    os.environ.update({k: "1" for k in _BLAS_ENV})
    try:
        pool = concurrent.futures.ProcessPoolExecutor(max_workers=workers, mp_context=ctx)
        list(pool.map(_noop, range(workers)))  # workers started before the clock
    finally:
        for k, v in saved.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v
    deadline = time.perf_counter() + CPU_SOLVE_LIMIT_S

    def kmap(fn, tasks):
        if time.perf_counter() > deadline:
            raise TimeoutError(f"the oracle's solve ran past {CPU_SOLVE_LIMIT_S} s")
        return pool.map(fn, tasks)

    kw2 = dict(SCF_KW)
    kw2.pop("n_bands")
    t0 = time.perf_counter()
    try:
        r = O.run_scf_unpolarized(s, nb, smearing=kw2.pop("smearing"), sigma=kw2.pop("sigma"), kmap=kmap, **kw2)
    except TimeoutError as e:
        pool.shutdown(cancel_futures=True)
        return {"unfinished": str(e)}
    cpu_s = time.perf_counter() - t0
    pool.shutdown()
    return {"result": r, "seconds": cpu_s, "workers": workers}


def _noop(_):
    return 0


def run_once():
    """Three H|psi> calls of the kernel-bench block per precision, mixed first
    (a short, bounded program for profiler captures)."""
    import torch

    from pwgpu.lib import PRECISION_FP64, PRECISION_MIXED, PwGpu
    from pwgpu.workloads import hpsi_system, si64_crystal
    sys_, veff_g, psi = hpsi_system(si64_crystal())
    nb, n_pw = psi.shape[1], sys_.n_pw
    with PwGpu(sys_) as dev:
        dev.set_veff_g(veff_g)
        d_psi = torch.from_numpy(np.ascontiguousarray(psi.T)).cuda()
        d_h = torch.empty_like(d_psi)
        for prec in (PRECISION_MIXED, PRECISION_FP64):
            dev.set_precision(prec)
            for _ in range(3):
                dev.apply_h_device(d_psi.data_ptr(), n_pw, nb, d_h.data_ptr(), n_pw)
        torch.cuda.synchronize()
    print("once: ok")


def run_scf_once():
    """One mixed-form solve of the headline cell (for profiler launch lists)."""
    from pwgpu.config3 import config3_system
    from pwgpu.lib import PRECISION_MIXED, PwGpu
    from pwgpu.upf import load_upf
    sys_ = config3_system(load_upf(SI_UPF))
    nb, kw, sw = scf_kwargs()
    with PwGpu(sys_) as dev:
        res, _, _, _ = dev.scf_run(sys_.rho_init_r, nb, precision=PRECISION_MIXED, fp64_switch=sw, **kw)
    print("scf once: ok", res["n_iterations"], res["total_energy"])


def run_dense():
    """The eigensolver's two dense kernels on seeded matrices of the Si64
    solve's subspace sizes, through the C-ABI (CUDA events around each
    launch, median of five after two warm-ups): the cluster eigensolver
    (lowest n_d = m/3 pairs, or all for m = 180) and the Cholesky factor with
    its inverse.  One JSON line; also the short program the dense-kernel
    profiler captures run."""
    import torch

    from pwgpu.lib import dense_cholesky_inverse, dense_eigh
    g = np.random.default_rng(SEED)
    out = {"mode": "dense", "eigh_ms": {}, "cholesky_inverse_ms": {}, "cusolver_syevd_ms": {},
           "cusolver_potrf_trsm_ms": {}, "cusolver_note": "torch.linalg (cuSOLVER) on the same matrices, "
           "all eigenpairs / Cholesky plus triangular inverse, CUDA events, for comparison only"}

    def torch_ms(fn, reps=5):
        for _ in range(2):
            fn()
        torch.cuda.synchronize()
        ts = []
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            fn()
            e1.record()
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1))
        return float(np.median(ts))

    for m in (180, 360, 540):
        nev = m if m <= 180 else m // 3
        a = g.standard_normal((m, m))
        a = a + a.T
        ts = [dense_eigh(a, nev, timed=True)[3] for _ in range(7)][2:]
        out["eigh_ms"][str(m)] = float(np.median(ts))
        ta = torch.tensor(a, device="cuda")
        out["cusolver_syevd_ms"][str(m)] = torch_ms(lambda: torch.linalg.eigh(ta))
    for q in (180, 360):
        y = g.standard_normal((3 * q, q))
        gm = y.T @ y
        ts = [dense_cholesky_inverse(gm, timed=True)[4] for _ in range(7)][2:]
        out["cholesky_inverse_ms"][str(q)] = float(np.median(ts))
        tg = torch.tensor(gm, device="cuda")
        eye = torch.eye(q, dtype=tg.dtype, device="cuda")
        out["cusolver_potrf_trsm_ms"][str(q)] = torch_ms(
            lambda: torch.linalg.solve_triangular(torch.linalg.cholesky(tg), eye, upper=False))
    print(json.dumps(out))


def config4_record(local: int) -> dict:
    """The batched-k LSDA case (Si8 and C8 conventional cells, 35 Ry, 20 IBZ
    k-points x 2 spins each, 24 bands, plain FP64 at the reference's default
    thresholds): each cell solved with its (spin, k) eigensolves on 8
    concurrent lanes and one at a time, device-synchronised wall time, kernel
    launches per SCF iteration, and |dE| against the committed oracle
    fixtures (converged to drho 1e-9, so the bar is the solve's own 1e-5 eV
    energy threshold)."""
    import torch

    from pwgpu.config4 import SCF_KW as C4_KW
    from pwgpu.config4 import config4_system
    from pwgpu.lib import PwGpu, kernel_launches
    from pwgpu.upf import load_upf
    out = {"workload": "si8_c8_lsda_35ry_6x6x6", "cells": {}}
    wall = {1: 0.0, 8: 0.0}
    for species, upf in (("Si", "Si.upf"), ("C", "C.upf")):
        s_, m = config4_system(species, load_upf(os.path.join(ROOT, "tests", "golden", "upf", upf)))
        with open(os.path.join(ROOT, "tests", "golden", f"config4_{species}_oracle.json")) as f:
            ref = json.load(f)
        kw = dict(C4_KW)
        nb = kw.pop("n_bands")
        rec = {"n_pw": s_.n_pw, "n_k": len(s_.kpoints)}
        for lanes in (8, 1):
            with PwGpu(s_, device=local, lanes=lanes) as dev:
                dev.scf_run(s_.rho_init_r, nb, starting_magnetization=m, **kw)  # warm-up
                torch.cuda.synchronize()
                n0 = kernel_launches()
                t0 = time.perf_counter()
                res, _, _, _ = dev.scf_run(s_.rho_init_r, nb, starting_magnetization=m, **kw)
                torch.cuda.synchronize()
                dt = time.perf_counter() - t0
                n1 = kernel_launches() - n0
            wall[lanes] += dt
            rec[f"lanes_{lanes}"] = {"s": dt, "scf_iterations": int(res["n_iterations"]),
                                     "launches_per_scf_iteration": n1 / max(1, int(res["n_iterations"])),
                                     "dE_vs_oracle_ev": abs(res["total_energy"] - ref["total_energy"]),
                                     "converged": bool(res["converged"])}
        out["cells"][species] = rec
    out["solves_per_s_lanes_8"] = 2.0 / wall[8]
    out["solves_per_s_sequential"] = 2.0 / wall[1]
    out["form"] = ("plain FP64; (spin, k) eigensolves of an SCF iteration on 8 host-thread lanes with a stream "
                   "each, against one at a time; the reference loops k with rayon (scf/driver.rs:461-472)")
    return out


def serving_record(n_requests: int, workers: int) -> dict:
    """Serving workload: the first n_requests requests of the seeded stream
    (Poisson 50/s; Si/C, 2-64 atoms, strain, displacements, 20-35 Ry, Gamma or
    2x2x2) replayed in real time through pwgpu_server_* (mixed precision);
    host setup of each request starts at its arrival on a thread pool.
    |dE| per atom against FP64 reruns of a seeded 5 % sample."""
    from pwgpu.lib import PRECISION_FP64, PRECISION_MIXED
    from pwgpu.serving import Server, request_stream, request_system, run_stream, summarize
    from pwgpu.upf import load_upf
    pps = {"Si": load_upf(SI_UPF), "C": load_upf(os.path.join(ROOT, "tests", "golden", "upf", "C.upf"))}
    reqs = request_stream(n_requests)
    with Server(workers=workers, precision=PRECISION_MIXED, lanes_per_job=2) as srv:
        recs, wall = run_stream(srv, reqs, pps, precision=PRECISION_MIXED)
        stats = srv.stats()
    summ = summarize(recs, wall)
    rng = np.random.default_rng(20261203)
    sample = sorted(rng.choice(len(reqs), size=max(1, len(reqs) // 20), replace=False).tolist())
    de = []
    with Server(workers=2, precision=PRECISION_FP64, lanes_per_job=2) as srv64:
        for i in sample:
            s, kw = request_system(reqs[i], pps)
            kw = dict(kw)
            nb = kw.pop("n_bands")
            jid = srv64.submit(s, nb, precision=PRECISION_FP64, **kw)
            srv64.wait(jid, 3600.0)
            res, ev, status, err = srv64.result(jid)
            srv64.release(jid)
            de.append(abs(res["total_energy"] - recs[i]["total_energy"]) / reqs[i].n_atoms)
    return {"workload": "serving_stream_poisson50", "requests": len(reqs), "arrival_rate_per_s": 50.0,
            "workers": workers, "lanes_per_job": 2, **summ, "server": stats,
            "accuracy": {"fp64_sample": len(sample), "max_dE_per_atom_ev": max(de) if de else None,
                         "max_dE_per_atom_ha": (max(de) / HA_TO_EV) if de else None,
                         "bar": "1e-6 Ha/atom against FP64 reruns"}}


def run_serve(args):
    """--mode serve: the serving record alone, as its own JSON line."""
    rec = serving_record(args.requests, args.workers)
    line = {"metric": "serving stream: SCF solves/s and latency (mixed precision)", "value": rec["solves_per_s"],
            "unit": "solves/s", "n_gpus": 1, "higher_is_better": True, "data": "synthetic (seeded request stream)",
            "config": {k: rec[k] for k in ("workload", "requests", "arrival_rate_per_s", "workers", "lanes_per_job")},
            **{k: v for k, v in rec.items() if k not in ("workload", "requests", "arrival_rate_per_s", "workers",
                                                          "lanes_per_job")}}
    print(json.dumps(line), flush=True)


def kernel_bench(local, steps, warmup, flush, hbm_peak, peak_kind):
    """H|psi> of the 160-band block (mixed and FP64): device ms per block and
    the per-stage profile; roofline of the dominant own kernel."""
    import torch

    from pwgpu.lib import PRECISION_FP64, PRECISION_MIXED, PwGpu
    from pwgpu.workloads import hpsi_algorithmic_bytes, hpsi_system, si64_crystal
    sys_, veff_g, psi = hpsi_system(si64_crystal())
    nb = psi.shape[1]
    n_pw, N = sys_.n_pw, sys_.n_grid
    out = {}
    with PwGpu(sys_, device=local) as dev:
        dev.set_veff_g(veff_g)
        d_psi = torch.from_numpy(np.ascontiguousarray(psi.T)).to(f"cuda:{local}")
        d_h = torch.empty_like(d_psi)
        stream = torch.cuda.Stream()
        for prec, tag in ((PRECISION_FP64, "fp64"), (PRECISION_MIXED, "mixed")):
            dev.set_precision(prec)
            ms = []
            with torch.cuda.stream(stream):
                for i in range(warmup + steps):
                    flush.fill_(float(i))
                    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    e0.record(stream)
                    dev.apply_h_device(d_psi.data_ptr(), n_pw, nb, d_h.data_ptr(), n_pw, stream=stream.cuda_stream)
                    e1.record(stream)
                    if i >= warmup:
                        ms.append((e0, e1))
            torch.cuda.synchronize()
            out[tag] = {"ms_per_block": statistics.mean(a.elapsed_time(b) for a, b in ms)}
        names = ["fft_z_inv_scatter", "fft_y_inv", "fft_x_mid", "fft_y_fwd", "fft_z_fwd_gather",
                 "nl_bh_psi_zgemm", "nl_d_apply", "nl_b_q_zgemm"]
        for prec, tag in ((PRECISION_MIXED, "mixed"), (PRECISION_FP64, "fp64")):
            dev.set_precision(prec)
            acc = np.zeros(8)
            for _ in range(3):
                flush.fill_(1.0)
                torch.cuda.synchronize()
                st_ms, st_n = dev.profile_apply_h(d_psi.data_ptr(), n_pw, nb, d_h.data_ptr(), n_pw)
                acc += st_ms
            acc /= 3
            out[tag]["stage_ms"] = dict(zip(names, [round(float(x), 5) for x in acc]))
            out[tag]["launches"] = dict(zip(names, [int(x) for x in st_n]))
    p = out["mixed"]
    own = {k: v for k, v in p["stage_ms"].items() if not k.endswith("zgemm") and p["launches"][k] > 0}
    dom = max(own, key=own.get)
    nl = max(1, p["launches"][dom])
    m = np.abs(sys_.basis.miller).max(axis=0)
    Xp, Yp = 2 * int(m[0]) + 1, 2 * int(m[1]) + 1
    d0, d1, d2 = sys_.dims
    cb = 8  # complex FP32 in the mixed form
    # fused middle kernel (one per z-plane and group of bands, the plane in shared memory) unless the
    # grid needed the three-kernel fallback
    fused = p["launches"]["fft_y_inv"] == 0
    bands = nb / nl
    per_launch = {
        "fft_z_inv_scatter": (16 * n_pw + cb * Xp * Yp * d2) * bands,
        "fft_y_inv": (cb * Xp * Yp * d2 + cb * Xp * d1 * d2) * bands,
        # fused: the middle kernel performs the x and y axes of both transforms and the V(r)
        # product, so it carries that share of the per-band algorithmic bytes of the local
        # H|psi> (2c n_pw + 4c N + (c/2) N): two thirds of the transforms' 4c N and the (c/2) N of
        # V(r); three-kernel form: the x pass's compact rows in and out and V(r) once per band
        "fft_x_mid": ((2.0 / 3.0) * 4 * cb * N + 0.5 * cb * N) * bands if fused
        else (2 * cb * Xp * d1 * d2 + 4.0 * N) * bands,
        "fft_y_fwd": (cb * Xp * d1 * d2 + cb * Xp * Yp * d2) * bands,
        "fft_z_fwd_gather": (cb * Xp * Yp * d2 + 3 * 16 * n_pw) * bands,
        "nl_d_apply": 2 * 16 * 256 * bands,
    }[dom]
    alg = per_launch
    ms_launch = own[dom] / nl
    achieved = alg / (ms_launch * 1e-3) / 1e9
    traffic = None
    if dom == "fft_x_mid" and not fused and (d0, d1, d2) == (72, 72, 72):
        cap, cap_bands = XV_TRAFFIC_CAPTURE
        v_bytes = 4.0 * N
        traffic = (cap - v_bytes) / cap_bands * bands + v_bytes
    elif dom == "fft_x_mid" and fused and (d0, d1, d2) == (72, 72, 72):
        cap, cap_bands = YXY_TRAFFIC_CAPTURE
        traffic = None if cap is None else cap / cap_bands * bands
    roofline = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
                "frac": achieved / hbm_peak,
                "traffic": traffic, "traffic_unit": "DRAM bytes per launch from one ncu capture, scaled by bands",
                "peak_kind": peak_kind,
                "alg_bytes_per_launch": alg, "ms_per_launch": ms_launch, "fused_middle": fused,
                "note": "dominant own kernel of H|psi> (the inner operator of every SCF step); fused middle "
                        "(y/x passes of both transforms and the V(r) product, the plane in shared memory): alg "
                        "bytes = its share of the local H|psi>'s per-band bytes, (2/3) 4c N + (c/2) N, c = 8 B"}
    if fused:
        comp = (2 * cb * Xp * Yp * d2) * bands + 4.0 * N
        roofline["compulsory_bytes_per_launch"] = comp
        roofline["compulsory_frac"] = comp / (ms_launch * 1e-3) / 1e9 / hbm_peak
        roofline["compulsory_note"] = ("what the fused kernel must move: the compact planes read and written once "
                                       "per band and V(r) once; it is bound by shared memory, not HBM")
    # the whole local H|psi> (the five FFT kernels) against its per-band algorithmic bytes
    # 2c n_pw + 4c N + (c/2) N, c = 8 B (FP32 complex)
    pipe_bytes = hpsi_algorithmic_bytes(n_pw, N, 8) * nb
    fft_stages = ("fft_z_inv_scatter", "fft_y_inv", "fft_x_mid", "fft_y_fwd", "fft_z_fwd_gather")
    pipe_ms = sum(p["stage_ms"][k] for k in fft_stages)
    pipe_gbs = pipe_bytes / (pipe_ms * 1e-3) / 1e9
    roofline["local_hpsi"] = {"bound": "hbm", "achieved": pipe_gbs, "peak": hbm_peak, "unit": "GB/s",
                              "frac": pipe_gbs / hbm_peak, "alg_bytes_per_block": pipe_bytes, "ms_per_block": pipe_ms,
                              "bands": nb,
                              "note": "five FFT kernels of one mixed H|psi> block, per-band bytes "
                                      "2c n_pw + 4c N + (c/2) N with c = 8 B"}
    return out, roofline, {"n_pw": n_pw, "grid": [d0, d1, d2], "n_bands": nb, "n_ch": 256}


def main():
    global BATCH
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="pwgpu", choices=["pwgpu", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--mode", default="full", choices=["full", "once", "scf-once", "serve", "dense"],
                    help="once: three untimed H|psi> calls per precision; scf-once: one mixed solve; "
                         "serve: the serving stream through pwgpu_server_* (own JSON line); "
                         "dense: the subspace eigensolver and Cholesky kernels alone (own JSON line)")
    ap.add_argument("--requests", type=int, default=200, help="serve: requests of the stream replayed")
    ap.add_argument("--workers", type=int, default=4, help="serve: concurrent jobs on the device")
    ap.add_argument("--serve-requests", type=int, default=60,
                    help="requests of the serving stream replayed after the headline (0: none)")
    ap.add_argument("--batch", type=int, default=BATCH, help="Si64 cells solved concurrently per step")
    ap.add_argument("--no-config4", action="store_true", help="skip the batched-k LSDA record")
    args = ap.parse_args()
    BATCH = max(1, args.batch)
    world, rank, local = dist_env()
    if args.mode == "serve":
        run_serve(args)
        return
    if args.mode == "once":
        run_once()
        return
    if args.mode == "scf-once":
        run_scf_once()
        return
    if args.mode == "dense":
        run_dense()
        return
    if args.impl == "reference":
        if world > 1:
            import torch.distributed as dist
            dist.init_process_group("gloo", init_method="env://")
        run_reference(args, world, rank)
        return
    args.warmup = max(args.warmup, 3)

    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", init_method="env://", timeout=datetime.timedelta(seconds=300))

    from pwgpu.config3 import config3_system
    from pwgpu.lib import PRECISION_FP64, PRECISION_MIXED, PwGpu, kernel_launches
    from pwgpu.upf import load_upf

    hbm_peak, bf16_peak, peak_kind = load_peaks()
    pp = load_upf(SI_UPF)
    nb, kw, sw = scf_kwargs()
    # the batch: BATCH cells of the workload (the canonical displacement seed
    # first, then the next seeds), each on its own handle and stream
    systems = [config3_system(pp)] + [config3_system(pp, seed=SEED + i) for i in range(1, BATCH)]
    sys_ = systems[0]
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{local}")
    devs = [PwGpu(s_, device=local, lanes=1) for s_ in systems]
    side = torch.cuda.Stream(device=f"cuda:{local}")

    def solve_one(i, prec, out):
        t0 = time.perf_counter()
        res, ev, rho, _ = devs[i].scf_run(systems[i].rho_init_r, nb, precision=prec, fp64_switch=sw,
                                          raise_on_unconverged=False, **kw)
        out[i] = (time.perf_counter() - t0, res, ev, rho)

    def solve_batch(prec, idx):
        """The solves of systems idx, concurrently (one host thread each);
        device time between events on a side stream after device-wide syncs."""
        flush.fill_(1.0)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(side)
        out = {}
        t0 = time.perf_counter()
        th = [threading.Thread(target=solve_one, args=(i, prec, out)) for i in idx]
        for t in th:
            t.start()
        for t in th:
            t.join()
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
        e1.record(side)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1), wall, out

    every = list(range(BATCH))
    stage("warm-up batches")
    for _ in range(args.warmup):
        solve_batch(PRECISION_MIXED, every)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    n0 = kernel_launches()
    stage("timed batches")
    with ClockSampler(local) as clk:
        runs = [solve_batch(PRECISION_MIXED, every) for _ in range(args.steps)]
    n_launch = kernel_launches() - n0
    # the plain FP64 form: one solve at a time, every cell once; then the FP64 form batched like the
    # headline, which separates the gain of the precision form from the gain of concurrency
    stage("FP64 solves")
    fp64_runs = [solve_batch(PRECISION_FP64, [i]) for i in every]
    fp64_batched = solve_batch(PRECISION_FP64, every)
    ms = statistics.mean(r[0] for r in runs)
    wall = statistics.mean(r[1] for r in runs)
    ms64 = statistics.mean(r[0] for r in fp64_runs)
    ms64b = fp64_batched[0]
    lat = sorted(o[0] for r in runs for o in r[2].values())
    ms, wall, ms64, ms64b = max_over_ranks([ms, wall, ms64, ms64b], dist, f"cuda:{local}")
    n_at = len(sys_.crystal.atoms)
    last = runs[-1][2]
    de = [abs(last[i][1]["total_energy"] - fp64_runs[i][2][i][1]["total_energy"]) / n_at / HA_TO_EV for i in every]
    dev_ev = [float(np.max(np.abs(last[i][2] - fp64_runs[i][2][i][2]))) / HA_TO_EV for i in every]
    rm, r64 = last[0][1], fp64_runs[0][2][0][1]
    accuracy = {"cells": BATCH, "dE_total_per_atom_ha": max(de), "max_eigenvalue_dev_ha": max(dev_ev),
                "bar": "|dE| <= 1e-6 Ha/atom, eigenvalues <= 1e-5 Ha vs the FP64 form (worst of the cells)",
                "e_total_mixed_ev": rm["total_energy"], "e_total_fp64_ev": r64["total_energy"],
                "iterations_mixed": rm["n_iterations"], "iterations_fp64": r64["n_iterations"],
                "h_band_applications_mixed": rm["h_applications"],
                "h_band_applications_fp64": r64["h_applications"],
                "converged_mixed": all(bool(last[i][1]["converged"]) for i in every),
                "converged_fp64": all(bool(fp64_runs[i][2][i][1]["converged"]) for i in every)}
    accuracy["gate_pass"] = bool(accuracy["converged_mixed"] and accuracy["converged_fp64"]
                                 and accuracy["dE_total_per_atom_ha"] <= 1e-6
                                 and accuracy["max_eigenvalue_dev_ha"] <= 1e-5)
    checker = rank == 0 and world == 1 and not args.no_cpu_baseline
    if checker:
        stage("oracle check of the headline cell")
        accuracy["vs_oracle"] = oracle_check(devs[0], sys_, fp64_runs[0][2][0], last[0], nb, kw)

    # end to end with the handle's creation inside the clock (the reference's run_scf builds its
    # ScfContext on every call): one more batch, each thread creating, solving and destroying
    for d in devs:
        d.close()
    out_c = {}

    def create_and_solve(i):
        t0 = time.perf_counter()
        with PwGpu(systems[i], device=local, lanes=1) as dv:
            res, _, _, _ = dv.scf_run(systems[i].rho_init_r, nb, precision=PRECISION_MIXED, fp64_switch=sw,
                                      raise_on_unconverged=False, **kw)
        out_c[i] = (time.perf_counter() - t0, res)

    stage("end to end with handle creation")
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    th = [threading.Thread(target=create_and_solve, args=(i,)) for i in every]
    for t in th:
        t.start()
    for t in th:
        t.join()
    torch.cuda.synchronize()
    wall_create = time.perf_counter() - t0
    stage("kernel bench")
    kb, roofline, kb_cfg = kernel_bench(local, 5, 3, flush, hbm_peak, peak_kind)

    cpu = None
    c1 = None
    if checker:
        stage("CPU sample of the headline solve")
        cpu = cpu_sample_baseline(sys_, int(r64["h_applications"]))
        stage("plain-method case: complete solves on GPU and CPU")
        c1 = config1_comparison(local)
    serving = None
    if rank == 0 and world == 1 and args.serve_requests > 0:
        stage(f"serving stream, first {args.serve_requests} requests")
        serving = serving_record(args.serve_requests, args.workers)
    c4 = None
    if rank == 0 and world == 1 and not args.no_config4:
        stage("batched-k LSDA case (config 4)")
        c4 = config4_record(local)
    stage("done")
    if rank == 0:
        value = world * BATCH * 1e3 / ms
        fp64_value = world * 1e3 / ms64
        fp64_b_value = world * BATCH * 1e3 / ms64b
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None,
            "dtype": "mixed: c64 FFT/V_eff product, f64 subspace/energies/mixing (Gamma-real bands)",
            "data": "synthetic (seeded Si64 cells; reference Si.upf)",
            "config": headline_config(sys_, nb, world),
            "latency_s": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                          "per": "solve, inside the concurrent batch"},
            "fp64": {"value": fp64_value, "unit": UNIT, "ms_per_step": ms64,
                     "form": "plain FP64, one solve at a time"},
            "fp64_batched": {"value": fp64_b_value, "unit": UNIT, "ms_per_step": ms64b,
                             "form": f"plain FP64, {BATCH} cells concurrently (as the headline)"},
            "mixed_batched_over_fp64_plain": value / fp64_value,
            "mixed_batched_over_fp64_batched": value / fp64_b_value,
            "accuracy": accuracy,
            "roofline": roofline,
            "kernel_bench": {"workload": "si64_hpsi_gamma_30ry", **kb_cfg, **kb},
            "gpu_launches": n_launch,
            "e2e": {"value": world * BATCH / wall, "unit": UNIT,
                    "h2d_bytes_per_step": int(BATCH * 8 * sys_.n_grid),
                    "d2h_bytes_per_step": int(BATCH * (8 * sys_.n_grid + 8 * nb + 16 * sys_.n_pw)),
                    "path": "pwgpu_scf_run per cell (C-ABI, host start density in, host eigenvalues/density out)",
                    "with_create": {"value": world * BATCH / wall_create, "unit": UNIT,
                                    "path": "pwgpu_create (device setup of projectors, V_loc, core and start "
                                            "densities) + pwgpu_scf_run + pwgpu_destroy per cell, one batch"}},
            "clocks": clk.summary(),
        }
        if cpu:
            line["cpu_baseline"] = cpu
        if c1:
            line["config1_complete_solves"] = c1
        if serving:
            line["serving"] = serving
        if c4:
            line["config4"] = c4
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def oracle_check(dev, sys_, fp64_out, mixed_out, nb, kw):
    """The headline cell against the FP64 oracle (checker, outside the timed
    region): one transplanted FP64 iteration from cell 0's converged FP64
    density on the device, handed to the oracle (its V_eff from that density,
    its FFT-form H on the device's bands, its occupations, density and total
    energy); the mixed solve of the same cell is compared with that energy and
    with the oracle's Rayleigh quotients."""
    from oracle import pwdft_oracle as O
    _, _, ev64, rho64 = fp64_out
    _, rmix, evmix, _ = mixed_out
    r1, ev1, _, _, rho_in1 = dev.scf_iter1_from_rho_g(O.density_r_to_g(rho64, sys_.dims), nb,
                                                       smearing=kw["smearing"], sigma=kw["sigma"], diag_tol=1e-9,
                                                       diag_max_iter=300)
    psi = dev.get_bands(nb)
    chk = O.fixed_point_check(sys_, rho_in1, psi, kw["smearing"], kw["sigma"])
    n_at = len(sys_.crystal.atoms)
    out = {"cell": 0,
           "dE_fp64_iteration_vs_oracle_ha": abs(chk["total_energy"] - r1["total_energy"]) / HA_TO_EV,
           "max_eigenvalue_dev_fp64_vs_oracle_ha": float(np.max(np.abs(chk["rayleigh"] - ev1[0]))) / HA_TO_EV,
           "max_residual_vs_oracle_h_ev": float(np.max(chk["residual"])),
           "drho_oracle_map_at_fixed_point": float(chk["drho_in_out"]),
           "dE_mixed_per_atom_vs_oracle_ha": abs(rmix["total_energy"] - chk["total_energy"]) / n_at / HA_TO_EV,
           "max_eigenvalue_dev_mixed_vs_oracle_ha": float(np.max(np.abs(evmix[0] - chk["rayleigh"]))) / HA_TO_EV,
           "bar": "plain FP64: 1e-8 Ha total, 1e-7 Ha eigenvalues; mixed: 1e-6 Ha/atom, 1e-5 Ha",
           "how": "one transplanted FP64 iteration from the converged FP64 density; the oracle rebuilds V_eff, "
                  "applies its FFT-form H to the device's bands, and builds occupations, density and energy"}
    out["gate_pass"] = bool(out["dE_fp64_iteration_vs_oracle_ha"] <= 1e-8
                            and out["max_eigenvalue_dev_fp64_vs_oracle_ha"] <= 1e-7
                            and out["dE_mixed_per_atom_vs_oracle_ha"] <= 1e-6
                            and out["max_eigenvalue_dev_mixed_vs_oracle_ha"] <= 1e-5)
    return out


if __name__ == "__main__":
    main()

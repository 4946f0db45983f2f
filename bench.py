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

Beside it, the synthetic H|psi> kernel bench of the same cell (160 seeded
bands, 256 Gaussian KB channels, V_eff seeded in [-1, 0] Ha) gives the
per-stage device times and the roofline of the dominant own kernel.

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
    from pwgpu.config3 import FP64_SWITCH, SCF_KW
    kw = dict(SCF_KW)
    nb = kw.pop("n_bands")
    return nb, kw, FP64_SWITCH


def sad_veff(sys_):
    """V_eff(G) of the start density, as the solve's first iteration builds it (for CPU sampling)."""
    from oracle import pwdft_oracle as O
    rho_g = O.density_r_to_g(sys_.rho_init_r, sys_.dims)
    _, vxc = O.lda_xc(O.add_core(sys_.rho_init_r, sys_.rho_core_r))
    return sys_.v_local_g + O.hartree(rho_g, sys_.g_squared) + O.density_r_to_g(vxc, sys_.dims)


def cpu_solve_sample(sys_, h_applications: int, nb_sample: int = 8):
    """Oracle FP64 H|psi> (FFT form + projector GEMMs, all host threads) on a
    band sample, scaled by the band applications of the FP64 GPU solve."""
    from oracle import pwdft_oracle as O
    O.set_workers(-1)
    p = sys_.projectors[0]
    d = p.d_dense()
    veff = sad_veff(sys_)
    rng = np.random.default_rng(1)
    psi = rng.standard_normal((sys_.n_pw, nb_sample)) + 1j * rng.standard_normal((sys_.n_pw, nb_sample))
    O.apply_h_fft(sys_.g_to_fft, sys_.kinetic[0], veff, sys_.dims, p.b, d, psi[:, :1])  # warm
    t0 = time.perf_counter()
    reps = 0
    while True:
        O.apply_h_fft(sys_.g_to_fft, sys_.kinetic[0], veff, sys_.dims, p.b, d, psi)
        reps += 1
        if time.perf_counter() - t0 > 10.0 or reps >= 3:
            break
    per_band = (time.perf_counter() - t0) / reps / nb_sample
    solve_s = per_band * h_applications
    return {"value": 1.0 / solve_s, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
            "sample": (f"oracle FP64 H|psi> on {nb_sample} bands x {reps} rep(s) ({per_band * 1e3:.2f} ms/band), "
                       f"scaled by the {h_applications} band applications of the FP64 GPU solve; "
                       "subspace algebra, density and potentials not counted (lower bound on CPU time)")}


def run_reference(args, world, rank):
    """CPU arm: the oracle restatement of the reference's per-iteration operator
    on all host cores, bounded samples scaled to one solve."""
    if rank != 0:
        return
    from pwgpu.config3 import config3_system
    from pwgpu.upf import load_upf
    sys_ = config3_system(load_upf(SI_UPF))
    h_apps = 12574  # band applications of the FP64 GPU solve of this cell (measured, bench "accuracy" block)
    vals = []
    base = None
    for i in range(args.warmup + args.steps):
        base = cpu_solve_sample(sys_, h_apps, nb_sample=4)
        if i >= args.warmup:
            vals.append(1.0 / base["value"])
    v = 1.0 / statistics.mean(vals)
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 / v, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "c128", "data": "synthetic (seeded Si64 cell)",
            "config": {"workload": "si64_scf_gamma_30ry", "n_pw": sys_.n_pw, "grid": list(sys_.dims),
                       "n_bands": 160, "n_ch": sys_.projectors[0].n_ch},
            "cpu_baseline": {**base, "value": v},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


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


def run_serve(args):
    """Serving workload: the first --requests requests of the seeded stream
    (Poisson 50/s; Si/C, 2-64 atoms, strain, displacements, 20-35 Ry, Gamma or
    2x2x2) replayed in real time through pwgpu_server_* (mixed precision);
    host setup of each request starts at its arrival on a thread pool.
    |dE| per atom against FP64 reruns of a seeded 5 % sample."""
    from pwgpu.lib import PRECISION_FP64, PRECISION_MIXED
    from pwgpu.serving import Server, request_stream, request_system, run_stream, summarize
    from pwgpu.upf import load_upf
    pps = {"Si": load_upf(SI_UPF), "C": load_upf(os.path.join(ROOT, "tests", "golden", "upf", "C.upf"))}
    reqs = request_stream(args.requests)
    with Server(workers=args.workers, precision=PRECISION_MIXED, lanes_per_job=2) as srv:
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
    line = {"metric": "serving stream: SCF solves/s and latency (mixed precision)", "value": summ["solves_per_s"],
            "unit": "solves/s", "n_gpus": 1, "higher_is_better": True, "data": "synthetic (seeded request stream)",
            "config": {"workload": "serving_stream_poisson50", "requests": len(reqs),
                       "arrival_rate_per_s": 50.0, "workers": args.workers, "lanes_per_job": 2},
            **summ, "server": stats,
            "accuracy": {"fp64_sample": len(sample), "max_dE_per_atom_ev": max(de) if de else None,
                         "max_dE_per_atom_ha": (max(de) / HA_TO_EV) if de else None}}
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
        names = ["fft_z_inv_scatter", "fft_y_inv", "fft_x_inv_v_fwd", "fft_y_fwd", "fft_z_fwd_gather",
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
    own = {k: v for k, v in p["stage_ms"].items() if not k.endswith("zgemm")}
    dom = max(own, key=own.get)
    nl = max(1, p["launches"][dom])
    m = np.abs(sys_.basis.miller).max(axis=0)
    Xp, Yp = 2 * int(m[0]) + 1, 2 * int(m[1]) + 1
    d0, d1, d2 = sys_.dims
    cb = 8  # complex FP32 in the mixed form
    per_band = {
        "fft_z_inv_scatter": 16 * n_pw + cb * Xp * Yp * d2,
        "fft_y_inv": cb * Xp * Yp * d2 + cb * Xp * d1 * d2,
        "fft_x_inv_v_fwd": 2 * cb * Xp * d1 * d2 + 4.0 * N / (nb / nl),
        "fft_y_fwd": cb * Xp * d1 * d2 + cb * Xp * Yp * d2,
        "fft_z_fwd_gather": cb * Xp * Yp * d2 + 3 * 16 * n_pw,
        "nl_d_apply": 2 * 16 * 256,
    }[dom]
    alg = per_band * nb / nl
    ms_launch = own[dom] / nl
    achieved = alg / (ms_launch * 1e-3) / 1e9
    traffic = None
    if dom == "fft_x_inv_v_fwd" and (d0, d1, d2) == (72, 72, 72):
        cap, cap_bands = XV_TRAFFIC_CAPTURE
        v_bytes = 4.0 * N
        traffic = (cap - v_bytes) / cap_bands * (nb / nl) + v_bytes
    roofline = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
                "frac": achieved / hbm_peak,
                # DRAM bytes of the mixed x-pass kernel from one ncu capture of a 22-band launch,
                # scaled to this launch's average band count
                "traffic": traffic, "traffic_unit": "bytes per launch (ncu capture of 22 bands, scaled by bands)",
                "peak_kind": peak_kind,
                "alg_bytes_per_launch": alg, "ms_per_launch": ms_launch,
                "note": "dominant own kernel of H|psi> (the inner operator of every SCF step); "
                        "alg bytes = compact-grid read+write per band x bands per launch, V(r) FP32 read"}
    # the whole local H|psi> (the five FFT kernels) against its per-band algorithmic bytes
    # 2c n_pw + 4c N + (c/2) N, c = 8 B (FP32 complex)
    pipe_bytes = hpsi_algorithmic_bytes(n_pw, N, 8) * nb
    fft_stages = ("fft_z_inv_scatter", "fft_y_inv", "fft_x_inv_v_fwd", "fft_y_fwd", "fft_z_fwd_gather")
    pipe_ms = sum(p["stage_ms"][k] for k in fft_stages)
    pipe_gbs = pipe_bytes / (pipe_ms * 1e-3) / 1e9
    roofline["local_hpsi"] = {"bound": "hbm", "achieved": pipe_gbs, "peak": hbm_peak, "unit": "GB/s",
                              "frac": pipe_gbs / hbm_peak, "alg_bytes_per_block": pipe_bytes, "ms_per_block": pipe_ms,
                              "bands": nb,
                              "note": "five FFT kernels of one mixed H|psi> block, per-band bytes "
                                      "2c n_pw + 4c N + (c/2) N with c = 8 B"}
    return out, roofline, {"n_pw": n_pw, "grid": [d0, d1, d2], "n_bands": nb, "n_ch": 256}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="pwgpu", choices=["pwgpu", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--mode", default="full", choices=["full", "once", "scf-once", "serve"],
                    help="once: three untimed H|psi> calls per precision; scf-once: one mixed solve; "
                         "serve: the serving stream through pwgpu_server_* (own JSON line)")
    ap.add_argument("--requests", type=int, default=200, help="serve: requests of the stream replayed")
    ap.add_argument("--workers", type=int, default=4, help="serve: concurrent jobs on the device")
    args = ap.parse_args()
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
        res, ev, _, _ = devs[i].scf_run(systems[i].rho_init_r, nb, precision=prec, fp64_switch=sw,
                                        raise_on_unconverged=False, **kw)
        out[i] = (time.perf_counter() - t0, res, ev)

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
    for _ in range(args.warmup):
        solve_batch(PRECISION_MIXED, every)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    n0 = kernel_launches()
    with ClockSampler(local) as clk:
        runs = [solve_batch(PRECISION_MIXED, every) for _ in range(args.steps)]
    n_launch = kernel_launches() - n0
    # the plain FP64 form: one solve at a time, every cell once
    fp64_runs = [solve_batch(PRECISION_FP64, [i]) for i in every]
    ms = statistics.mean(r[0] for r in runs)
    wall = statistics.mean(r[1] for r in runs)
    ms64 = statistics.mean(r[0] for r in fp64_runs)
    lat = sorted(o[0] for r in runs for o in r[2].values())
    ms, wall, ms64 = max_over_ranks([ms, wall, ms64], dist, f"cuda:{local}")
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

    for d in devs:
        d.close()
    kb, roofline, kb_cfg = kernel_bench(local, 5, 3, flush, hbm_peak, peak_kind)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_solve_sample(sys_, int(r64["h_applications"]))
    if rank == 0:
        value = world * BATCH * 1e3 / ms
        fp64_value = world * 1e3 / ms64
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None,
            "dtype": "mixed: c64 FFT/V_eff product, c128 projector GEMMs, f64 subspace/energies/mixing",
            "data": "synthetic (seeded Si64 cells; reference Si.upf)",
            "config": {"workload": "si64_scf_gamma_30ry", "n_pw": sys_.n_pw, "grid": list(sys_.dims),
                       "n_bands": nb, "n_ch": sys_.projectors[0].n_ch, "n_atoms": n_at,
                       "smearing": "gaussian 0.01 Ry", "mixing": "anderson beta 0.4 + kerker",
                       "batch": f"{BATCH} cells (displacement seeds {SEED}..{SEED + BATCH - 1}) solved "
                                "concurrently, one handle and stream each; a step = the batch",
                       "l2": "flushed before every step (256 MB write); working set > L2",
                       "parallelism": f"replicas x{world}"},
            "latency_s": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                          "per": "solve, inside the concurrent batch"},
            "fp64": {"value": fp64_value, "unit": UNIT, "ms_per_step": ms64,
                     "form": "plain FP64, one solve at a time"},
            "mixed_batched_over_fp64_plain": value / fp64_value,
            "accuracy": accuracy,
            "roofline": roofline,
            "kernel_bench": {"workload": "si64_hpsi_gamma_30ry", **kb_cfg, **kb},
            "gpu_launches": n_launch,
            "e2e": {"value": world * BATCH / wall, "unit": UNIT,
                    "h2d_bytes_per_step": int(BATCH * 8 * sys_.n_grid),
                    "d2h_bytes_per_step": int(BATCH * (8 * sys_.n_grid + 8 * nb + 16 * sys_.n_pw)),
                    "path": "pwgpu_scf_run per cell (C-ABI, host start density in, host eigenvalues/density out)"},
            "clocks": clk.summary(),
        }
        if cpu:
            line["cpu_baseline"] = cpu
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()

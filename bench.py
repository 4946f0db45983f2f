"""Benchmark of the SCF hot path on B200 (one JSON line on stdout).

Workload: the synthetic H|psi> kernel bench -- 64-atom Si cubic supercell,
Γ, ecutwfc 30 Ry (n_pw 23,847, 72^3 grid), 160 bands, 256 KB channels,
seeded inputs (pwgpu.workloads.hpsi_system).  One step = one H|psi> of the
160-band block, inputs resident in HBM, L2 flushed (256 MB write) before
every timed step.  `value` is the mixed form (FP32 FFT / V_eff product);
the FP64 plain form is reported beside it.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl pwgpu|reference]

Multi-GPU: one process per GPU (torchrun), independent replicas of the
workload (the path has no cross-GPU exchange at this size), barrier and
max-over-ranks device time.
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

METRIC = "H|psi> 160-band blocks/s (Si64 Γ 30 Ry synthetic kernel bench of the SCF solves/s metric)"
UNIT = "blocks/s"


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
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if len(s) > 3 + i and "Active" in s[3 + i]
                          and "Not" not in s[3 + i]})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def cpu_baseline_sample(sys_, veff_g, psi, nb_sample=8):
    """Oracle FP64 H|psi> (FFT form, all host threads) on a band sample."""
    from oracle import pwdft_oracle as O
    O.set_workers(-1)
    p = sys_.projectors[0]
    d = p.d_dense()
    sub = np.ascontiguousarray(psi[:, :nb_sample])
    O.apply_h_fft(sys_.g_to_fft, sys_.kinetic[0], veff_g, sys_.dims, p.b, d, sub[:, :1])  # warm
    t0 = time.perf_counter()
    reps = 0
    while True:
        O.apply_h_fft(sys_.g_to_fft, sys_.kinetic[0], veff_g, sys_.dims, p.b, d, sub)
        reps += 1
        if time.perf_counter() - t0 > 10.0 or reps >= 3:
            break
    dt = (time.perf_counter() - t0) / reps
    per_block = dt * psi.shape[1] / nb_sample
    return {"value": 1.0 / per_block, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
            "sample": f"{nb_sample} of {psi.shape[1]} bands, {reps} rep(s), scaled to a 160-band block"}


def run_reference(args, world, rank):
    if rank != 0:
        return
    from pwgpu.workloads import hpsi_system, si64_crystal
    sys_, veff_g, psi = hpsi_system(si64_crystal())
    times = []
    base = None
    for i in range(args.warmup + args.steps):
        b = cpu_baseline_sample(sys_, veff_g, psi, nb_sample=4)
        if i >= args.warmup:
            times.append(1.0 / b["value"])
        base = b
    v = 1.0 / statistics.mean(times)
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 / v, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "c128", "data": "synthetic",
            "config": {"workload": "si64_hpsi_gamma_30ry", "n_pw": sys_.n_pw, "grid": list(sys_.dims),
                       "n_bands": 160, "n_ch": 256},
            "cpu_baseline": {**base, "value": v},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_once():
    """Three H|psi> calls of the bench workload per precision, mixed first
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


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="pwgpu", choices=["pwgpu", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--mode", default="full", choices=["full", "once"],
                    help="once: three untimed H|psi> calls per precision (for profiler captures)")
    args = ap.parse_args()
    world, rank, local = dist_env()
    if args.mode == "once":
        run_once()
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
        dist.init_process_group("nccl", init_method="env://", timeout=datetime.timedelta(seconds=120))

    from pwgpu.lib import PRECISION_FP64, PRECISION_MIXED, PwGpu
    from pwgpu.workloads import hpsi_algorithmic_bytes, hpsi_system, nonlocal_flops, si64_crystal

    sys_, veff_g, psi = hpsi_system(si64_crystal())
    nb = psi.shape[1]
    n_pw, N = sys_.n_pw, sys_.n_grid
    dev = PwGpu(sys_, device=local)
    dev.set_veff_g(veff_g)
    d_psi = torch.from_numpy(np.ascontiguousarray(psi.T)).to(f"cuda:{local}")  # row b = band b (column-major view)
    d_h = torch.empty_like(d_psi)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{local}")
    stream = torch.cuda.Stream()

    def timed(precision, steps, warmup):
        dev.set_precision(precision)
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
        return [a.elapsed_time(b) for a, b in ms]

    hbm_peak, bf16_peak, peak_kind = load_peaks()
    # untimed correctness spot check against the FP64 form
    timed(PRECISION_FP64, 1, 0)
    ref_h = d_h.clone()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        t64 = timed(PRECISION_FP64, args.steps, args.warmup)
        t32 = timed(PRECISION_MIXED, args.steps, args.warmup)
    mixed_err = float((d_h - ref_h).abs().max() / ref_h.abs().max())
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    ms32 = statistics.mean(t32)
    ms64 = statistics.mean(t64)
    if dist:
        t = torch.tensor([ms32, ms64], device=f"cuda:{local}", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms32, ms64 = t.tolist()

    # per-stage profile (events after every launch, on the handle's stream)
    stage_names = ["fft_z_inv_scatter", "fft_y_inv", "fft_x_inv_v_fwd", "fft_y_fwd", "fft_z_fwd_gather",
                   "nl_bh_psi_zgemm", "nl_d_apply", "nl_b_q_zgemm"]
    prof = {}
    launches = 0
    for prec, tag in ((PRECISION_MIXED, "mixed"), (PRECISION_FP64, "fp64")):
        dev.set_precision(prec)
        acc = np.zeros(8)
        for _ in range(3):
            flush.fill_(1.0)
            torch.cuda.synchronize()
            st_ms, st_n = dev.profile_apply_h(d_psi.data_ptr(), n_pw, nb, d_h.data_ptr(), n_pw)
            acc += st_ms
        acc /= 3
        prof[tag] = {"stage_ms": dict(zip(stage_names, [round(x, 5) for x in acc])),
                     "launches": dict(zip(stage_names, [int(x) for x in st_n]))}
        if tag == "mixed":
            launches = int(st_n[[0, 1, 2, 3, 4, 6]].sum())

    # roofline of the dominant own kernel in the mixed form (HBM-bound FFT stage)
    g = dev_grid = None
    p = prof["mixed"]
    own = {k: v for k, v in p["stage_ms"].items() if not k.endswith("zgemm")}
    dom = max(own, key=own.get)
    dom_ms_per_launch = own[dom] / max(1, p["launches"][dom])
    cb = 8  # complex FP32 in the mixed form
    from pwgpu.crystal import BasisSet  # noqa: F401
    m = np.abs(sys_.basis.miller).max(axis=0)
    Xp, Yp = 2 * m[0] + 1, 2 * m[1] + 1
    d0, d1, d2 = sys_.dims
    nb_launch = nb / max(1, p["launches"][dom])
    per_band = {
        "fft_z_inv_scatter": 16 * n_pw + cb * Xp * Yp * d2,
        "fft_y_inv": cb * Xp * Yp * d2 + cb * Xp * d1 * d2,
        "fft_x_inv_v_fwd": 2 * cb * Xp * d1 * d2 + 4 * N / nb,
        "fft_y_fwd": cb * Xp * d1 * d2 + cb * Xp * Yp * d2,
        "fft_z_fwd_gather": cb * Xp * Yp * d2 + 3 * 16 * n_pw,
        "nl_d_apply": 2 * 16 * 256,
    }[dom]
    alg_bytes = per_band * nb_launch
    achieved = alg_bytes / (dom_ms_per_launch * 1e-3) / 1e9
    roofline = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
                "frac": achieved / hbm_peak, "traffic": None, "peak_kind": peak_kind,
                "alg_bytes_per_launch": alg_bytes, "ms_per_launch": dom_ms_per_launch}

    # end to end through the C-ABI with host buffers (pinned), mixed form
    dev.set_precision(PRECISION_MIXED)
    h_psi = torch.from_numpy(np.ascontiguousarray(psi.T)).pin_memory()
    h_out = torch.empty_like(h_psi).pin_memory()
    import ctypes as ct
    lib = dev.lib
    f64p = ct.POINTER(ct.c_double)
    e2e_t = []
    for i in range(args.warmup + args.steps):
        flush.fill_(float(i))
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        rc = lib.pwgpu_apply_h(dev.h, 0, 0, ct.cast(h_psi.data_ptr(), f64p), nb, ct.cast(h_out.data_ptr(), f64p))
        t1 = time.perf_counter()
        if rc != 0:
            raise RuntimeError(lib.pwgpu_last_error())
        if i >= args.warmup:
            e2e_t.append(t1 - t0)
    e2e_s = statistics.mean(e2e_t)
    if dist:
        t = torch.tensor([e2e_s], device=f"cuda:{local}", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = t.item()

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline_sample(sys_, veff_g, psi)

    if rank == 0:
        nl_gflop = nonlocal_flops(n_pw, 256, nb) / 1e9
        line = {
            "metric": METRIC, "value": world * 1e3 / ms32, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms32, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "c64 FFT/V_eff + c128 projector GEMMs (mixed form)",
            "data": "synthetic (seeded; shapes of the Si64 Γ 30 Ry kernel bench)",
            "config": {"workload": "si64_hpsi_gamma_30ry", "n_pw": n_pw, "grid": [d0, d1, d2], "n_bands": nb,
                       "n_ch": 256, "l2": "flushed before every timed step (256 MB write)",
                       "parallelism": f"replicas x{world}"},
            "fp64": {"value": world * 1e3 / ms64, "unit": UNIT, "ms_per_step": ms64},
            "mixed_vs_fp64_max_rel_err": mixed_err,
            "roofline": roofline,
            "stages": prof,
            "gpu_launches": launches * args.steps,
            "e2e": {"value": world / e2e_s, "unit": UNIT, "h2d_bytes_per_step": int(16 * n_pw * nb),
                    "d2h_bytes_per_step": int(16 * n_pw * nb), "path": "pwgpu_apply_h (C-ABI, pinned host)"},
            "nonlocal_gflop_per_step": nl_gflop,
            "alg_local_bytes_per_step_fp32": hpsi_algorithmic_bytes(n_pw, N, 8) * nb,
            "clocks": clk.summary(),
        }
        if cpu:
            line["cpu_baseline"] = cpu
        print(json.dumps(line), flush=True)
    dev.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()

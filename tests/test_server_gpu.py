"""The serving job queue (pwgpu_server_*): results equal direct
pwgpu_scf_run calls on the same systems, admission keeps the estimated
footprint of running jobs within the budget, oversized jobs are refused,
every finished job is handed out once, and a short wait times out."""

import numpy as np
import pytest

from pwgpu.context import build_system
from pwgpu.crystal import KPoint, diamond_primitive, gamma_only
from pwgpu.lib import PRECISION_FP64, PwGpu, PwGpuError
from pwgpu.serving import Server, request_stream, request_system

pytestmark = pytest.mark.gpu

KW = dict(max_iter=80, conv_threshold=1e-7, energy_threshold=1e-6, mixing_beta=0.3, smearing="fermi_dirac",
          sigma=0.05)


def systems(si_pp, c_pp):
    return [
        (build_system(diamond_primitive("Si", 5.431), {"Si": si_pp}, 100.0, gamma_only(), fft_grid=(16, 16, 16)), 6),
        (build_system(diamond_primitive("C", 3.5667), {"C": c_pp}, 200.0, gamma_only()), 6),
        (build_system(diamond_primitive("Si", 5.431), {"Si": si_pp}, 120.0,
                      [KPoint(np.array([0.1, 0.05, -0.2]), 0.5), KPoint(np.array([0.0, 0.0, 0.0]), 0.5)]), 8),
    ]


def test_server_results_match_direct_runs(si_pp, c_pp):
    cases = systems(si_pp, c_pp)
    direct = []
    for s, nb in cases:
        with PwGpu(s, lanes=2) as dev:
            res, ev, _, _ = dev.scf_run(s.rho_init_r, nb, precision=PRECISION_FP64, **KW)
        direct.append((res, ev))
    with Server(workers=3, precision=PRECISION_FP64) as srv:
        ids = [srv.submit(s, nb, precision=PRECISION_FP64, **KW) for s, nb in cases]
        seen = set()
        while len(seen) < len(ids):
            jid = srv.wait_any(60.0)
            assert jid is not None and jid not in seen
            seen.add(jid)
        assert srv.wait_any(0.05) is None  # each finished job is handed out once
        for jid, (res0, ev0) in zip(ids, direct):
            res, ev, status, err = srv.result(jid)
            assert status == 0, err
            assert abs(res["total_energy"] - res0["total_energy"]) < 1e-6
            assert np.max(np.abs(ev - ev0)) < 1e-6
            srv.release(jid)
        st = srv.stats()
        assert st["done"] == 3 and st["failed"] == 0 and st["bytes_in_use"] == 0


def test_admission_budget_and_refusal(si_pp, c_pp):
    cases = systems(si_pp, c_pp)
    with Server(workers=3, precision=PRECISION_FP64, hbm_budget_bytes=1 << 40) as probe:
        jid = probe.submit(*cases[0][:1], cases[0][1], precision=PRECISION_FP64, **KW)
        one = probe.wait(jid, 60.0)["footprint_bytes"]
    # room for one small job at a time: the others wait at the queue head
    budget = int(one * 1.5)
    with Server(workers=3, precision=PRECISION_FP64, hbm_budget_bytes=budget) as srv:
        ids = [srv.submit(cases[0][0], cases[0][1], precision=PRECISION_FP64, **KW) for _ in range(3)]
        for jid in ids:
            info = srv.wait(jid, 120.0)
            assert info["state"] == 2 and info["status"] == 0
        st = srv.stats()
        assert st["peak_bytes"] <= budget
        big, nb = cases[2]
        with pytest.raises(PwGpuError) as e:
            srv.submit(big, nb, precision=PRECISION_FP64, **dict(KW, mixing_ndim=4000))
        assert e.value.code == -3


def test_wait_times_out_then_completes(si_pp, c_pp):
    s, nb = systems(si_pp, c_pp)[2]
    with Server(workers=1, precision=PRECISION_FP64) as srv:
        jid = srv.submit(s, nb, precision=PRECISION_FP64, **KW)
        with pytest.raises(PwGpuError) as e:
            srv.wait(jid, 0.0)
        assert e.value.code == -5
        assert srv.wait(jid, 120.0)["state"] == 2


def test_stream_requests_build_and_solve(si_pp, c_pp):
    """Small requests of the serving stream (projectors, local potential and
    start density built on the device; Gamma and 2x2x2 meshes, Si and C) run
    four at a time through the queue and give the energies of the same
    requests solved one by one."""
    pps = {"Si": si_pp, "C": c_pp}
    reqs = [r for r in request_stream(40) if r.n_atoms <= 8][:8]
    built = []
    for r in reqs:
        s, kw = request_system(r, pps)
        kw = dict(kw)
        built.append((r, s, kw.pop("n_bands"), kw))
    with Server(workers=4) as srv:
        ids = [srv.submit(s, nb, **kw) for _, s, nb, kw in built]
        got = []
        for jid in ids:
            info = srv.wait(jid, 300.0)
            assert info["status"] == 0
            res, ev, status, err = srv.result(jid)
            assert res["converged"] == 1 and np.all(np.isfinite(ev))
            got.append(res["total_energy"])
    for (r, s, nb, kw), e in zip(built, got):
        with PwGpu(s, lanes=2) as dev:
            res, _, _, _ = dev.scf_run(dev.initial_density(), nb, **kw)
        assert abs(res["total_energy"] - e) / r.n_atoms < 1e-4, (r, res["total_energy"], e)

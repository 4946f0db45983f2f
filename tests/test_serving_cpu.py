"""Host logic of the serving workload on the CPU: the seeded request stream
(Poisson arrivals at 50/s, Si/C, 2/8/16/64 atoms weighted 4:3:2:1, +-2 %
strain, displacements up to 0.05 bohr, ecutwfc in {20, 25, 30, 35} Ry,
Gamma or 2x2x2), the per-request crystal and system, and the replay loop
(setup pool, submission, out-of-order completion, latency summary) driven
against a fake server, so no device is touched."""

import threading
import time

import numpy as np
import pytest

from pwgpu import serving as S
from pwgpu.consts import BOHR_TO_ANG


def test_stream_is_seeded_and_has_the_workload_mix():
    a = S.request_stream(2000)
    b = S.request_stream(2000)
    assert [(r.arrival_s, r.species, r.n_atoms, r.ecut_ry, r.kgrid, r.seed) for r in a] == \
           [(r.arrival_s, r.species, r.n_atoms, r.ecut_ry, r.kgrid, r.seed) for r in b]
    assert S.request_stream(50, seed=1)[0].arrival_s != a[0].arrival_s
    t = np.array([r.arrival_s for r in a])
    gaps = np.diff(np.concatenate([[0.0], t]))
    assert np.all(gaps > 0)
    # Poisson at 50/s: mean gap 20 ms, standard error 20 ms / sqrt(2000)
    assert abs(gaps.mean() - 0.02) < 5 * 0.02 / np.sqrt(2000)
    # exponential gaps: the coefficient of variation is 1
    assert abs(gaps.std() / gaps.mean() - 1.0) < 0.1
    sizes = np.array([r.n_atoms for r in a])
    for n, w in zip(S.SIZES, S.SIZE_WEIGHTS):
        assert abs(np.mean(sizes == n) - w / sum(S.SIZE_WEIGHTS)) < 0.035, n
    assert abs(np.mean([r.species == "Si" for r in a]) - 0.5) < 0.04
    assert abs(np.mean([r.kgrid == (1, 1, 1) for r in a]) - 0.5) < 0.04
    assert {r.kgrid for r in a} == {(1, 1, 1), (2, 2, 2)}
    assert {r.ecut_ry for r in a} == set(S.ECUTS_RY)
    strains = np.array([r.strain for r in a])
    assert strains.min() >= -0.02 and strains.max() <= 0.02 and strains.std() > 0.01


def _ideal(req):
    a = S.LATTICE_BOHR[req.species] * BOHR_TO_ANG * (1.0 + req.strain)
    if req.n_atoms == 2:
        return S.diamond_primitive(req.species, a)
    reps = {8: (1, 1, 1), 16: (2, 1, 1), 64: (2, 2, 2)}[req.n_atoms]
    return S.diamond_supercell(req.species, a, reps)


def test_request_crystal_strain_and_displacements():
    reqs = S.request_stream(200)
    seen = set()
    for req in reqs:
        if req.n_atoms in seen:
            continue
        seen.add(req.n_atoms)
        cr = S.request_crystal(req)
        ideal = _ideal(req)
        assert len(cr.atoms) == req.n_atoms
        assert all(at.symbol == req.species for at in cr.atoms)
        m = np.array([cr.lattice.a, cr.lattice.b, cr.lattice.c]).T
        assert np.allclose(m, np.array([ideal.lattice.a, ideal.lattice.b, ideal.lattice.c]).T)
        d = np.array([m @ (np.array(x.frac) - np.array(y.frac)) for x, y in zip(cr.atoms, ideal.atoms)])
        d_bohr = np.abs(d) / BOHR_TO_ANG
        assert d_bohr.max() <= 0.05 + 1e-12 and d_bohr.max() > 0.01
        # the displacements are the request's own (seeded): rebuilding gives the same cell
        again = S.request_crystal(req)
        assert [at.frac for at in again.atoms] == [at.frac for at in cr.atoms]
    assert seen == set(S.SIZES)


def _small(n, kgrid=None):
    reqs = [r for r in S.request_stream(400) if r.n_atoms == 2 and r.ecut_ry <= 25.0]
    if kgrid is not None:
        reqs = [r for r in reqs if r.kgrid == kgrid]
    assert len(reqs) >= n
    return reqs[:n]


@pytest.mark.parametrize("kgrid", [(1, 1, 1), (2, 2, 2)])
def test_request_system_bands_and_kpoints(si_pp, c_pp, kgrid):
    req = _small(1, kgrid)[0]
    s, kw = S.request_system(req, {"Si": si_pp, "C": c_pp})
    assert abs(s.n_electrons - 8.0) < 1e-9
    # N_el/2 + max(4, N_el/20) bands
    assert kw["n_bands"] == 4 + 4
    assert (len(s.kpoints) == 1) == (kgrid == (1, 1, 1))
    assert abs(s.kpt_weights.sum() - 1.0) < 1e-12
    for k, v in S.SERVE_KW.items():
        assert kw[k] == v


class FakeServer:
    """The Server interface run_stream drives: jobs finish in reverse order of
    submission, each after all of them have been submitted."""

    def __init__(self, n):
        self.n = n
        self.lock = threading.Lock()
        self.submitted = []
        self.finished = []
        self.released = []
        self.cv = threading.Condition(self.lock)

    def submit(self, s, nb, precision=None, **kw):
        with self.cv:
            jid = 1000 + len(self.submitted)
            self.submitted.append((jid, s.n_pw, nb, precision, kw))
            if len(self.submitted) == self.n:
                self.finished = [j for j, *_ in reversed(self.submitted)]
                self.cv.notify_all()
            return jid

    def wait_any(self, timeout_s=1.0):
        with self.cv:
            if not self.finished:
                self.cv.wait(timeout_s)
            return self.finished.pop(0) if self.finished else None

    def result(self, jid):
        i = jid - 1000
        return ({"total_energy": -100.0 - i, "n_iterations": 10 + i, "converged": 1}, np.full((1, 8), float(i)), 0, "")

    def poll(self, jid):
        return {"queue_s": 0.25, "run_s": 0.5, "status": 0}

    def release(self, jid):
        with self.lock:
            self.released.append(jid)


def test_run_stream_records_out_of_order_completions(si_pp, c_pp):
    reqs = _small(4)
    srv = FakeServer(len(reqs))
    recs, wall = S.run_stream(srv, reqs, {"Si": si_pp, "C": c_pp}, setup_threads=2, precision=7, realtime=False)
    assert len(recs) == len(reqs) and wall > 0
    assert sorted(srv.released) == sorted(j for j, *_ in srv.submitted)
    assert all(p == 7 for _, _, _, p, _ in srv.submitted)
    by_jid = {j: n_pw for j, n_pw, *_ in srv.submitted}
    for req, r in zip(reqs, recs):
        assert r["arrival_s"] == req.arrival_s and r["n_atoms"] == 2
        assert r["submit_s"] <= r["done_s"]
        assert r["converged"] == 1 and r["status"] == 0 and r["queue_s"] == 0.25
        # the record got the result of its own job, not another request's
        jid = 1000 + int(r["eigenvalues"][0, 0])
        assert by_jid[jid] == r["n_pw"]
        assert r["total_energy"] == -100.0 - (jid - 1000)
    summ = S.summarize(recs, wall)
    assert summ["requests"] == len(reqs) and summ["converged"] == len(reqs) and summ["finished"] == len(reqs)
    assert summ["server_latency_p50_s"] == pytest.approx(0.75)
    assert summ["latency_p99_s"] >= summ["latency_p50_s"]


def test_run_stream_honours_arrival_times(si_pp, c_pp):
    reqs = _small(2)
    t0 = reqs[0].arrival_s
    for i, r in enumerate(reqs):
        r.arrival_s = (r.arrival_s - t0) + 0.2 * i + 0.05
    srv = FakeServer(len(reqs))
    start = time.perf_counter()
    recs, _ = S.run_stream(srv, reqs, {"Si": si_pp, "C": c_pp}, setup_threads=2, realtime=True)
    assert time.perf_counter() - start >= reqs[-1].arrival_s
    for req, r in zip(reqs, recs):
        assert r["submit_s"] >= req.arrival_s

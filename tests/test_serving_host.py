"""The serving loop's host logic (cm3d_b200.serving.Server) without a GPU:
a stand-in engine records what the server asks of it, so the admission
order, the memory budget, the chunked asynchronous steps and the latency
bookkeeping can be checked on the CPU.  (tests/test_serving.py runs the real
engine on a GPU and checks the jobs' results.)"""
import threading

import numpy as np
import pytest

from cm3d_b200 import serving
from cm3d_b200.serving import Job, Server, device_bytes, summarize


class FakeSystem(dict):
    """the fields device_bytes reads, for a cube of side L with n atoms"""

    def __init__(self, n, L=30.0, rl=11.0, ktot=100):
        super().__init__(hmat=np.diag([L, L, L]).ravel(), rmaxl_skin2=np.array([rl * rl]), ninter=1,
                         ktot=ktot, rmaxl_skin2_e=rl * rl)
        self.natoms = n


class FakeEngine:
    """records the steps launched; a launch completes after two polls"""
    lock = threading.Lock()
    resident = 0
    most = 0
    launches = []

    def __init__(self, system, mode, device, tpa, use_graph):
        self.system, self.pending, self.polls = system, None, 0
        with FakeEngine.lock:
            FakeEngine.resident += 1
            FakeEngine.most = max(FakeEngine.most, FakeEngine.resident)

    def step_init(self):
        pass

    def synchronize(self):
        pass

    def step_async(self, istep0, k):
        assert self.pending is None, "a launch while the previous one is in flight"
        self.pending = (istep0, k)
        self.polls = 0
        FakeEngine.launches.append((id(self), istep0, k))

    def step_done(self):
        self.polls += 1
        if self.polls >= 2:
            self.pending = None
            return True
        return False

    def energies(self):
        return {"poter": -1.0}

    def positions(self):
        return np.zeros((3, self.system.natoms))

    def status(self):
        return {}

    def close(self):
        with FakeEngine.lock:
            FakeEngine.resident -= 1


@pytest.fixture
def fake(monkeypatch):
    FakeEngine.resident, FakeEngine.most, FakeEngine.launches = 0, 0, []
    monkeypatch.setattr(serving, "Engine", FakeEngine)
    return FakeEngine


def make_jobs(sizes, steps, arrivals=None):
    arrivals = arrivals or [0.0] * len(sizes)
    return [Job(k, FakeSystem(n), s, arrival=a, name=f"j{k}") for k, (n, s, a) in
            enumerate(zip(sizes, steps, arrivals))]


def test_every_job_runs_its_steps_in_chunks(fake):
    jobs = make_jobs([300, 900, 2000], [120, 50, 75])
    srv = Server(hbm_budget=1e15, chunk=50, idle_sleep=0.0)
    for j in jobs:
        srv.submit(j)
    done = srv.run(realtime=False)
    assert sorted(j.id for j in done) == [0, 1, 2]
    by_engine = {}
    for eid, istep0, k in fake.launches:
        by_engine.setdefault(eid, []).append((istep0, k))
    assert sorted(sum(k for _, k in v) for v in by_engine.values()) == [50, 75, 120]
    for v in by_engine.values():
        # consecutive chunks of at most `chunk` steps, numbered from 1
        assert v[0][0] == 1 and all(k <= 50 for _, k in v)
        assert all(v[i + 1][0] == v[i][0] + v[i][1] for i in range(len(v) - 1))
    for j in done:
        assert j.done_steps == j.nsteps and j.latency is not None and j.latency >= 0.0
        assert j.result["energies"]["poter"] == -1.0
    assert fake.resident == 0


def test_budget_keeps_jobs_out_until_memory_frees(fake):
    jobs = make_jobs([4000, 4000, 4000], [40, 40, 40])
    one = device_bytes(jobs[0].system)
    srv = Server(hbm_budget=1.5 * one, chunk=10, idle_sleep=0.0)
    for j in jobs:
        srv.submit(j)
    done = srv.run(realtime=False)
    assert len(done) == 3
    assert fake.most == 1 and srv.max_active == 1
    # first come, first served
    assert [j.id for j in done] == [0, 1, 2]
    assert srv.max_bytes <= 1.5 * one


def test_a_job_larger_than_the_budget_still_runs_alone(fake):
    jobs = make_jobs([100000, 300], [10, 10])
    srv = Server(hbm_budget=device_bytes(jobs[1].system) * 2, chunk=10, idle_sleep=0.0)
    for j in jobs:
        srv.submit(j)
    done = srv.run(realtime=False)
    assert [j.id for j in done] == [0, 1] and fake.most == 1


def test_device_bytes_grows_with_atoms_and_k_vectors():
    assert device_bytes(FakeSystem(2000)) > device_bytes(FakeSystem(1000))
    assert device_bytes(FakeSystem(1000, ktot=5000)) > device_bytes(FakeSystem(1000, ktot=100))


def test_summarize_reports_throughput_and_percentiles():
    jobs = make_jobs([100, 200, 300, 400], [10, 10, 10, 10], arrivals=[0.0, 1.0, 2.0, 3.0])
    for k, j in enumerate(jobs):
        j.finished = j.arrival + 1.0 + k
    s = summarize(jobs, wall=10.0)
    assert s["jobs"] == 4 and s["atom_steps"] == 10 * (100 + 200 + 300 + 400)
    assert s["atom_steps_per_s"] == pytest.approx(1000.0)
    assert s["latency_s"]["max"] == pytest.approx(4.0)
    assert s["latency_s"]["p50"] == pytest.approx(2.5)

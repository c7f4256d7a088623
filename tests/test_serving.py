"""The serving loop (cm3d_b200.serving): jobs that arrive while others run
are admitted as memory allows, run concurrently (asynchronous steps on
their own streams), and each job's result is the same as when it runs
alone.

"The same": positions bit-identical and energies within relative 1e-12.
Each job has its own context, and every force the mixed engine computes is
summed in a fixed order, so a trajectory does not depend on what else runs
on the device; only the energy totals are added with atomics.
"""
import numpy as np
import pytest

from cm3d_b200 import _abi, configs, setup
from cm3d_b200.engine import Engine
from cm3d_b200.serving import Job, Server, device_bytes, summarize

pytestmark = pytest.mark.gpu


def jobs(arrivals=(0.0, 0.0, 0.01, 0.05), grids=(3, 4, 5, 4), steps=(300, 400, 250, 120)):
    out = []
    for k, (t, g, ns) in enumerate(zip(arrivals, grids, steps)):
        req = configs.ServingRequest(k, t, g, ns, 100 + k)
        out.append(Job(k, setup.build_system(configs.serving_workload(req)), ns, arrival=t, name=f"job{k}"))
    return out


def alone(job):
    e = Engine(job.system, mode=_abi.MIXED)
    e.step_init()
    e.step(1, job.nsteps)
    en, pos = e.energies(), e.positions()
    e.close()
    return en, pos


def same(job):
    en, pos = alone(job)
    got = job.result["energies"]
    for k in ("poter", "zke", "vinter", "velec", "vewald"):
        assert abs(got[k] - en[k]) <= 1e-12 * max(abs(en[k]), 1.0), (job.name, k, got[k], en[k])
    assert np.array_equal(job.result["positions"], pos), job.name


def test_serving_results_match_alone(engine_lib):
    js = jobs()
    srv = Server(chunk=20)
    for j in js:
        srv.submit(j)
    done = srv.run()
    assert len(done) == len(js)
    assert srv.max_active >= 2, "jobs should have overlapped"
    for j in done:
        assert j.done_steps == j.nsteps and j.admitted >= j.arrival - 1e-6
        same(j)
    s = summarize(done, max(j.finished for j in done))
    assert s["jobs"] == len(js) and s["latency_s"]["p99"] >= s["latency_s"]["p50"] > 0


def test_serving_admits_against_the_budget(engine_lib):
    js = jobs(arrivals=(0.0, 0.0, 0.0, 0.0))
    budget = sorted(device_bytes(j.system) for j in js)[-1] + sorted(device_bytes(j.system) for j in js)[-2]
    srv = Server(chunk=20, hbm_budget=budget)
    for j in js:
        srv.submit(j)
    done = srv.run()
    assert len(done) == len(js)
    assert srv.max_active <= 2 and srv.max_bytes <= budget
    for j in done:
        same(j)

"""Serving loop: continuous batching of CM3D MD jobs on one GPU.

Jobs -- a CM3D system (cm3d_b200.system.System, e.g. from
cm3d_b200.setup.build_system) and a number of outer steps -- arrive over
time.  The server

  * admits a job as soon as it has arrived and its device-memory estimate
    fits the HBM budget next to the jobs already resident (first come, first
    served: a job that does not fit holds the queue until memory frees up);
  * keeps every admitted job's state resident in its own engine context,
    with its own CUDA stream and step graph; a job's context is created and
    its start-up (lists, first forces) run on a worker thread, so that an
    admission does not hold up the polling of the jobs already running;
  * advances every active job in chunks of steps launched asynchronously
    (cm3d_nb_step_async), so that the chunks of all active jobs are in
    flight together and their kernels overlap on the device, and polls them
    without blocking (cm3d_nb_step_query);
  * retires a job when its steps are done: final energies and positions
    are read back, the context is destroyed and its memory returns to the
    budget.

A job's result does not depend on the other jobs: each has its own context,
lists, tables and stream.  Latency = completion time - arrival time.

The comparator of the metric (`mode=PLAIN_FP64`) runs the same loop with the
plain FP64 engine, one job per context and per launch.
"""
from __future__ import annotations

import concurrent.futures as cf
import math
import time
from dataclasses import dataclass, field

import numpy as np

from . import _abi
from .engine import Engine


@dataclass
class Job:
    """One MD request."""
    id: int
    system: object                 # cm3d_b200.system.System
    nsteps: int
    arrival: float = 0.0           # seconds after the server starts
    name: str = ""
    # filled by the server
    admitted: float | None = None
    finished: float | None = None
    done_steps: int = 0
    result: dict = field(default_factory=dict)

    @property
    def natoms(self) -> int:
        return int(self.system.natoms)

    @property
    def latency(self) -> float | None:
        return None if self.finished is None else self.finished - self.arrival


def device_bytes(system) -> int:
    """Estimate of a job's device memory: per-atom state, the full neighbour
    list (1.3 x the mean number of atoms in a list sphere + 64 entries per
    atom, 4 bytes each), the k-space work arrays, plus a fixed part."""
    n = int(system.natoms)
    h = np.asarray(system["hmat"], float).reshape(3, 3)
    vol = abs(float(np.linalg.det(h)))
    r2 = float(np.max(system["rmaxl_skin2"])) if system["ninter"] > 0 else 0.0
    if int(system.get("ktot", 0)) > 0:
        r2 = max(r2, float(system.get("rmaxl_skin2_e", 0.0)))
    rl = math.sqrt(r2)
    stride = min(1.3 * n / vol * 4.0 / 3.0 * math.pi * rl ** 3 + 64.0, n + 31.0)
    ktot = int(system.get("ktot", 0))
    kbytes = ktot * (math.ceil(n / 2048) * 16 + 64)
    return int(n * (4.0 * stride + 420.0) + kbytes + (8 << 20))


class Server:
    """Continuous-batching MD server on one device (see the module text)."""

    def __init__(self, device: int = 0, hbm_budget: float = 150e9, mode: int = _abi.MIXED,
                 chunk: int = 50, use_graph: bool = True, tpa: int = 0, idle_sleep: float = 2e-4,
                 setup_workers: int = 2):
        self.device, self.budget, self.mode = device, float(hbm_budget), mode
        self.chunk, self.use_graph, self.tpa, self.idle_sleep = chunk, use_graph, tpa, idle_sleep
        self.setup_workers = setup_workers
        self.queue: list[Job] = []
        self.finished: list[Job] = []
        self.max_active = 0
        self.max_bytes = 0

    def submit(self, job: Job) -> None:
        self.queue.append(job)
        self.queue.sort(key=lambda j: (j.arrival, j.id))

    def _prepare(self, job: Job) -> Engine:
        """a job's context and start-up (runs on a worker thread)"""
        eng = Engine(job.system, mode=self.mode, device=self.device, tpa=self.tpa, use_graph=self.use_graph)
        try:
            eng.step_init()
            eng.synchronize()
        except Exception:
            eng.close()
            raise
        return eng

    def _finish(self, job: Job, eng: Engine, now: float) -> None:
        en = eng.energies()
        job.result = {"energies": en, "positions": eng.positions(), "status": eng.status()}
        eng.close()
        job.finished = now
        self.finished.append(job)

    def run(self, clock=time.perf_counter, realtime: bool = True) -> list[Job]:
        """Serve every submitted job; returns them in completion order.  With
        realtime, arrivals are honoured on the wall clock (a job is not
        admitted before its arrival time)."""
        t0 = clock()
        active: list[list] = []            # [job, engine, bytes, steps in flight]
        starting: list[tuple] = []         # (job, bytes, future of its engine)
        used = 0
        pending = list(self.queue)
        self.queue = []
        pool = cf.ThreadPoolExecutor(max_workers=self.setup_workers)
        try:
            return self._loop(clock, realtime, t0, active, starting, used, pending, pool)
        finally:
            pool.shutdown(wait=True)

    def _loop(self, clock, realtime, t0, active, starting, used, pending, pool):
        while pending or active or starting:
            # admission: first come, first served, against the budget; the
            # context is set up on a worker thread
            while pending and (not realtime or pending[0].arrival <= clock() - t0):
                job = pending[0]
                need = device_bytes(job.system)
                if (active or starting) and used + need > self.budget:
                    break
                pending.pop(0)
                used += need
                starting.append((job, need, pool.submit(self._prepare, job)))
            # jobs whose start-up has finished join the running set
            still_starting = []
            for job, need, fut in starting:
                if not fut.done():
                    still_starting.append((job, need, fut))
                    continue
                eng = fut.result()
                job.admitted = clock() - t0
                k = min(self.chunk, job.nsteps)
                eng.step_async(1, k)
                active.append([job, eng, need, k])
                self.max_active = max(self.max_active, len(active))
                self.max_bytes = max(self.max_bytes, used)
            starting[:] = still_starting
            # completions: non-blocking polls, then the next chunk or retirement
            progressed = False
            still = []
            for slot in active:
                job, eng, nb, inflight = slot
                if inflight:
                    if not eng.step_done():
                        still.append(slot)
                        continue
                    job.done_steps += inflight
                    slot[3] = 0
                    progressed = True
                if job.done_steps >= job.nsteps:
                    self._finish(job, eng, clock() - t0)
                    used -= nb
                    continue
                k = min(self.chunk, job.nsteps - job.done_steps)
                eng.step_async(1 + job.done_steps, k)
                slot[3] = k
                still.append(slot)
            active[:] = still
            if not progressed and (not pending or (realtime and pending[0].arrival > clock() - t0)):
                time.sleep(self.idle_sleep)
        return self.finished


def summarize(jobs: list[Job], wall: float) -> dict:
    """Aggregate throughput and latency percentiles of served jobs."""
    lat = np.array([j.latency for j in jobs])
    atom_steps = float(sum(j.natoms * j.nsteps for j in jobs))
    return {"jobs": len(jobs), "atom_steps": atom_steps, "wall_s": wall,
            "atom_steps_per_s": atom_steps / wall if wall > 0 else None,
            "latency_s": {"p50": float(np.percentile(lat, 50)), "p95": float(np.percentile(lat, 95)),
                          "p99": float(np.percentile(lat, 99)), "max": float(lat.max())}}

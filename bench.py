"""Benchmark of the CM3D nonbonded engine on one B200 (or N ranks).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload ensemble1024|water12288|water331776|argon864]

A step is one CM3D outer step (integrate/md_step.c:62: inner bonded levels,
neighbour-list check/rebuild with RESETPOS, full nonbonded + Ewald forces,
kicks) of every system of the workload.  Default workload: the uneven
ensemble of 1024 independent boxes (N log-uniform in [64, 4096], reduced
density U(0.6, 0.9), T* U(0.7, 1.5), 75% argon LJ, 25% charged +/-0.5 e
binary with Ewald alpha = 3.2/rc and kmax 5, rc = min(2.5 sigma, 0.45 L), FCC
start, dt 5 fs), run as one batch.  Inputs are synthetic and seeded
(cm3d_b200.configs) and written in CM3D's own input formats.

Printed: one JSON line (rank 0) with the contract's keys plus
  plain_fp64      the same systems through the plain FP64 engine, one system
                  per context and per launch (the comparator of the metric)
  roofline        the fused pair kernel against its FP32 / HBM roofline
  cpu_baseline    CM3D itself (oracle/_ref/ref_bench) on this host's cores
  e2e             the same metric through the public API with host buffers
  latency         per-step device time p50 / p99
  other_workloads the water-12288 box, mixed and plain, and 1024 boxes of
                  CM3D's abutane molecule (the torsion level), in the same run
  serving         the serving loop on a Poisson stream of water-box jobs
                  (4 jobs/s over 5 s): job latency p50/p95/p99 and aggregate
                  atom-steps/s, mixed against plain FP64 on the same jobs
Under torchrun (N > 1) every rank runs its own ensemble (seed + rank): the
systems are independent and no collective touches the step path.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "atom-steps/s batched mixed vs plain FP64 GPU at ≤1e-5 force err; p50/p99 latency"
UNIT = "atom-steps/s"
# per unique listed pair (i < j) of CM3D's te / t lists (algorithmic counts)
FLOPS_ELEC_PAIR = 57.0
FLOPS_LJ_EXTRA = 14.0
FLOPS_LJ_ONLY = FLOPS_ELEC_PAIR - 16.0 + FLOPS_LJ_EXTRA   # no charge product / erfc tables
BYTES_PAIR = 4.0                  # one 32-bit neighbour index
BYTES_ATOM = 16.0 + 24.0          # float4 position/charge in, FP64 force out


def workload(name: str, seed: int):
    """(list of Workloads, description, default steps)"""
    from cm3d_b200 import configs
    if name == "ensemble1024":
        return configs.ensemble(1024, seed=2024 + seed - 1), \
            "ensemble-1024: 1024 independent boxes, N log-uniform in [64, 4096] (953,101 atoms at seed 2024), " \
            "rho* U(0.6,0.9), T* U(0.7,1.5), 75% argon LJ / 25% charged +/-0.5 e binary (Ewald alpha 3.2/rc, " \
            "kmax 5), rc min(2.5 sigma, 0.45 L), skin 0.3 sigma, FCC start, dt 5 fs, one batch", 300
    if name == "water12288":
        return [configs.water_box(ngrid=16, seed=seed, ntime=1000)], \
            "water-12288: 4096 flexible 3-site waters on a 16^3 grid (seeded orientations, no intermolecular " \
            "contact under 1.9 A), L 49.66 A, alpha 0.31, kmax 7, rc 10 A, skin 0.5 A, RESPA 0.5/2 fs " \
            "(nres_intra 4), 300 K", 1000
    if name == "water331776":
        return [configs.water_box(ngrid=48, seed=seed, skin=1.5, kmax=21, ntime=500, placement="octant")], \
            "water-331776: 110592 flexible 3-site waters on a 48^3 grid (seeded orientations, no " \
            "intermolecular contact under 1.9 A), L 148.98 A, alpha 0.31, kmax 21, rc 10 A, skin 1.5 A, " \
            "RESPA 0.5/2 fs", 100
    if name == "argon864":
        return [configs.argon_fcc(seed=seed, ntime=1000)], \
            "argon-864: LJ argon FCC 6^3x4, rho* 0.8442, rc 2.5 sigma, skin 0.3 sigma, dt 5 fs, 120 K", 1000
    raise SystemExit(f"unknown workload {name}")


# ----------------------------------------------------------------- clocks
class ClockSampler:
    """SM clock and throttle reasons sampled through NVML during a region."""

    REASONS = {0x1: "gpu_idle", 0x2: "applications_clocks_setting", 0x4: "sw_power_cap",
               0x8: "hw_slowdown", 0x10: "sync_boost", 0x20: "sw_thermal_slowdown",
               0x40: "hw_thermal_slowdown", 0x80: "hw_power_brake_slowdown",
               0x100: "display_clock_setting"}

    def __init__(self, device: int):
        self.samples, self.reasons, self.max_mhz = [], set(), None
        self._stop = threading.Event()
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nv = pynvml
            self.h = pynvml.nvmlDeviceGetHandleByIndex(device)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
        except Exception:
            self.nv = None

    def _run(self):
        while not self._stop.is_set():
            try:
                self.samples.append(self.nv.nvmlDeviceGetClockInfo(self.h, self.nv.NVML_CLOCK_SM))
                r = self.nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
                for bit, name in self.REASONS.items():
                    if r & bit and name != "gpu_idle":
                        self.reasons.add(name)
            except Exception:
                pass
            time.sleep(0.05)

    def __enter__(self):
        if self.nv:
            self.t = threading.Thread(target=self._run, daemon=True)
            self.t.start()
        return self

    def __exit__(self, *exc):
        self._stop.set()
        if self.nv:
            self.t.join()

    def summary(self) -> dict:
        return {"sm_mhz": float(statistics.median(self.samples)) if self.samples else None,
                "sm_max_mhz": self.max_mhz, "reasons": sorted(self.reasons),
                "samples": len(self.samples)}


# ----------------------------------------------------------------- helpers
def measured_peaks() -> dict:
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            return json.load(fh)
    except Exception:
        return {}


def l2_flusher(device: int):
    """Write a buffer larger than L2 (126 MB) and wait for it, so the next
    step starts with a cold L2 (the write is outside the step's events)."""
    import torch
    buf = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{device}")

    def flush():
        buf.fill_(1.0)
        torch.cuda.synchronize(device)
    return flush


def timed_run(eng, steps: int, warmup: int, istep0: int, flush) -> tuple[float, int, list]:
    """W untimed steps, then K steps each timed on the device (CUDA events
    around the step's graph replay on the engine's stream), with an L2 flush
    between steps outside the timed events.  Returns (total ms, kernels
    launched in the timed steps, per-step ms)."""
    istep = istep0
    for _ in range(warmup):
        eng.step(istep, 1)
        istep += 1
    eng.synchronize()
    eng.enable_timing(2)
    l0 = eng.launch_count()
    per, prev = [], 0.0
    for _ in range(steps):
        flush()
        eng.step(istep, 1)
        istep += 1
        tot, _ = eng.kernel_time(4)
        per.append(tot - prev)
        prev = tot
    launches = eng.launch_count() - l0
    eng.enable_timing(0)
    return prev, launches, per


def pinned(n: int):
    try:
        import torch
        return torch.empty(n, dtype=torch.float64, pin_memory=True).numpy()
    except Exception:
        return np.empty(n)


def e2e_run(eng, steps: int, istep0: int, n: int) -> tuple[float, int, int]:
    """The public API with host buffers: every step uploads positions and
    velocities from pinned host memory, runs one step, and reads positions,
    velocities and every system's energies back (CM3D's host loop owning the
    state).  The host arrays are registered as the step's outputs
    (cm3d_nb_set_host_outputs), so the positions come back while the step's
    forces are computed; cm3d_nb_step_host uploads the inputs and runs the
    step."""
    px, vx = [pinned(3 * n).reshape(3, n) for _ in range(2)]
    px[:] = eng.positions()
    vx[:] = eng.velocities()
    etab = eng.energies_table()
    eng.set_host_outputs(px, vx)
    eng.synchronize()
    t0 = time.perf_counter()
    for s in range(steps):
        eng.step_host(istep0 + s, px, vx)
        eng.energies_table(out=etab)
    dt = time.perf_counter() - t0
    eng.set_host_outputs(None, None)
    h2d = 2 * 3 * n * 8
    d2h = 2 * 3 * n * 8 + 144 * 8 * eng.nsys     # + every system's accumulator block (ACC_STRIDE doubles)
    return dt, h2d, d2h


def roofline(eng, steps: int, istep0: int, fp32_tflops: float, hbm_gbs: float) -> dict:
    """Time the fused pair kernel with CUDA events around every launch (eager
    launches on the engine's stream) and compare with its roofline: the
    slower of its algorithmic bytes / HBM bandwidth and its algorithmic flops
    / FP32 FMA throughput (both measured).  Pairs are CM3D's unique listed
    pairs (te for charged systems, t otherwise), counted from its own lists."""
    from cm3d_b200 import _abi
    eng.enable_timing(1)
    eng.step(istep0, steps)
    ms, launches = eng.kernel_time(0)
    eng.enable_timing(0)
    ite, _ = eng.pair_list(_abi.LIST_TE)
    it, _ = eng.pair_list(_abi.LIST_T)
    starts = np.array([a for a, _ in eng.ranges] + [eng.n])
    pte_s = np.bincount(np.searchsorted(starts, ite, side="right") - 1, minlength=eng.nsys)
    pt_s = np.bincount(np.searchsorted(starts, it, side="right") - 1, minlength=eng.nsys)
    charged = pte_s > 0
    flops = float((pte_s * FLOPS_ELEC_PAIR + pt_s * FLOPS_LJ_EXTRA)[charged].sum()
                  + (pt_s * FLOPS_LJ_ONLY)[~charged].sum())
    pairs = float(pte_s[charged].sum() + pt_s[~charged].sum())
    nbytes = pairs * BYTES_PAIR + eng.n * BYTES_ATOM
    t = ms / 1e3 / max(launches, 1)
    t_bw = nbytes / (hbm_gbs * 1e9)
    t_fl = flops / (fp32_tflops * 1e12)
    # DRAM bytes per launch from an ncu capture (profiles/pair_kernel_traffic.json),
    # used only while the kernel's source is the one that was captured
    kind, tpa = eng.pair_kernel()
    traffic, traffic_src = None, "no capture of this kernel"
    try:
        import hashlib
        with open(os.path.join(ROOT, "profiles", "pair_kernel_traffic.json")) as fh:
            tr = json.load(fh).get(eng.workload_name, {})
        src = os.path.join(ROOT, "cm3d_b200", "csrc", "nb_cwin.cu" if kind == "compact" else "nb_pair.cu")
        with open(src, "rb") as fh:
            sha = hashlib.sha256(fh.read()).hexdigest()[:16]
        if tr.get("pair_kernel") == kind and tr.get("source_sha16") == sha:
            traffic = tr.get("dram_bytes_per_launch")
            traffic_src = f"{tr.get('source')} (captured {tr.get('date')}, kernel source sha {sha})"
        elif tr:
            traffic_src = f"capture of {tr.get('pair_kernel')} at source sha {tr.get('source_sha16')} is stale " \
                          f"(now {kind}, sha {sha}): not used"
    except Exception:
        pass
    if t_fl >= t_bw:
        out = {"bound": "fp32", "achieved": flops / t / 1e12, "peak": fp32_tflops, "unit": "TFLOP/s",
               "frac": (flops / t / 1e12) / fp32_tflops}
    else:
        out = {"bound": "hbm", "achieved": nbytes / t / 1e9, "peak": hbm_gbs, "unit": "GB/s",
               "frac": (nbytes / t / 1e9) / hbm_gbs}
    out.update({"traffic": traffic, "traffic_source": traffic_src,
                "kernel": f"{kind} pair kernel (fused LJ + real-space Ewald), {tpa} lanes per atom",
                "ms_per_launch": t * 1e3, "launches": launches, "unique_pairs": pairs,
                "pairs_te": int(pte_s.sum()), "pairs_t": int(pt_s.sum()),
                "algorithmic_flops": flops, "algorithmic_bytes": nbytes,
                "hbm_frac": (nbytes / t / 1e9) / hbm_gbs,
                "fp32_frac": (flops / t / 1e12) / fp32_tflops,
                "peak_source": "fp32: cm3d_nb_measure_peaks (this run, of measured); "
                               "hbm: MEASURED_PEAKS.json (of measured)"})
    return out


def compact_roofline(systems, device: int, name: str, fp32: float, hbm: float) -> dict:
    """The compact pair kernel's roofline on a one-system workload (cell
    scale 1.0, the kernel the context takes by default), from eager launches
    timed with CUDA events as in roofline()."""
    from cm3d_b200 import _abi
    from cm3d_b200.engine import Engine
    eng = Engine(systems, mode=_abi.MIXED, device=device, tpa=32)
    eng.workload_name = name
    eng.step_init()
    eng.step(1, 5)
    out = roofline(eng, 20, 6, fp32, hbm)
    eng.close()
    return out


# ------------------------------------------------------------ CPU baseline
def ref_bench_bin() -> str | None:
    p = os.path.join(ROOT, "oracle", "_ref", "ref_bench")
    return p if os.path.exists(p) else None


def cpu_cost(wl) -> float:
    """estimated seconds of one CM3D step of a workload's system on one core
    (fit to ref_bench timings of 96 ensemble boxes: t = n (0.63 + 41 rho) us
    for LJ boxes, n (443 rho) us for charged Ewald boxes, rho = n / V in
    atoms per A^3; the water boxes fall near the charged line)"""
    rho = wl.natoms / float(wl.box) ** 3
    charged = "kmax" in wl.keywords
    return wl.natoms * ((443.0 * rho) if charged else (0.63 + 41.4 * rho)) * 1e-6


def cpu_bounded_steps(wls, cores: int, steps: int, budget_s: float = 30.0) -> int:
    """the timed steps of a CPU run: `steps`, fewer where the workload's
    estimated step time on `cores` cores (one system per core, cpu_cost)
    would make them take longer than budget_s"""
    per_core = sorted((cpu_cost(w) for w in wls), reverse=True)
    est = max(sum(per_core) / max(1, min(cores, len(wls))), per_core[0])
    return max(1, min(steps, int(budget_s / max(est, 1e-9))))


def run_deck(exe: str, inp: str, steps: int, warmup: int) -> dict:
    """CM3D's start-up, `warmup` untimed and `steps` timed iterations of its
    MD loop body in one process (ref_bench); its JSON line"""
    out = subprocess.run([exe, os.path.basename(inp), str(steps), str(warmup)], cwd=os.path.dirname(inp),
                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True, check=True).stdout
    return json.loads([ln for ln in out.splitlines() if ln.startswith("{")][-1])


def cpu_reference(wls, cores: int, steps: int, warmup: int) -> dict:
    """CM3D itself (oracle/_ref/ref_bench, built from its sources with gcc
    -O2) on the host cores over the whole workload: every system runs
    `warmup` untimed and then `steps` timed iterations of CM3D's MD loop
    body (main/md_mdcntr.new.c:176-178), one process per system (CM3D is
    single-threaded), `cores` processes at any moment from a queue ordered
    by estimated cost, so every core stays busy until the queue runs dry.
    Each process times its own steps.  value = all atom-steps / (the timed
    seconds of all processes / cores): the rate of `cores` cores that do
    nothing but CM3D steps (start-up and the queue's tail excluded, which
    favours the CPU)."""
    import concurrent.futures as cf
    exe = ref_bench_bin()
    order = sorted(range(len(wls)), key=lambda k: -cpu_cost(wls[k]))
    cores = max(1, min(cores, len(wls)))
    t0 = time.perf_counter()
    with tempfile.TemporaryDirectory() as tmp:
        decks = {k: wls[k].write(os.path.join(tmp, f"s{k}")) for k in order}
        with cf.ThreadPoolExecutor(max_workers=cores) as ex:
            res = list(ex.map(lambda k: run_deck(exe, decks[k], steps, warmup), order))
    elapsed = time.perf_counter() - t0
    busy = sum(r["seconds"] for r in res)
    total = sum(r["natoms"] * r["steps"] for r in res)
    natoms = sum(r["natoms"] for r in res)
    return {"value": total / (busy / cores), "unit": UNIT, "cores": cores, "kind": "reference",
            "sample": f"the whole workload ({len(wls)} systems, {natoms} atoms), {warmup} untimed + {steps} timed "
                      f"steps each of CM3D's MD loop body (oracle/_ref/ref_bench, gcc -O2), one process per "
                      f"system, {cores} at a time from a queue; value = atom-steps / (summed timed seconds / "
                      f"{cores} cores)",
            "steps": steps, "warmup": warmup, "timed_core_s": busy,
            "elapsed_s_with_startup": elapsed, "atom_steps": total,
            "single_core_rate": total / busy}


def cpu_port(systems, steps: int) -> dict:
    from oracle import Oracle
    o = Oracle(systems[0])
    o.step_init()
    t0 = time.perf_counter()
    o.step(1, steps)
    dt = time.perf_counter() - t0
    return {"value": systems[0].natoms * steps / dt, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": f"oracle (C restatement of CM3D) for {steps} steps of one system"}


# ------------------------------------------------------------ GPU arms
def plain_arm(systems, device: int, steps: int, warmup: int, flush) -> dict:
    """The plain FP64 engine, one system per context: each system's steps run
    as their own launches (graph replays), one system after another, so the
    ensemble's step time is the sum of its systems' step times."""
    from cm3d_b200 import _abi
    from cm3d_b200.engine import Engine
    ms_tot, atoms = 0.0, 0
    for sm in systems:
        pe = Engine(sm, mode=_abi.PLAIN_FP64, device=device)
        pe.step_init()
        ms, _, _ = timed_run(pe, steps, warmup, 1, lambda: None)
        pe.close()
        ms_tot += ms
        atoms += sm.natoms
    flush()
    return {"value": atoms * steps / (ms_tot / 1e3), "unit": UNIT, "ms_per_step": ms_tot / steps,
            "steps": steps, "systems": len(systems),
            "timing": "CUDA events around each system's step graph replay, summed over systems"}


def mixed_arm(systems, device: int, steps: int, warmup: int, flush, fp32: float, hbm: float, name: str,
              e2e_steps: int, dist=None, pin=None) -> dict:
    """pin = (lanes per atom, "gather" | "staged" | "compact" | "compact8"): skip the autotuner and use
    that choice (a profiler run reproduces the choice the autotuner makes
    without the profiler, whose serialised timings would mislead it)."""
    import torch
    from cm3d_b200 import _abi
    from cm3d_b200.engine import Engine, tune_cell_scale
    if pin and pin[1] in ("gather", "staged"):
        os.environ["CM3D_NB_PAIR_KERNEL"] = "list" if pin[1] == "gather" else "window"
    if pin and pin[1] == "compact8":
        os.environ["CM3D_NB_CW_ROW"] = "8"
    # the cell size by measurement (fresh contexts per candidate, before the
    # measured one; every rank the same way)
    cells = None if pin else tune_cell_scale(systems, device=device)
    eng = Engine(systems, mode=_abi.MIXED, device=device, tpa=pin[0] if pin else 0,
                 cell_scale=cells["cell_scale"] if cells else 1.0)
    if pin:
        os.environ.pop("CM3D_NB_PAIR_KERNEL", None)
        os.environ.pop("CM3D_NB_CW_ROW", None)
    eng.workload_name = name
    eng.step_init()
    tune = {"tpa": pin[0], "kernel": pin[1], "pinned": True} if pin else eng.autotune()
    if cells:
        tune["cell_scale"] = cells["cell_scale"]
        tune["cell_scale_candidates"] = {str(k): v for k, v in cells["candidates"].items()}
    n = eng.n
    if dist:
        dist.barrier()
    torch.cuda.synchronize(device)
    with ClockSampler(device) as clk:
        ms, launches, per = timed_run(eng, steps, warmup, 1, flush)
    torch.cuda.synchronize(device)
    if dist:
        t = torch.tensor([ms], dtype=torch.float64, device=f"cuda:{device}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
        dist.barrier()
    status = eng.status()
    istep = 1 + warmup + steps
    if dist:
        dist.barrier()
    dt_e2e, h2d, d2h = e2e_run(eng, e2e_steps, istep, n)
    istep += e2e_steps
    if dist:
        t = torch.tensor([dt_e2e], dtype=torch.float64, device=f"cuda:{device}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dt_e2e = float(t.item())
    roof = roofline(eng, 20, istep, fp32, hbm)
    en = eng.all_energies()
    eng.close()
    return {"ms": ms, "launches": launches, "per_step_ms": per, "n": n, "status": status,
            "e2e": (dt_e2e, h2d, d2h, e2e_steps), "roofline": roof, "energies": en,
            "clocks": clk.summary(), "autotune": tune}


def intra_arm(device: int, copies: int, steps: int, warmup: int, flush) -> dict:
    """The torsion path: CM3D's test/abutane molecule (14 atoms: torsions,
    1-4 pairs, cross bonds, two frozen atoms, Ewald; RESPA nres_tors 2,
    nres_intra 2), `copies` independent boxes in one batch, from the
    state CM3D itself dumped (tests/golden/abutane.npz)."""
    from cm3d_b200 import _abi
    from cm3d_b200.engine import Engine
    from cm3d_b200.system import System
    d = dict(np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "tests", "golden", "abutane.npz")))
    base = System.from_arrays(d)
    eng = Engine([base.copy() for _ in range(copies)], mode=_abi.MIXED, device=device)
    eng.step_init()
    ms, launches, _ = timed_run(eng, steps, warmup, 1, flush)
    n = eng.n
    eng.close()
    return {"workload": f"abutane-{copies}: CM3D's test/abutane molecule (14 atoms, 27 torsions, 27 1-4 "
                        f"pairs, 3 cross bonds, 2 frozen atoms, Ewald), {copies} boxes in one batch",
            "value": n * steps / (ms / 1e3), "unit": UNIT, "ms_per_step": ms / steps, "steps": steps,
            "gpu_launches_per_step": launches / steps}


def nve_arm(device: int) -> dict:
    """Energy conservation (cm3d_b200.drift): the least-squares drift of
    CM3D's conserved energy ham per atom per ns over 1000 NVE steps, for the
    mixed and plain FP64 engines and for CM3D itself from the same initial
    state.  argon864 starts on its FCC lattice, and CM3D runs here on the host
    (oracle/_ref/ref_bench in its trace mode).  water12288 starts from the
    state CM3D equilibrated at 300 K (tests/golden/water12288_eq.npz); CM3D's
    1000 steps of it (about 7 minutes on one core) are the committed
    trajectory of tests/golden/make_nve.py."""
    from cm3d_b200 import _abi, configs
    from cm3d_b200.drift import drift_stats, engine_series
    from cm3d_b200.setup import build_system
    golden = os.path.join(ROOT, "tests", "golden")
    with open(os.path.join(golden, "nve_cm3d.json")) as fh:
        ref = json.load(fh)
    eq = np.load(os.path.join(golden, "water12288_eq.npz"))
    wls = {"argon864": configs.argon_fcc(seed=1, ntime=1000),
           "water12288": configs.water_box(ngrid=16, seed=1, ntime=1000).with_state(eq["pos"], eq["vel"])}
    out = {}
    for name, wl in wls.items():
        r = ref[name]
        n, dt, nsteps = r["natoms"], r["dt_ps"], r["nsteps"]
        sm = build_system(wl)
        row = {"steps": nsteps, "dt_fs": dt * 1e3, "start": r["start"]}
        for key, mode in (("mixed", _abi.MIXED), ("plain_fp64", _abi.PLAIN_FP64)):
            row[key] = drift_stats(engine_series(sm, mode, nsteps, device), dt, n)
        cm3d_ham, src = r["ham"], "tests/golden/nve_cm3d.json (CM3D run by tests/golden/make_nve.py)"
        if name == "argon864" and ref_bench_bin():
            with tempfile.TemporaryDirectory() as tmp:
                inp = wl.write(tmp)
                txt = subprocess.run([ref_bench_bin(), os.path.basename(inp), str(nsteps), "0", "trace"], cwd=tmp,
                                     stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True, check=True).stdout
            cm3d_ham = [sum(float(v) for v in ln.split()[2:5]) for ln in txt.splitlines() if ln.startswith("T ")]
            src = "oracle/_ref/ref_bench on this host, this run"
        row["cm3d"] = {**drift_stats(cm3d_ham, dt, n), "source": src}
        out[name] = row
    return out


def serving_arm(rate: float, window: float, device: int, plain: bool) -> dict:
    """The serving loop (cm3d_b200.serving) on a Poisson stream of water-box
    jobs (configs.serving_plan: molecules log-uniform in [256, 16384], steps
    U[500, 5000], RESPA 0.5/2 fs), mixed engine and -- on the same jobs --
    the plain FP64 engine, one job per context and per launch."""
    from cm3d_b200 import _abi, configs, setup
    from cm3d_b200.serving import Job, Server, summarize
    plan = configs.serving_plan(rate, window)
    systems = [setup.build_system(configs.serving_workload(r)) for r in plan]
    out = {"rate_jobs_per_s": rate, "arrival_window_s": window, "hbm_budget_gb": 150.0,
           "jobs": len(plan), "natoms_total": int(sum(sm.natoms for sm in systems))}
    for key, mode in (("mixed", _abi.MIXED), ("plain_fp64", _abi.PLAIN_FP64)):
        if key == "plain_fp64" and not plain:
            continue
        srv = Server(device=device, mode=mode, chunk=100)
        for r, sm in zip(plan, systems):
            srv.submit(Job(r.index, sm, r.nsteps, arrival=r.arrival))
        t0 = time.perf_counter()
        done = srv.run()
        res = summarize(done, time.perf_counter() - t0)
        res["max_concurrent"] = srv.max_active
        out[key] = res
    if plain:
        out["speedup_mixed_vs_plain"] = out["mixed"]["atom_steps_per_s"] / out["plain_fp64"]["atom_steps_per_s"]
    return out


# ------------------------------------------------------------------- main
def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None)
    ap.add_argument("--warmup", type=int, default=None)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="ensemble1024")
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-extra", action="store_true", help="skip the secondary workloads")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline (profiling runs)")
    ap.add_argument("--no-serving", action="store_true", help="skip the serving leg")
    ap.add_argument("--tpa", type=int, default=0, choices=[0, 4, 8, 16, 32],
                    help="pin the pair kernel's lanes per atom instead of autotuning (profiling runs)")
    ap.add_argument("--pair-kernel", default="gather", choices=["gather", "staged", "compact", "compact8"],
                    help="with --tpa: the pair kernel to pin")
    ap.add_argument("--partition", action="store_true",
                    help="N > 1: split one ensemble over the ranks (LPT on the cost model, strong scaling) "
                         "instead of one ensemble per rank (weak scaling)")
    ap.add_argument("--serving-sweep", action="store_true",
                    help="serving at 0.5, 1, 2, 4, 8 jobs/s over --serving-window s windows (long)")
    ap.add_argument("--serving-window", type=float, default=120.0,
                    help="arrival window of each --serving-sweep rate, seconds")
    ap.add_argument("--serving-only", action="store_true",
                    help="with --serving-sweep: run the sweep alone and print its list (one GPU)")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank != 0:
            return
        wls, desc, dsteps = workload(args.workload, seed=1)
        steps = args.steps if args.steps is not None else dsteps
        warmup = args.warmup if args.warmup is not None else 20
        procs = max(1, min(os.cpu_count() or 1, 64))
        rsteps = cpu_bounded_steps(wls, procs, steps)
        if ref_bench_bin():
            base = cpu_reference(wls, procs, rsteps, min(warmup, rsteps))
        else:
            from cm3d_b200.setup import build_system
            base = cpu_port([build_system(wls[0])], rsteps)
        natoms = sum(w.natoms for w in wls)
        line = {"impl": "reference", "metric": METRIC, "value": base["value"], "unit": UNIT,
                "n_gpus": args.gpus, "steps": rsteps, "warmup": min(warmup, rsteps),
                "ms_per_step": 1e3 * natoms / base["value"],
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic", "config": {"workload": desc, "natoms": natoms,
                                                "parallelism": f"{base['cores']} host processes"},
                "cpu_baseline": base,
                "e2e": {"value": base["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return

    if args.serving_sweep and args.serving_only:
        sweep = []
        for r in (0.5, 1.0, 2.0, 4.0, 8.0):
            t0 = time.perf_counter()
            res = serving_arm(r, args.serving_window, local, not args.no_plain)
            res["wall_total_s"] = time.perf_counter() - t0
            print(json.dumps(res), flush=True)
            sweep.append(res)
        print(json.dumps({"serving_sweep": sweep}))
        return

    import torch
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    from cm3d_b200.engine import measure_peaks
    from cm3d_b200.setup import build_system

    partitioned = args.partition and world > 1
    wls, desc, dsteps = workload(args.workload, seed=1 if partitioned else 1 + rank)
    steps = args.steps if args.steps is not None else dsteps
    warmup = args.warmup if args.warmup is not None else 20
    systems = [build_system(w) for w in wls]
    natoms_job = sum(sm.natoms for sm in systems)
    if partitioned:
        # whole systems dealt to the ranks by LPT on the per-system cost model
        from cm3d_b200.shard import imbalance, partition, system_cost
        costs = [system_cost(sm) for sm in systems]
        parts = partition(costs, world)
        if any(len(p) == 0 for p in parts):
            raise SystemExit("--partition: fewer systems than ranks")
        shard_info = {"ranks": world, "imbalance": imbalance(costs, parts),
                      "systems_per_rank": [len(p) for p in parts]}
        systems = [systems[k] for k in parts[rank]]
        wls = [wls[k] for k in parts[rank]]
    peaks = measured_peaks()
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    fp32, fp64 = measure_peaks(local)
    flush = l2_flusher(local)

    pin = (args.tpa, args.pair_kernel) if args.tpa else None
    m = mixed_arm(systems, local, steps, warmup, flush, fp32, hbm, args.workload, min(steps, 100), dist, pin)
    n = m["n"]
    ms = m["ms"]
    value = (natoms_job if partitioned else world * n) * steps / (ms / 1e3)
    dt_e2e, h2d, d2h, e2e_steps = m["e2e"]
    atoms_all = natoms_job if partitioned else world * n
    e2e_value = atoms_all * e2e_steps / dt_e2e

    plain = None
    if not args.no_plain:
        psteps = 10 if len(systems) > 1 else min(steps, 300)
        plain = plain_arm(systems, local, psteps, 3 if len(systems) > 1 else 10, flush)
        pms = plain["ms_per_step"]
        if dist:
            t = torch.tensor([pms], dtype=torch.float64, device=f"cuda:{local}")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            pms = float(t.item())
        plain["ms_per_step"] = pms
        plain["value"] = atoms_all / (pms / 1e3)
        plain["speedup_mixed_vs_plain"] = value / plain["value"]

    other = {}
    if not args.no_extra and args.workload != "water12288" and world == 1:
        wwl, wdesc, _ = workload("water12288", seed=1)
        wsys = [build_system(w) for w in wwl]
        wm = mixed_arm(wsys, local, 500, 20, flush, fp32, hbm, "water12288", 100)
        wval = wm["n"] * 500 / (wm["ms"] / 1e3)
        wplain = None if args.no_plain else plain_arm(wsys, local, 300, 10, flush)
        other["water12288"] = {
            "workload": wdesc, "value": wval, "unit": UNIT, "ms_per_step": wm["ms"] / 500, "steps": 500,
            "ns_per_day": (500 / (wm["ms"] / 1e3)) * float(wsys[0]["dt"]) * 86400.0 / 1e3,
            "plain_fp64": wplain,
            "speedup_mixed_vs_plain": (wval / wplain["value"]) if wplain else None,
            "roofline": wm["roofline"], "autotune": wm["autotune"],
            "status": {k: wm["status"][k] for k in ("rebuilds", "resets")}}

    if not args.no_extra and world == 1:
        # the single large box (C3) and the small argon box (C1), mixed and
        # plain FP64, with the pair kernel's roofline
        for wname, wsteps, wwarm, psteps in (("water331776", 50, 5, 10), ("argon864", 500, 20, 300)):
            if args.workload == wname:
                continue
            wwl, wdesc, _ = workload(wname, seed=1)
            wsys = [build_system(w) for w in wwl]
            wm = mixed_arm(wsys, local, wsteps, wwarm, flush, fp32, hbm, wname, 10)
            wval = wm["n"] * wsteps / (wm["ms"] / 1e3)
            wplain = None if args.no_plain else plain_arm(wsys, local, psteps, 3, flush)
            other[wname] = {
                "workload": wdesc, "value": wval, "unit": UNIT, "ms_per_step": wm["ms"] / wsteps,
                "steps": wsteps, "ns_per_day": (wsteps / (wm["ms"] / 1e3)) * float(wsys[0]["dt"]) * 86400.0 / 1e3,
                "plain_fp64": wplain, "speedup_mixed_vs_plain": (wval / wplain["value"]) if wplain else None,
                "roofline": wm["roofline"], "autotune": wm["autotune"],
                "status": {k: wm["status"][k] for k in ("rebuilds", "resets", "table_underflow")}}
            if wname == "water331776" and wm["autotune"].get("kernel") != "compact":
                # the step's fastest choice is another kernel (the step is
                # bound by the reciprocal space on its side stream): the
                # compact pair kernel's own roofline, measured the same way
                other[wname]["roofline_compact"] = compact_roofline(wsys, local, wname, fp32, hbm)
        other["abutane1024"] = intra_arm(local, 1024, 200, 10, flush)

    nve = None
    if not args.no_extra and world == 1:
        nve = nve_arm(local)

    serving = None
    if not args.no_extra and not args.no_serving and world == 1:
        if args.serving_sweep:
            serving = [serving_arm(r, args.serving_window, local, not args.no_plain) for r in (0.5, 1.0, 2.0, 4.0, 8.0)]
        else:
            serving = serving_arm(4.0, 5.0, local, not args.no_plain)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cores = max(1, min(os.cpu_count() or 1, 64))
        csteps = cpu_bounded_steps(wls, cores, 10)
        cpu = (cpu_reference(wls, cores, csteps, min(2, csteps)) if ref_bench_bin()
               else cpu_port(systems, csteps))

    if rank == 0:
        dt_ps = float(systems[0]["dt"])
        per = np.array(m["per_step_ms"])
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": steps,
            "warmup": warmup, "ms_per_step": ms / steps, "higher_is_better": True,
            "scaling": "strong" if partitioned else "weak", "vs_baseline": None, "dtype": "f32",
            "accumulate": "f64",
            "data": "synthetic (seeded; CM3D input decks from cm3d_b200.configs)",
            "config": {"workload": desc, "natoms": n, "systems": len(systems),
                       "mode": "mixed (FP32 compute, FP64 accumulation), one batch",
                       "parallelism": (f"{world} ranks, the ensemble's systems split by LPT ({shard_info})"
                                       if partitioned else
                                       f"{world} ranks, each its own ensemble (seed + rank)" if world > 1
                                       else "one GPU"),
                       "l2": "flushed between timed steps (256 MB write outside the step's events)",
                       "timing": "CUDA events around each step's graph replay on the engine stream; "
                                 "max over ranks"},
            "ns_per_day": (steps / (ms / 1e3)) * dt_ps * 86400.0 / 1e3,
            "latency": {"unit": "ms per step (device)", "p50": float(np.percentile(per, 50)),
                        "p99": float(np.percentile(per, 99))},
            "gpu_launches": m["launches"],
            "roofline": m["roofline"],
            "autotune": m["autotune"],
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "steps": e2e_steps},
            "plain_fp64": plain,
            "other_workloads": other,
            "serving": serving,
            "nve_drift": nve,
            "peaks": {"fp32_tflops": fp32, "fp64_tflops": fp64, "hbm_gbs": hbm},
            "clocks": m["clocks"],
            "status": {k: m["status"][k] for k in ("rebuilds", "resets", "overflows", "table_underflow")},
            "final_energy": {"poter_sum": float(sum(e["poter"] for e in m["energies"])),
                             "zke_sum": float(sum(e["zke"] for e in m["energies"]))},
        }
        print(json.dumps(line))
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()

"""Benchmark of the CM3D nonbonded engine on one B200 (or N replicas).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload water12288|argon864|water331776]

A step is one CM3D RESPA outer step (integrate/md_step.c:62: inner bonded
levels, neighbour-list check/rebuild, full nonbonded + Ewald forces, kicks)
of the workload on the GPU.  The default workload is the flexible-water box of
4096 molecules (12,288 atoms, 16^3 grid, L = 49.66 A, Ewald alpha 0.31,
kmax 7, rc 10 A, RESPA 0.5/2 fs) run for the 1000 outer steps the workload
names; inputs are synthetic and seeded (cm3d_b200.configs).

Printed: one JSON line (rank 0) with the contract's keys plus
  plain_fp64   the same run through the plain FP64 one-system engine
  roofline     the fused pair kernel against its FP32 / HBM roofline
  cpu_baseline CM3D itself (oracle/_ref/ref_bench) on this host's cores
  e2e          the same metric through the public API with host buffers
Under torchrun (N > 1) every rank runs an independent replica (the path has
no collective: "replicas only"); value = all ranks' atom-steps / max time.
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
BYTES_PAIR = 4.0                  # one 32-bit neighbour index
BYTES_ATOM = 16.0 + 24.0          # float4 position/charge in, FP64 force out


def workload(name: str, seed: int):
    from cm3d_b200 import configs
    if name == "water12288":
        return configs.water_box(ngrid=16, seed=seed, ntime=1000), \
            "water-12288: 4096 flexible 3-site waters on a 16^3 grid, L 49.66 A, alpha 0.31, kmax 7, " \
            "rc 10 A, skin 0.5 A, RESPA 0.5/2 fs (nres_intra 4), 300 K"
    if name == "water331776":
        return configs.water_box(ngrid=48, seed=seed, skin=1.5, kmax=21, ntime=500), \
            "water-331776: 110592 flexible 3-site waters on a 48^3 grid, L 148.98 A, alpha 0.31, kmax 21, " \
            "rc 10 A, skin 1.5 A, RESPA 0.5/2 fs"
    if name == "argon864":
        return configs.argon_fcc(seed=seed, ntime=1000), \
            "argon-864: LJ argon FCC 6^3x4, rho* 0.8442, rc 2.5 sigma, skin 0.3 sigma, dt 5 fs, 120 K"
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


def timed_run(eng, steps: int, warmup: int, istep0: int, flush) -> tuple[float, int]:
    """W untimed steps, then K steps each timed on the device (CUDA events
    around the step's graph replay on the engine's stream), with an L2 flush
    between steps outside the timed events.  Returns (total ms, kernels)."""
    istep = istep0
    for _ in range(warmup):
        eng.step(istep, 1)
        istep += 1
    eng.synchronize()
    eng.enable_timing(2)
    l0 = eng.launch_count()
    for _ in range(steps):
        flush()
        eng.step(istep, 1)
        istep += 1
    ms, n = eng.kernel_time(4)
    launches = eng.launch_count() - l0
    eng.enable_timing(0)
    return ms, launches


def pinned(n: int):
    try:
        import torch
        return torch.empty(n, dtype=torch.float64, pin_memory=True).numpy()
    except Exception:
        return np.empty(n)


def e2e_run(eng, steps: int, istep0: int, n: int) -> tuple[float, int, int]:
    """The public API with host buffers: every step uploads positions and
    velocities from pinned host memory, runs one step, and reads positions,
    velocities and the energies back (CM3D's host loop owning the state)."""
    px, vx = [pinned(3 * n).reshape(3, n) for _ in range(2)]
    px[:] = eng.positions()
    vx[:] = eng.velocities()
    eng.synchronize()
    t0 = time.perf_counter()
    for s in range(steps):
        eng.set_positions(px)
        eng.set_velocities(vx)
        eng.step(istep0 + s, 1)
        px[:] = eng.positions()
        vx[:] = eng.velocities()
        eng.energies()
    dt = time.perf_counter() - t0
    h2d = 2 * 3 * n * 8
    d2h = 2 * 3 * n * 8 + 72 * 8
    return dt, h2d, d2h


def roofline(eng, steps: int, istep0: int, n: int, fp32_tflops: float, hbm_gbs: float) -> dict:
    """Time the fused pair kernel with CUDA events around every launch (eager
    launches on the engine's stream) and compare with its roofline: the
    slower of its algorithmic bytes / HBM bandwidth and its algorithmic flops
    / FP32 FMA throughput (both measured)."""
    from cm3d_b200 import _abi
    eng.enable_timing(1)
    eng.step(istep0, steps)
    ms, launches = eng.kernel_time(0)
    eng.enable_timing(0)
    pte = len(eng.pair_list(_abi.LIST_TE)[0])
    pt = len(eng.pair_list(_abi.LIST_T)[0])
    flops = pte * FLOPS_ELEC_PAIR + pt * FLOPS_LJ_EXTRA
    if pte == 0:
        flops = pt * (FLOPS_ELEC_PAIR - 16 + FLOPS_LJ_EXTRA)
    nbytes = (pte if pte else pt) * BYTES_PAIR + n * BYTES_ATOM
    t = ms / 1e3 / max(launches, 1)
    t_bw = nbytes / (hbm_gbs * 1e9)
    t_fl = flops / (fp32_tflops * 1e12)
    traffic = None
    try:
        with open(os.path.join(ROOT, "profiles", "pair_kernel_traffic.json")) as fh:
            tr = json.load(fh)
        traffic = tr.get("dram_bytes_per_launch_scaled", tr.get("dram_bytes_per_launch"))
    except Exception:
        pass
    if t_fl >= t_bw:
        out = {"bound": "fp32", "achieved": flops / t / 1e12, "peak": fp32_tflops, "unit": "TFLOP/s",
               "frac": (flops / t / 1e12) / fp32_tflops}
    else:
        out = {"bound": "hbm", "achieved": nbytes / t / 1e9, "peak": hbm_gbs, "unit": "GB/s",
               "frac": (nbytes / t / 1e9) / hbm_gbs}
    out.update({"traffic": traffic, "kernel": "k_pair_mixed (fused LJ + real-space Ewald)",
                "ms_per_launch": t * 1e3, "launches": launches, "pairs_te": pte, "pairs_t": pt,
                "algorithmic_flops": flops, "algorithmic_bytes": nbytes,
                "hbm_frac": (nbytes / t / 1e9) / hbm_gbs,
                "fp32_frac": (flops / t / 1e12) / fp32_tflops,
                "peak_source": "fp32: cm3d_nb_measure_peaks (this run); hbm: MEASURED_PEAKS.json"})
    return out


# ------------------------------------------------------------ CPU baseline
def ref_bench_bin() -> str | None:
    p = os.path.join(ROOT, "oracle", "_ref", "ref_bench")
    return p if os.path.exists(p) else None


def cpu_reference(wl, steps: int, procs: int) -> dict:
    """CM3D itself on the host: `procs` independent replicas of the deck, each
    timing `steps` of CM3D's step() after its own start-up."""
    exe = ref_bench_bin()
    with tempfile.TemporaryDirectory() as tmp:
        jobs = []
        for p in range(procs):
            d = os.path.join(tmp, f"r{p}")
            inp = wl.write(d)
            jobs.append(subprocess.Popen([exe, os.path.basename(inp), str(steps)], cwd=d,
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True))
        res = []
        for j in jobs:
            out, _ = j.communicate()
            line = [ln for ln in out.splitlines() if ln.startswith("{")][-1]
            res.append(json.loads(line))
    tmax = max(r["seconds"] for r in res)
    total = sum(r["natoms"] * r["steps"] for r in res)
    return {"value": total / tmax, "unit": UNIT, "cores": procs, "kind": "reference",
            "sample": f"{procs} x CM3D step() (oracle/_ref/ref_bench, gcc -O2) for {steps} steps of the "
                      f"same deck after start-up; single-process {res[0]['atom_steps_per_s']:.4g} atom-steps/s",
            "single_process": res[0]["atom_steps_per_s"]}


def cpu_port(sysm, steps: int) -> dict:
    from oracle import Oracle
    o = Oracle(sysm)
    o.step_init()
    t0 = time.perf_counter()
    o.step(1, steps)
    dt = time.perf_counter() - t0
    return {"value": sysm.natoms * steps / dt, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": f"oracle (C restatement of CM3D) for {steps} steps"}


def cpu_sample_steps(natoms: int) -> int:
    # ~10-20 s of CM3D on one core: water runs at ~3.5e4 atom-steps/s
    return max(2, min(200, int(4.0e5 / max(natoms, 1))))


# ------------------------------------------------------------------- main
def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="water12288")
    ap.add_argument("--no-plain", action="store_true")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank != 0:
            return
        wl, desc = workload(args.workload, seed=1)
        steps = cpu_sample_steps(wl.natoms)
        procs = max(1, min(os.cpu_count() or 1, 32))
        if ref_bench_bin():
            base = cpu_reference(wl, steps, procs)
        else:
            from cm3d_b200.setup import build_system
            base = cpu_port(build_system(wl), steps)
        line = {"impl": "reference", "metric": METRIC, "value": base["value"], "unit": UNIT,
                "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": 1e3 * wl.natoms / base["value"] * base["cores"],
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic", "config": {"workload": desc, "natoms": wl.natoms,
                                                "parallelism": f"{base['cores']} host processes (replicas)"},
                "cpu_baseline": base,
                "e2e": {"value": base["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return

    import torch
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    from cm3d_b200 import _abi
    from cm3d_b200.engine import Engine, measure_peaks
    from cm3d_b200.setup import build_system

    wl, desc = workload(args.workload, seed=1 + rank)
    sysm = build_system(wl)
    n = sysm.natoms
    peaks = measured_peaks()
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    fp32, fp64 = measure_peaks(local)

    eng = Engine(sysm, mode=_abi.MIXED, device=local)
    eng.step_init()
    flush = l2_flusher(local)
    if dist:
        dist.barrier()
    torch.cuda.synchronize(local)
    with ClockSampler(local) as clk:
        ms, launches = timed_run(eng, args.steps, args.warmup, 1, flush)
    torch.cuda.synchronize(local)
    if dist:
        t = torch.tensor([ms], dtype=torch.float64, device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
        dist.barrier()
    value = world * n * args.steps / (ms / 1e3)
    status = eng.status()
    istep = 1 + args.warmup + args.steps

    # end to end through the public API with host buffers
    e2e_steps = min(args.steps, 300)
    if dist:
        dist.barrier()
    dt_e2e, h2d, d2h = e2e_run(eng, e2e_steps, istep, n)
    istep += e2e_steps
    if dist:
        t = torch.tensor([dt_e2e], dtype=torch.float64, device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dt_e2e = float(t.item())
    e2e_value = world * n * e2e_steps / dt_e2e

    roof = roofline(eng, 50, istep, n, fp32, hbm)
    en = eng.energies()
    eng.close()

    plain = None
    if not args.no_plain:
        psteps = min(args.steps, 300)
        pe = Engine(sysm, mode=_abi.PLAIN_FP64, device=local)
        pe.step_init()
        pms, _ = timed_run(pe, psteps, min(args.warmup, 10), 1, flush)
        pe.close()
        if dist:
            t = torch.tensor([pms], dtype=torch.float64, device=f"cuda:{local}")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            pms = float(t.item())
        pval = world * n * psteps / (pms / 1e3)
        plain = {"value": pval, "unit": UNIT, "ms_per_step": pms / psteps, "steps": psteps,
                 "speedup_mixed_vs_plain": value / pval}

    cpu = None
    if rank == 0 and world == 1:
        steps = cpu_sample_steps(n)
        cpu = cpu_reference(wl, steps, 1) if ref_bench_bin() else cpu_port(sysm, steps)

    if rank == 0:
        dt_ps = float(sysm["dt"])
        ms_step = ms / args.steps
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "accumulate": "f64",
            "data": "synthetic (seeded; CM3D input decks from cm3d_b200.configs)",
            "config": {"workload": desc, "natoms": n, "mode": "mixed (FP32 compute, FP64 accumulation)",
                       "parallelism": "replicas only" if world > 1 else "single system",
                       "l2": "flushed between timed steps (256 MB write outside the step's events)",
                       "timing": "CUDA events around each step's graph replay on the engine stream; "
                                 "max over ranks"},
            "ns_per_day": (args.steps / (ms / 1e3)) * dt_ps * 86400.0 / 1e3,
            "gpu_launches": launches,
            "roofline": roof,
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "steps": e2e_steps},
            "plain_fp64": plain,
            "peaks": {"fp32_tflops": fp32, "fp64_tflops": fp64, "hbm_gbs": hbm},
            "clocks": clk.summary(),
            "status": {k: status[k] for k in ("rebuilds", "resets", "overflows", "table_underflow")},
            "final_energy": {"poter": en["poter"], "zke": en["zke"]},
        }
        print(json.dumps(line))
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()

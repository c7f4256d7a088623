"""Host-side measurement helpers without a GPU: the NVE drift fit
(cm3d_b200.drift) and bench.py's CPU-sample sizing and roofline constants."""
import importlib.util
import os

import numpy as np
import pytest

from cm3d_b200.drift import conserved, drift_stats

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def load_bench():
    spec = importlib.util.spec_from_file_location("bench_module", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_drift_recovers_a_linear_trend_per_atom_per_ns():
    rng = np.random.default_rng(3)
    dt_ps, natoms, n = 0.005, 864, 1000
    t = np.arange(1, n + 1) * dt_ps
    slope_per_ps = 2.5                           # K per ps for the whole system
    ham = -5.0e5 + slope_per_ps * t + rng.normal(0.0, 0.05, n)
    s = drift_stats(ham, dt_ps, natoms)
    assert s["steps"] == n and s["natoms"] == natoms
    # K/ps -> K per atom per ns
    assert s["drift_per_atom_per_ns"] == pytest.approx(slope_per_ps * 1e3 / natoms, rel=1e-2)
    assert 0.0 < s["drift_se_per_atom_per_ns"] < 0.01 * abs(s["drift_per_atom_per_ns"])
    assert s["dE_cm3d"] == pytest.approx(np.std(ham, ddof=1) / abs(np.mean(ham)))
    assert s["ham_first"] == ham[0] and s["ham_last"] == ham[-1]


def test_conserved_energy_is_cm3d_nve_ham():
    assert conserved({"poth": -10.0, "potra": 2.5, "zke": 4.0, "poter": 99.0}) == -3.5


def test_cpu_sample_stays_within_its_budget():
    bench = load_bench()
    from cm3d_b200 import configs
    wls = configs.ensemble(64, seed=3)
    cores = 8
    steps = bench.cpu_bounded_steps(wls, cores, 10, budget_s=30.0)
    assert 1 <= steps <= 10
    per_core = sorted((bench.cpu_cost(w) for w in wls), reverse=True)
    est = max(sum(per_core) / cores, per_core[0])
    assert steps == 10 or steps * est <= 30.0
    # a tighter budget never gives more steps
    assert bench.cpu_bounded_steps(wls, cores, 10, budget_s=1e-3) <= steps


def test_roofline_work_per_pair():
    bench = load_bench()
    # an electrostatic pair 57 flops, 14 more with LJ; an LJ-only pair has no
    # charge product or erfc interpolation
    assert bench.FLOPS_ELEC_PAIR == 57.0 and bench.FLOPS_LJ_EXTRA == 14.0
    assert bench.FLOPS_LJ_ONLY == 55.0
    assert bench.BYTES_PAIR == 4.0 and bench.BYTES_ATOM == 40.0

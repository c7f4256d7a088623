"""The pair-kernel autotuner (cm3d_nb_autotune): it picks one of the
candidate lane counts and, for a single system with 3 or more cells per axis,
the gather, windowed or compact-window kernel; it leaves forces as they were
(lane count and kernel only reorder FP32 partial sums: relative 1e-6) and
energies within the mixed engine's bound (1e-5: the kernels sum energies in
FP32 chunks of different lengths before FP64), and a trajectory continues
after it as the mixed engine's bound requires."""
import numpy as np
import pytest

from conftest import force_scale, golden, rel_rms
from cm3d_b200 import _abi
from cm3d_b200.engine import Engine
from cm3d_b200.system import System

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("names", [["water216"], ["water4096"], ["argon864", "binary256"]],
                         ids=["single", "single-window", "batch"])
def test_autotune_keeps_state(engine_lib, names):
    ds = [golden(n) for n in names]
    e = Engine([System.from_arrays(d) for d in ds], mode=_abi.MIXED)
    e.step_init()
    f0 = e.forces(_abi.FXL)
    en0 = e.all_energies()
    res = e.autotune(reps=3)
    assert res["tpa"] in (4, 8, 16, 32)
    assert res["kernel"] in ("gather", "window", "system", "compact", "compact8")
    if len(names) > 1:
        assert res["kernel"] in ("gather", "system")   # a batch: gather or whole systems staged
    elif names[0] == "water216":
        assert res["kernel"] == "gather"               # too few cells for windows
    assert all(v > 0 for v in res["ms_per_launch"].values())
    f1 = e.forces(_abi.FXL)
    en1 = e.all_energies()
    fs = max(force_scale(d) / float(np.sqrt((d["amass"] ** 2).mean())) for d in ds)
    assert rel_rms(f1, f0, fs) <= 1e-6
    for a, b in zip(en0, en1):
        for k in ("vinter", "velec", "vewald", "U", "W", "zke"):
            assert abs(a[k] - b[k]) <= 1e-5 * max(abs(b[k]), 1.0), k
    e.step(1, 5)                      # the step graph is recaptured with the new lane count
    assert np.isfinite(e.positions()).all()
    e.close()

"""Shared test helpers.  GPU tests are marked `gpu`; everything else runs on
the CPU (`pytest -m "not gpu"`)."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")
CASES = ["lj2", "lj256", "abutane", "argon864", "water216", "binary256", "water4096"]


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (run on the B200 box)")


def golden(name: str) -> dict:
    with np.load(os.path.join(GOLDEN, f"{name}.npz")) as z:
        return {k: z[k] for k in z.files}


def xyz(d: dict, key: str) -> np.ndarray:
    return d[key].reshape(3, -1)


def rel_rms(a: np.ndarray, b: np.ndarray, scale: float = 0.0) -> float:
    """relative RMS error of force set a against reference b (over all atoms).
    `scale` is a per-component RMS force that floors the denominator: a
    perfect lattice (argon's FCC start) has forces that are pure round-off,
    against which a relative error means nothing"""
    den = max(float(np.sqrt((b * b).sum())), scale * np.sqrt(b.size))
    return float(np.sqrt(((a - b) ** 2).sum())) / (den if den > 0 else 1.0)


def force_scale(d: dict) -> float:
    """RMS force component of the system once it has moved (CM3D's forces
    after the dumped trajectory), used to floor relative errors"""
    key = "final_acc_l" if "final_acc_l" in d else "acc_l"
    f = d[key].reshape(3, -1) * d["amass"]
    return float(np.sqrt((f * f).mean()))


@pytest.fixture(scope="session")
def engine_lib():
    from cm3d_b200 import build
    build.build()
    from cm3d_b200 import engine
    return engine.load_library()

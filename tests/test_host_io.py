"""Host-owned state without a round trip per array: cm3d_nb_set_host_outputs
registers page-locked host arrays that every step fills with its final
positions (copied beside the step's list build and forces) and velocities;
cm3d_nb_step_host uploads the inputs and runs one step.

Checked against the call-per-array loop (set_positions, set_velocities,
step, positions, velocities) from the same state: positions and velocities
bit for bit and potential energies to summation-order rounding, after every
step, in graph and eager mode, for a batch and for one system; the inputs and
outputs may be the same arrays; unpinned arrays are refused.
"""
import numpy as np
import pytest

from conftest import golden
from cm3d_b200 import _abi
from cm3d_b200.engine import Engine, EngineError
from cm3d_b200.system import System

pytestmark = pytest.mark.gpu


def pinned(shape):
    import torch
    return torch.empty(int(np.prod(shape)), dtype=torch.float64, pin_memory=True).numpy().reshape(shape)


def systems(kind):
    if kind == "batch":
        from cm3d_b200 import configs, setup
        return [setup.build_system(w) for w in configs.ensemble(6, seed=5, nmin=300, nmax=1200)]
    return System.from_arrays(golden("water216"))


@pytest.mark.parametrize("kind", ["batch", "one"])
@pytest.mark.parametrize("graph", [True, False])
def test_step_host_matches_per_array_calls(engine_lib, kind, graph):
    nsteps = 8
    sysm = systems(kind)
    ref = Engine(sysm, mode=_abi.MIXED, use_graph=graph)
    ref.step_init()
    p, v = ref.positions(), ref.velocities()
    ref_traj = []
    for s in range(nsteps):
        ref.set_positions(p)
        ref.set_velocities(v)
        ref.step(1 + s, 1)
        p, v = ref.positions(), ref.velocities()
        ref_traj.append((p.copy(), v.copy(), ref.energies_table()))
    ref.close()

    e = Engine(sysm, mode=_abi.MIXED, use_graph=graph)
    e.step_init()
    px, vx = pinned((3, e.n)), pinned((3, e.n))
    px[:] = e.positions()
    vx[:] = e.velocities()
    e.set_host_outputs(px, vx)
    for s in range(nsteps):
        e.step_host(1 + s, px, vx)
        rp, rv, rt = ref_traj[s]
        np.testing.assert_array_equal(px, rp)
        np.testing.assert_array_equal(vx, rv)
        # (a system's reciprocal-space energy total is summed with FP64
        # atomics, in an order that can vary between runs)
        np.testing.assert_allclose(e.energies_table()["poter"], rt["poter"], rtol=1e-12, atol=0)
    # outputs off: the arrays keep the last step's state
    e.set_host_outputs(None, None)
    last = px.copy()
    e.step(1 + nsteps, 1)
    np.testing.assert_array_equal(px, last)
    e.close()


def test_host_outputs_must_be_page_locked(engine_lib):
    e = Engine(System.from_arrays(golden("water216")), mode=_abi.MIXED)
    with pytest.raises(EngineError, match="page-locked"):
        e.set_host_outputs(np.empty((3, e.n)), None)
    with pytest.raises(EngineError):
        e.set_host_outputs(pinned((3, e.n + 1)), None)
    e.close()

"""Batches: several independent systems in one context (cm3d_nb_create_batch).

Every system of a batch must come out as it does alone.  The checks:
  - its pair lists, cut out of the batch's lists, are bit-exact with CM3D's;
  - its forces and energies match the same system in its own context
    with the same pair kernel (relative 1e-12 / 1e-10).  A system with 3 or
    more cells per axis at the full force level runs in the compact kernel
    in a batch as alone; the others run in the list-gather kernel in a
    batch, and alone CM3D_NB_PAIR_KERNEL=list keeps them on it (a lone
    system would otherwise take the staged-window kernel); against the
    lone default kernel the forces agree to FP32 summation order (1e-6);
    and CM3D's within the mixed engine's stated bounds (forces 1e-5,
    energies 1e-5, virials 5e-5);
  - its trajectory tracks CM3D's per-step energies (2e-4, as for a single
    system) and its own single-context run (positions within 1e-9 A), with
    the same number of list rebuilds and RESETPOS events.

Systems are grouped by time step and RESPA levels, which a batch shares.
"""
import hashlib

import numpy as np
import pytest

from conftest import force_scale, golden, rel_rms, xyz
from cm3d_b200 import _abi
from cm3d_b200.engine import Engine, EngineError
from cm3d_b200.system import System
from tests.golden.make_golden import pair_key

pytestmark = pytest.mark.gpu

GROUPS = {
    "dt5fs": ["argon864", "binary256"],
    "dt1fs": ["lj256", "lj2"],
    "water": ["water216", "water4096"],
    # two copies of CM3D's abutane molecule: torsions, 1-4 pairs, cross bonds,
    # frozen atoms, and a batch whose systems all take the one-warp k-space tiles
    "tors": ["abutane", "abutane"],
    # two copies of CM3D's NVT deck: one Nose-Hoover chain per system
    "nvt": ["lj256nvt", "lj256nvt"],
}
ETOL, VTOL, FTOL = 1e-5, 5e-5, 1e-5
VIRIAL_KEYS = {"winter", "welec", "W", "prsi"}


TPA = 16          # lanes per atom, fixed so that a system sums its pairs alike alone and in a batch


def batch(names, **kw):
    ds = [golden(n) for n in names]
    return ds, Engine([System.from_arrays(d) for d in ds], mode=_abi.MIXED, tpa=TPA, **kw)


def close(a, b, tol):
    return abs(a - b) <= tol * max(abs(b), 1e-300) or abs(a - b) <= 1e-9


def lone_env(d):
    """CM3D_NB_PAIR_KERNEL for the lone run that uses the kernel the system
    gets in a batch: none where alone it takes the compact kernel, "list"
    (the gather kernel) otherwise"""
    one = Engine(System.from_arrays(d), mode=_abi.MIXED, tpa=TPA)
    one.get_ngbr()
    one.force(1)
    kind = one.pair_kernel()[0]
    one.close()
    return None if kind == "compact" else "list"


@pytest.mark.parametrize("group", list(GROUPS))
def test_batch_lists_bit_exact(engine_lib, group):
    ds, e = batch(GROUPS[group])
    e.get_ngbr()
    for tag, w in (("t", _abi.LIST_T), ("s", _abi.LIST_S), ("te", _abi.LIST_TE), ("se", _abi.LIST_SE)):
        i, j = e.pair_list(w)
        for s, d in enumerate(ds):
            a0, n = e.ranges[s]
            sel = (i >= a0) & (i < a0 + n)
            assert ((j[sel] >= a0) & (j[sel] < a0 + n)).all(), "a pair crosses systems"
            assert int(sel.sum()) == int(d[f"npr{tag}"][0]), (tag, s)
            if sel.any():
                h = hashlib.sha256(pair_key(i[sel] - a0, j[sel] - a0, n).tobytes()).hexdigest()
                assert h == str(d[f"list_{tag}_hash"]), (tag, s)
    e.close()


@pytest.mark.parametrize("group", list(GROUPS))
def test_batch_forces_and_energies(engine_lib, group, monkeypatch):
    names = GROUPS[group]
    ds, e = batch(names)
    e.get_ngbr()
    e.force(1)
    e.force(2)
    fb = e.forces(_abi.FXL)
    en = e.all_energies()
    e.close()
    for s, (name, d) in enumerate(zip(names, ds)):
        a0, n = e.ranges[s]
        one = Engine(System.from_arrays(d), mode=_abi.MIXED, tpa=TPA)
        one.get_ngbr()
        one.force(1)
        fw = one.forces(_abi.FXL)
        one.close()
        env = lone_env(d)
        if env:
            monkeypatch.setenv("CM3D_NB_PAIR_KERNEL", env)
        one = Engine(System.from_arrays(d), mode=_abi.MIXED, tpa=TPA)
        if env:
            monkeypatch.delenv("CM3D_NB_PAIR_KERNEL")
        one.get_ngbr()
        one.force(1)
        one.force(2)
        f1 = one.forces(_abi.FXL)
        e1 = one.energies()
        one.close()
        fs = force_scale(d) / float(np.sqrt((d["amass"] ** 2).mean()))
        assert rel_rms(fb[:, a0:a0 + n], f1, fs) <= 1e-12, name
        assert rel_rms(fb[:, a0:a0 + n], fw, fs) <= 1e-6, name
        assert rel_rms(fb[:, a0:a0 + n], xyz(d, "acc_l"), fs) <= FTOL, name
        for k in ("vinter", "velec", "vewald", "U", "W", "prsi", "zke", "vbond", "vbend"):
            assert close(en[s][k], e1[k], 1e-10), (name, k, en[s][k], e1[k])
        for k in ("vinter", "velec", "vewald", "U", "W", "prsi", "zke"):
            tol = VTOL if k in VIRIAL_KEYS else ETOL
            assert close(en[s][k], float(d[f"e0_{k}"][0]), tol), (name, k)


@pytest.mark.parametrize("graph", [False, True], ids=["eager", "graph"])
@pytest.mark.parametrize("group", list(GROUPS))
def test_batch_trajectory(engine_lib, group, graph, monkeypatch):
    names = GROUPS[group]
    ds, e = batch(names, use_graph=graph)
    nsteps = min(int(d["nsteps"][0]) for d in ds)
    e.step_init()
    for k in range(nsteps):
        e.step(1 + k, 1)
        en = e.all_energies()
        for s, d in enumerate(ds):
            ref = d["traj_eng"].reshape(-1, 8)
            for c, key in enumerate(("poter", "potra", "zke")):
                tol = 2e-4 if c != 1 else 2e-3
                assert close(en[s][key], ref[k, c], tol), (names[s], k, key)
    pos = e.positions()
    rb, rs = e.system_counts()
    e.close()
    for s, d in enumerate(ds):
        a0, n = e.ranges[s]
        env = lone_env(d)
        if env:
            monkeypatch.setenv("CM3D_NB_PAIR_KERNEL", env)
        one = Engine(System.from_arrays(d), mode=_abi.MIXED, tpa=TPA, use_graph=graph)
        if env:
            monkeypatch.delenv("CM3D_NB_PAIR_KERNEL")
        one.step_init()
        one.step(1, nsteps)
        p1 = one.positions()
        rb1, rs1 = one.system_counts()
        one.close()
        assert np.abs(pos[:, a0:a0 + n] - p1).max() <= 1e-9, names[s]
        assert rb[s] == rb1[0] and rs[s] == rs1[0], (names[s], rb[s], rb1[0], rs[s], rs1[0])


def test_host_buffers_and_energies_table(engine_lib):
    """positions/velocities into caller arrays (e.g. pinned) and the
    structured energies table give what the allocating calls give"""
    ds, e = batch(GROUPS["water"])
    e.step_init()
    e.step(1, 2)
    px = np.empty((3, e.n))
    assert e.positions(out=px) is px
    np.testing.assert_array_equal(px, e.positions())
    vx = np.empty((3, e.n))
    np.testing.assert_array_equal(e.velocities(out=vx), e.velocities())
    with pytest.raises(ValueError):
        e.positions(out=np.empty((e.n, 3)))
    tab = e.energies_table()
    for s, en in enumerate(e.all_energies()):
        for k in ("poter", "vinter", "velec", "vewald", "prsi", "zke"):
            assert tab[k][s] == en[k], k
        np.testing.assert_array_equal(tab["prs_tensor"][s], en["prs_tensor"])
    e.close()


def test_batch_rejects_mismatched_steps(engine_lib):
    with pytest.raises(EngineError, match="dt"):
        batch(["argon864", "water216"])
    d = golden("lj256")
    with pytest.raises(EngineError, match="mixed"):
        Engine([System.from_arrays(d), System.from_arrays(d)], mode=_abi.PLAIN_FP64)


def _thermostat_variants():
    """two NVT systems from CM3D's lj256nvt deck with other thermostat
    layouts: A splits the atoms over two thermostats (even / odd index), B
    leaves the first 16 atoms without a thermostat (ithm -1, as
    \\mol_therm_opt{none} beside a thermostatted species does)"""
    d = golden("lj256nvt")
    nc = int(d["nchain"][0])
    a = System.from_arrays(d)
    a["ntherm"] = np.array([2], dtype=np.int32)
    a["ithm"] = (np.arange(256) % 2).astype(np.int32)
    half = d["gkt"].copy()
    half[0] *= 0.5
    a["gkt"] = np.concatenate([half, half])
    a["mnh"] = np.concatenate([d["mnh"], d["mnh"]])
    a["nhc_eta"] = np.zeros(2 * nc)
    a["nhc_veta"] = np.zeros(2 * nc)
    b = System.from_arrays(d)
    ithm = np.zeros(256, dtype=np.int32)
    ithm[:16] = -1
    b["ithm"] = ithm
    return [a, b]


def test_nvt_thermostat_layouts_plain_match_oracle(engine_lib):
    """several thermostats in one system and atoms without a thermostat: the
    plain FP64 engine's chain state (cm3d_nb_get_nhc) and positions after 10
    steps against CM3D's algorithm (the oracle) to 1e-9"""
    from oracle import Oracle
    nsteps = 10
    for s in _thermostat_variants():
        one = Engine(s.copy(), mode=_abi.PLAIN_FP64)
        one.step_init()
        one.step(1, nsteps)
        eta1, veta1 = one.nhc_state()
        p1 = one.positions()
        one.close()
        o = Oracle(s.copy())
        o.step_init()
        o.step(1, nsteps)
        eo, vo = o.nhc_state()
        shape = (int(np.asarray(s["ntherm"]).ravel()[0]), int(np.asarray(s["nchain"]).ravel()[0]))
        assert eta1.shape == shape
        np.testing.assert_allclose(eta1, np.asarray(eo).reshape(shape), rtol=1e-9, atol=1e-12)
        np.testing.assert_allclose(veta1, np.asarray(vo).reshape(shape), rtol=1e-9, atol=1e-12)
        np.testing.assert_allclose(p1, o.positions(), rtol=0, atol=1e-9)


def test_nvt_thermostat_layouts_alone_and_in_batch(engine_lib, monkeypatch):
    """the same systems, with different numbers of thermostats, in one batch
    of the mixed engine: each system's chain state (also system 1's) and
    positions after 10 steps are bit for bit those of the system alone with
    the batch's pair kernel (the thermostats' kinetic sums run in a fixed
    order, whatever else shares the device)"""
    systems = _thermostat_variants()
    nsteps = 10
    e = Engine([s.copy() for s in systems], mode=_abi.MIXED, tpa=TPA)
    e.step_init()
    e.step(1, nsteps)
    pos = e.positions()
    states = [e.nhc_state(k) for k in range(2)]
    e.close()
    for k, s in enumerate(systems):
        a0, n = e.ranges[k]
        monkeypatch.setenv("CM3D_NB_PAIR_KERNEL", "list")
        one = Engine(s.copy(), mode=_abi.MIXED, tpa=TPA)
        monkeypatch.delenv("CM3D_NB_PAIR_KERNEL")
        one.step_init()
        one.step(1, nsteps)
        eta1, veta1 = one.nhc_state()
        p1 = one.positions()
        one.close()
        shape = (int(np.asarray(s["ntherm"]).ravel()[0]), int(np.asarray(s["nchain"]).ravel()[0]))
        assert states[k][0].shape == eta1.shape == shape
        np.testing.assert_allclose(states[k][0], eta1, rtol=1e-12, atol=1e-15)
        np.testing.assert_allclose(states[k][1], veta1, rtol=1e-12, atol=1e-15)
        assert np.abs(pos[:, a0:a0 + n] - p1).max() <= 1e-9

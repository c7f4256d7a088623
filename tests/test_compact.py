"""The compact-window pair path (nb_cwin.cu): one system with three or more
cells per axis, full force level.  Its list is the master full list
rewritten after each rebuild as 16-bit window indices; its kernel reads j
from the staged 27-cell window and the tables from bank-replicated copies.

Checked here:
  - it is the kernel a lone system with >= 3 cells per axis runs (one
    LJ interaction, several LJ interactions with the per-pair type map, no
    charges, charges), within the mixed bounds of CM3D's dumped forces,
    energies and virials or of the plain FP64 engine, and within FP32
    summation order of the window and list-gather kernels on the same lists;
  - a force evaluation repeats bit for bit (every sum in a fixed order);
  - a cell window larger than the kernel's capacity turns the path off on
    the host and the context falls back to the window kernel, with the same
    results;
  - the 331,776-atom water box (110,592 molecules, kmax 21, skin 1.5 A): the
    mixed engine's level-1 forces, energies and virials against the plain
    FP64 engine (itself pinned to CM3D at 1e-11 by the golden fixtures) on
    the same positions.

Tolerances (the mixed engine's): forces relative RMS <= 1e-5, energies
<= 1e-5, virials <= 5e-5 against CM3D's dumps, <= 1e-5 against the plain
FP64 engine at 331,776 atoms.
"""
import json
import os

import numpy as np
import pytest

from conftest import force_scale, golden, rel_rms, xyz
from cm3d_b200 import _abi
from cm3d_b200.engine import Engine
from cm3d_b200.system import System

pytestmark = pytest.mark.gpu

FTOL, ETOL, VTOL = 1e-5, 1e-5, 5e-5
ENERGY_KEYS = ("vinter", "vhinter", "velec", "vewald", "U", "zke")
VIRIAL_KEYS = ("winter", "welec", "W", "prsi")


def close(a, b, tol):
    return abs(a - b) <= tol * max(abs(b), 1e-300) or abs(a - b) <= 1e-9


def error_stats(f, ref):
    """relative RMS force error, and the largest per-atom error |dF_i| over
    the RMS atom force (a per-atom relative error means little for atoms
    whose force nearly cancels; it is reported too)"""
    d = np.sqrt(((f - ref) ** 2).sum(axis=0))
    mag = np.sqrt((ref * ref).sum(axis=0))
    rms_f = float(np.sqrt((mag * mag).mean()))
    return {"rel_rms": float(np.sqrt(((f - ref) ** 2).sum() / (ref * ref).sum())),
            "max_atom_over_rms": float(d.max() / rms_f),
            "max_atom_rel": float((d / np.maximum(mag, 1e-300)).max())}


def record(name, stats):
    """error figures of a configuration: printed, and appended to the file
    CM3D_NB_ERRLOG names (a JSON line each) when it is set"""
    line = json.dumps({"config": name, **stats})
    print("ERRSTAT", line)
    path = os.environ.get("CM3D_NB_ERRLOG")
    if path:
        with open(path, "a") as fh:
            fh.write(line + "\n")


def level1(sysm, mode, env=None, tpa=0, monkeypatch=None):
    if env is not None:
        monkeypatch.setenv("CM3D_NB_PAIR_KERNEL", env)
    e = Engine(sysm, mode=mode, tpa=tpa)
    if env is not None:
        monkeypatch.delenv("CM3D_NB_PAIR_KERNEL")
    e.get_ngbr()
    e.force(1)
    kind = e.pair_kernel()[0] if mode == _abi.MIXED else "plain"
    f = e.forces(_abi.FXL)
    e.force(2)
    en = e.energies()
    e.close()
    return f, en, kind


@pytest.mark.parametrize("name", ["argon864", "water4096"])
def test_compact_is_default_and_matches(engine_lib, name, monkeypatch):
    d = golden(name)
    out = {}
    for kind, env in (("compact", None), ("window", "window"), ("gather", "list")):
        f, en, used = level1(System.from_arrays(d), _abi.MIXED, env, monkeypatch=monkeypatch)
        assert used == kind, (kind, used)
        out[kind] = (f, en)
    fs = force_scale(d) / float(np.sqrt((d["amass"] ** 2).mean()))
    for kind, (f, en) in out.items():
        assert rel_rms(f, xyz(d, "acc_l"), fs) <= FTOL, kind
        for k in ("vinter", "velec", "vewald", "U", "W", "prsi", "zke"):
            tol = VTOL if k in VIRIAL_KEYS else ETOL
            assert close(en[k], float(d[f"e0_{k}"][0]), tol), (kind, k, en[k], float(d[f"e0_{k}"][0]))
    for kind in ("window", "gather"):
        assert rel_rms(out["compact"][0], out[kind][0], fs) <= 1e-6, kind
        for k in ("vinter", "velec", "W"):
            assert close(out["compact"][1][k], out[kind][1][k], 2e-6), (kind, k)


def test_compact_binary_mixture_several_lj_types(engine_lib, monkeypatch):
    """4000-atom charged LJ binary (three LJ interactions: the per-pair type
    map path), positions shaken off the FCC start: the compact kernel against
    the plain FP64 engine and the gather kernel on the same positions"""
    from cm3d_b200 import configs, setup
    sm = setup.build_system(configs.charged_binary(natoms=4000, seed=3))
    rng = np.random.default_rng(5)
    pos = None
    out = {}
    for key, mode, env in (("plain", _abi.PLAIN_FP64, None), ("compact", _abi.MIXED, None),
                           ("gather", _abi.MIXED, "list")):
        if env:
            monkeypatch.setenv("CM3D_NB_PAIR_KERNEL", env)
        e = Engine(sm, mode=mode)
        if env:
            monkeypatch.delenv("CM3D_NB_PAIR_KERNEL")
        if pos is None:
            pos = e.positions() + rng.normal(scale=0.15, size=(3, e.n))
        e.set_positions(pos)
        e.get_ngbr()
        e.force(1)
        if mode == _abi.MIXED:
            assert e.pair_kernel()[0] == key
        f = e.forces(_abi.FXL)
        e.force(2)
        out[key] = (f, e.energies())
        e.close()
    st = error_stats(out["compact"][0], out["plain"][0])
    record("binary4000", {"level1": st})
    assert st["rel_rms"] <= FTOL
    assert rel_rms(out["compact"][0], out["gather"][0]) <= 1e-6
    for k in ENERGY_KEYS:
        assert close(out["compact"][1][k], out["plain"][1][k], ETOL), k
    for k in VIRIAL_KEYS:
        assert close(out["compact"][1][k], out["plain"][1][k], VTOL), k


def test_compact_repeats_bit_for_bit(engine_lib):
    d = golden("water4096")
    e = Engine(System.from_arrays(d), mode=_abi.MIXED)
    e.get_ngbr()
    runs = []
    for _ in range(3):
        e.force(1)
        runs.append((e.forces(_abi.FXL), e.getsvirter_e(), e.getsvirter()))
    assert e.pair_kernel()[0] == "compact"
    # every block's window copies (bulk copies on an mbarrier) completed
    assert e.status()["stage_timeouts"] == 0
    e.close()
    for f, ve, vl in runs[1:]:
        np.testing.assert_array_equal(f, runs[0][0])
        assert ve["velec"] == runs[0][1]["velec"] and ve["welec"] == runs[0][1]["welec"]
        np.testing.assert_array_equal(ve["welectensor"], runs[0][1]["welectensor"])
        assert vl["vinter"] == runs[0][2]["vinter"] and vl["winter"] == runs[0][2]["winter"]


def test_compact_window_overflow_falls_back(engine_lib, monkeypatch):
    """CM3D_NB_CW_CAP caps the window below water4096's ~5200-atom windows:
    the host-driven build finds the overflow and turns the compact path off;
    forces and energies are then the window kernel's"""
    d = golden("water4096")
    monkeypatch.setenv("CM3D_NB_CW_CAP", "1000")
    f, en, used = level1(System.from_arrays(d), _abi.MIXED)
    monkeypatch.delenv("CM3D_NB_CW_CAP")
    assert used == "window"
    fw, enw, _ = level1(System.from_arrays(d), _abi.MIXED, "window", monkeypatch=monkeypatch)
    np.testing.assert_array_equal(f, fw)
    # (the window kernel's energy sums end in FP64 atomics: last-bit order)
    assert close(en["W"], enw["W"], 1e-13) and close(en["U"], enw["U"], 1e-13)


@pytest.fixture(scope="module")
def water331776():
    from cm3d_b200 import configs, setup
    wl = configs.water_box(ngrid=48, seed=1, skin=1.5, kmax=21, ntime=500, placement="octant")
    return setup.build_system(wl)


def test_water331776_mixed_against_plain_fp64(engine_lib, water331776):
    """the C3 box: level-1 forces (pairs + k-space + ecorr), the pair terms
    alone, energies and virials of the mixed engine against the plain FP64
    engine on the same positions"""
    sm = water331776
    fp, ep, _ = level1(sm, _abi.PLAIN_FP64)
    fm, em, kind = level1(sm, _abi.MIXED)
    assert kind == "compact"
    st = error_stats(fm, fp)
    # the real-space pair terms alone (the compact kernel's own error)
    pair = {}
    for mode in (_abi.PLAIN_FP64, _abi.MIXED):
        e = Engine(sm, mode=mode)
        e.get_ngbr()
        e.zero_forces(_abi.FXL)
        e.force_ter(1)
        e.force_ter_e(1)
        pair[mode] = (e.forces(_abi.FXL), e.getsvirter(), e.getsvirter_e())
        e.close()
    sp = error_stats(pair[_abi.MIXED][0], pair[_abi.PLAIN_FP64][0])
    rel = {k: abs(em[k] - ep[k]) / abs(ep[k]) for k in ENERGY_KEYS + VIRIAL_KEYS if ep[k] != 0}
    record("water331776", {"level1": st, "pairs": sp, "energies_rel": rel})
    assert st["rel_rms"] <= FTOL
    assert sp["rel_rms"] <= FTOL
    for k in ENERGY_KEYS:
        assert close(em[k], ep[k], ETOL), (k, em[k], ep[k])
    for k in VIRIAL_KEYS:
        assert close(em[k], ep[k], 1e-5), (k, em[k], ep[k])
    vm, vp = pair[_abi.MIXED][2]["welectensor"], pair[_abi.PLAIN_FP64][2]["welectensor"]
    assert np.abs(vm - vp).max() <= 1e-5 * np.abs(vp).max()


# ------------------------------------------------------------------ error table
def _mixed_vs_plain(sysm, positions=None):
    """level-1 forces, energies and virials of the mixed engine (default
    kernels) against the plain FP64 engine on the same positions"""
    out = {}
    for key, mode in (("plain", _abi.PLAIN_FP64), ("mixed", _abi.MIXED)):
        e = Engine(sysm, mode=mode)
        if positions is not None:
            e.set_positions(positions)
        e.get_ngbr()
        e.force(1)
        f = e.forces(_abi.FXL)
        e.force(2)
        out[key] = (f, e.energies(), e.pair_kernel()[0] if mode == _abi.MIXED else "plain")
        e.close()
    st = error_stats(out["mixed"][0], out["plain"][0])
    rel = {k: abs(out["mixed"][1][k] - out["plain"][1][k]) / abs(out["plain"][1][k])
           for k in ENERGY_KEYS + VIRIAL_KEYS if out["plain"][1][k] != 0}
    return st, rel, out["mixed"][2]


@pytest.mark.parametrize("name", ["argon864", "water12288"])
def test_error_table_small_configs(engine_lib, name):
    """C1 (argon, its FCC start shaken by 0.1 A so that forces are not pure
    round-off) and C2 (water, the bench's start): mixed against plain FP64"""
    from cm3d_b200 import configs, setup
    wl = configs.argon_fcc(seed=1) if name == "argon864" else configs.water_box(ngrid=16, seed=1)
    sm = setup.build_system(wl)
    pos = None
    if name == "argon864":
        pos = np.asarray(wl.pos, float).T + np.random.default_rng(2).normal(scale=0.1, size=(3, wl.natoms))
    st, rel, kind = _mixed_vs_plain(sm, pos)
    record(name, {"kernel": kind, "level1": st, "energies_rel": rel})
    assert st["rel_rms"] <= FTOL
    for k, v in rel.items():
        assert v <= (VTOL if k in VIRIAL_KEYS else ETOL), (k, v)


@pytest.mark.parametrize("ngrid", [6, 25])
def test_error_table_serving_jobs(engine_lib, ngrid):
    """C5: water jobs at the two ends of the serving workload's sizes (216
    and 15,625 molecules; rc = min(10 A, 0.45 L), alpha = 3.1 / rc, kmax =
    ceil(7 L / 49.66))"""
    from cm3d_b200 import configs, setup
    req = configs.ServingRequest(index=0, arrival=0.0, ngrid=ngrid, nsteps=500, seed=5)
    sm = setup.build_system(configs.serving_workload(req))
    st, rel, kind = _mixed_vs_plain(sm)
    record(f"serving_water{3 * ngrid ** 3}", {"kernel": kind, "level1": st, "energies_rel": rel})
    assert st["rel_rms"] <= FTOL
    for k, v in rel.items():
        assert v <= (VTOL if k in VIRIAL_KEYS else ETOL), (k, v)

"""GPU engine against CM3D (golden fixtures dumped from the reference) and the
CPU oracle.  Every call goes through the C ABI (libcm3d_nb.so) via Engine.

Tolerances
  pair lists          bit-exact (sorted (min, max) pairs hashed), both modes
  plain FP64 engine   relative RMS force error <= 1e-11 (only the summation
                      order differs from CM3D), energies relative <= 1e-10
  mixed engine        relative RMS force error <= 1e-5 against CM3D's FP64
                      energies relative <= 1e-5,
                      virials (and the pressure) relative <= 5e-5: a virial
                      sums -r^2 f over ~1e5 pairs of both signs, so the FP32
                      rounding of each pair term (~5e-7) is amplified by the
                      cancellation more than in a per-atom force
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

MODES = [_abi.PLAIN_FP64, _abi.MIXED]
MODE_ID = {_abi.PLAIN_FP64: "plain", _abi.MIXED: "mixed"}
FTOL = {_abi.PLAIN_FP64: 1e-11, _abi.MIXED: 1e-5}
ETOL = {_abi.PLAIN_FP64: 1e-10, _abi.MIXED: 1e-5}
VTOL = {_abi.PLAIN_FP64: 1e-10, _abi.MIXED: 5e-5}
VIRIAL_KEYS = {"winter", "welec", "W", "prsi"}
ALL = ["lj2", "lj256", "abutane", "argon864", "water216", "binary256", "water4096"]
DYN = ALL


def engine(name, mode, **kw):
    d = golden(name)
    return d, Engine(System.from_arrays(d), mode=mode, **kw)


class close:
    """|a - b| <= tol |b| (or an absolute 1e-9); truthy, and prints the
    numbers when an assertion on it fails"""

    def __init__(self, a, b, tol):
        self.a, self.b, self.tol = float(a), float(b), tol

    def __bool__(self):
        return abs(self.a - self.b) <= self.tol * max(abs(self.b), 1e-300) or abs(self.a - self.b) <= 1e-9

    def __repr__(self):
        rel = abs(self.a - self.b) / max(abs(self.b), 1e-300)
        return f"close(got={self.a!r}, want={self.b!r}, rel={rel:.3e}, tol={self.tol:g})"


@pytest.mark.parametrize("mode", MODES, ids=lambda m: MODE_ID[m])
@pytest.mark.parametrize("name", ALL)
def test_pair_lists_bit_exact(engine_lib, name, mode):
    d, e = engine(name, mode)
    e.get_ngbr()
    n = int(d["natoms"][0])
    for tag, w in (("t", _abi.LIST_T), ("s", _abi.LIST_S), ("te", _abi.LIST_TE), ("se", _abi.LIST_SE)):
        i, j = e.pair_list(w)
        assert len(i) == int(d[f"npr{tag}"][0]), tag
        if len(i):
            h = hashlib.sha256(pair_key(i, j, n).tobytes()).hexdigest()
            assert h == str(d[f"list_{tag}_hash"]), tag
    e.close()


@pytest.mark.parametrize("mode", MODES, ids=lambda m: MODE_ID[m])
@pytest.mark.parametrize("name", ALL)
def test_force_terms(engine_lib, name, mode):
    d, e = engine(name, mode, need_short=True)
    e.get_ngbr()
    tol = FTOL[mode]
    fs = force_scale(d)
    # LJ: force_ter(1) adds the full force to fxl and the switched part to fxs
    e.zero_forces(_abi.FXL)
    e.zero_forces(_abi.FXS)
    e.force_ter(1)
    assert rel_rms(e.forces(_abi.FXL), xyz(d, "f_lj_l"), fs) <= tol
    if "f_lj_s" in d:                  # not stored for the large fixtures
        assert rel_rms(e.forces(_abi.FXS), xyz(d, "f_lj_s"), fs) <= tol
    v = e.getsvirter()
    assert close(v["vinter"], d["lj_vinter"][0], ETOL[mode])
    assert close(v["vhinter"], d["lj_vhinter"][0], ETOL[mode])
    assert close(v["winter"], d["lj_winter"][0], VTOL[mode])
    # real-space Ewald: force_ter_e(1)
    e.zero_forces(_abi.FXL)
    e.zero_forces(_abi.FXS)
    e.force_ter_e(1)
    assert rel_rms(e.forces(_abi.FXL), xyz(d, "f_el_l"), fs) <= tol
    if "f_el_s" in d:
        assert rel_rms(e.forces(_abi.FXS), xyz(d, "f_el_s"), fs) <= tol
    v = e.getsvirter_e()
    assert close(v["velec"], d["el_velec"][0], ETOL[mode])
    assert close(v["welec"], d["el_welec"][0], VTOL[mode])
    if int(d["ncharge"][0]) > 0:
        e.zero_forces(_abi.FXL)
        e.fk_ewald()
        assert rel_rms(e.forces(_abi.FXL), xyz(d, "f_k"), fs) <= tol
        e.zero_forces(_abi.FXL)
        e.ecorr()
        assert rel_rms(e.forces(_abi.FXL), xyz(d, "f_ecorr"), fs) <= FTOL[_abi.PLAIN_FP64]
    e.close()


@pytest.mark.parametrize("mode", MODES, ids=lambda m: MODE_ID[m])
@pytest.mark.parametrize("name", ALL)
def test_short_level(engine_lib, name, mode):
    """force_ter(...,0) over the s list with the RESPA switch, force_ter_e(...,0)
    over the se list with CM3D's fall-through (no switch, full cutoff)"""
    d, e = engine(name, mode)
    e.get_ngbr()
    fs = force_scale(d)
    for key, fn in (("f_lj_short", e.force_ter), ("f_el_short", e.force_ter_e)):
        if key not in d:          # not stored for the large fixtures
            continue
        e.zero_forces(_abi.FXS)
        fn(0)
        assert rel_rms(e.forces(_abi.FXS), xyz(d, key), fs) <= FTOL[mode], key
    e.close()


@pytest.mark.parametrize("mode", MODES, ids=lambda m: MODE_ID[m])
@pytest.mark.parametrize("name", DYN)
def test_level1_forces_and_energies(engine_lib, name, mode):
    d, e = engine(name, mode)
    e.get_ngbr()
    e.force(1)
    fs = force_scale(d) / float(np.sqrt((d["amass"] ** 2).mean()))
    assert rel_rms(e.forces(_abi.FXL), xyz(d, "acc_l"), fs) <= FTOL[mode]
    e.force(2)
    en = e.energies()
    for k in ("vinter", "velec", "vewald", "U", "W", "prsi", "zke"):
        tol = VTOL[mode] if k in VIRIAL_KEYS else ETOL[mode]
        assert close(en[k], float(d[f"e0_{k}"][0]), tol), k
    e.close()


def frozen_zeroed(d, f):
    """f with the frozen atoms' rows zeroed, as freeze_atom leaves a level"""
    f = f.copy()
    if int(d.get("nfreeze", [0])[0]) > 0:
        f[:, d["ifreeze"]] = 0.0
    return f


@pytest.mark.parametrize("name", DYN)
def test_bonded_level(engine_lib, name):
    """force(2): bonds + bends + cross bonds, then rmass and freeze"""
    d, e = engine(name, _abi.MIXED)
    e.force(2)
    m = d["amass"]
    want = xyz(d, "f_bond") + xyz(d, "f_bend")
    if "f_bondx" in d:
        want = want + xyz(d, "f_bondx")
    want = frozen_zeroed(d, want / m)
    # the generated molecules start at exactly r0 / theta0, where the bonded
    # forces are round-off: floor the denominator with the system's force scale
    fs = force_scale(d) / float(np.sqrt((m ** 2).mean()))
    assert rel_rms(e.forces(_abi.FXA), want, fs) <= 1e-12
    e.close()


@pytest.mark.parametrize("graph", [False, True], ids=["eager", "graph"])
@pytest.mark.parametrize("mode", MODES, ids=lambda m: MODE_ID[m])
@pytest.mark.parametrize("name", DYN)
def test_trajectory(engine_lib, name, mode, graph):
    """CM3D's step() for the dumped number of steps: per-step energies,
    final positions and the rebuild count against the reference"""
    d, e = engine(name, mode, use_graph=graph)
    e.step_init()
    eng = d["traj_eng"].reshape(-1, 8)
    ns = int(d["nsteps"][0])
    # plain FP64 tracks CM3D to round-off; mixed within its force tolerance,
    # which a chaotic trajectory amplifies over the steps
    ptol = 1e-9 if mode == _abi.PLAIN_FP64 else 2e-4
    for k in range(ns):
        e.step(1 + k, 1)
        en = e.energies()
        for c, key in enumerate(("poter", "potra", "zke")):
            assert close(en[key], eng[k, c], ptol if c != 1 else 10 * ptol), (k, key)
    # the pressure tensor after the last step, bend virial included (the
    # traceless part that the scalar pressure does not see)
    pt, want = np.array(en["prs_tensor"]), d["ef_prs_tensor"]
    assert np.abs(pt - want).max() <= (ptol if mode == _abi.PLAIN_FP64 else 1e-3) * np.abs(want).max()
    pos = e.positions()
    ref = np.stack([d["final_px"], d["final_py"], d["final_pz"]])
    assert np.abs(pos - ref).max() <= (1e-9 if mode == _abi.PLAIN_FP64 else 1e-3)
    st = e.status()
    if mode == _abi.PLAIN_FP64:
        assert st["rebuilds"] - 1 == int(eng[-1, 7])
    e.close()


def test_errors_are_reported(engine_lib):
    d = golden("lj256")
    e = Engine(System.from_arrays(d), mode=_abi.MIXED)
    with pytest.raises(EngineError, match="get_ngbr"):
        e.force(1)
    with pytest.raises(EngineError):
        e.force_ter(7)
    e.close()
    bad = System.from_arrays(d)
    bad["iperd"] = 2
    with pytest.raises(EngineError, match="iperd"):
        Engine(bad)


@pytest.mark.parametrize("name", ["argon864", "water4096"])
def test_window_kernel_matches_list_kernel(engine_lib, name, monkeypatch):
    """Boxes with >= 3 cells per axis run the staged-window pair kernel; the
    list-gather kernel (CM3D_NB_PAIR_KERNEL=list) evaluates the same pairs
    in another order.  Both stay within the mixed tolerance of CM3D, and of
    each other at FP32 summation-order level."""
    d = golden(name)
    out = {}
    for kind in ("window", "list"):
        # (a lone system with >= 3 cells per axis would otherwise take the
        # compact-window kernel, tests/test_compact.py)
        monkeypatch.setenv("CM3D_NB_PAIR_KERNEL", kind)
        e = Engine(System.from_arrays(d), mode=_abi.MIXED)
        monkeypatch.delenv("CM3D_NB_PAIR_KERNEL")
        e.get_ngbr()
        e.force(1)
        assert e.pair_kernel()[0] == {"window": "window", "list": "gather"}[kind]
        out[kind] = (e.forces(_abi.FXL), e.energies())
        e.close()
    fs = force_scale(d) / float(np.sqrt((d["amass"] ** 2).mean()))
    for kind in ("window", "list"):
        assert rel_rms(out[kind][0], xyz(d, "acc_l"), fs) <= FTOL[_abi.MIXED], kind
    assert rel_rms(out["window"][0], out["list"][0], fs) <= 1e-6
    for k in ("vinter", "velec", "W"):
        assert close(out["window"][1][k], out["list"][1][k], 1e-6), k


def test_status_counts_resets(engine_lib):
    """water216 starts hot: CM3D's RESETPOS fires (reference log: 12 resets in
    20 steps); the engine counts the same events in plain FP64"""
    d, e = engine("water216", _abi.PLAIN_FP64)
    e.step_init()
    e.step(1, 20)
    st = e.status()
    assert st["resets"] == 12
    assert st["rebuilds"] == 14      # step_init's build + 13 during the run
    e.close()


TORS_ENERGIES = ("vtors", "wtors", "vonfo", "vonfo_e", "wonfo", "wonfo_e", "UI", "WI", "vbond", "wbond", "potra")


@pytest.mark.parametrize("mode", MODES, ids=lambda m: MODE_ID[m])
def test_torsion_level(engine_lib, mode):
    """force(3) (ftors + fonfo, rmass, freeze) against CM3D's fxr after
    step_init, and the torsion, 1-4 and cross-bond energies and virials of
    getvireal; these terms are FP64 in both engines"""
    d, e = engine("abutane", mode)
    e.get_ngbr()
    e.force(1)
    e.force(2)
    e.force(3)
    fs = force_scale(d) / float(np.sqrt((d["amass"] ** 2).mean()))
    assert rel_rms(e.forces(_abi.FXR), xyz(d, "acc_r"), fs) <= 1e-12
    en = e.energies()
    for k in TORS_ENERGIES:
        assert close(en[k], float(d[f"e0_{k}"][0]), 1e-12 if k != "wtors" else 1e-9), k
    wit, want = np.array(en["WItensor"]), d["e0_WItensor"]
    assert np.abs(wit - want).max() <= 1e-12 * np.abs(want).max()
    e.close()


def test_torsion_terms_refused_form(engine_lib):
    """the phased cosine form (ind_pot 2), on which CM3D's getvtors stops, is
    refused at create with the reason"""
    d = golden("abutane")
    s = System.from_arrays(d)
    ind = s["tors_ind_pot"].copy()
    ind[0] = 2
    s["tors_ind_pot"] = ind
    with pytest.raises(EngineError, match="ind_pot 2"):
        Engine(s, mode=_abi.MIXED)


@pytest.mark.parametrize("graph", [False, True], ids=["eager", "graph"])
@pytest.mark.parametrize("mode", MODES, ids=lambda m: MODE_ID[m])
def test_nvt_trajectory(engine_lib, mode, graph):
    """CM3D's test/lj NVT deck (one global Nose-Hoover chain of length 3):
    the engine's step with the chain update between the inner half drifts
    (k_nvt_a / k_nvt_chain / k_nvt_c) against CM3D's per-step energies and
    final positions.  The thermostat's kinetic sum is accumulated with
    atomics, so even the plain engine differs from CM3D in summation order."""
    d, e = engine("lj256nvt", mode, use_graph=graph)
    e.step_init()
    eng = d["traj_eng"].reshape(-1, 8)
    ptol = 1e-9 if mode == _abi.PLAIN_FP64 else 2e-4
    for k in range(int(d["nsteps"][0])):
        e.step(1 + k, 1)
        en = e.energies()
        for c, key in enumerate(("poter", "potra", "zke")):
            assert close(en[key], eng[k, c], ptol), (k, key)
    pos = e.positions()
    ref = np.stack([d["final_px"], d["final_py"], d["final_pz"]])
    assert np.abs(pos - ref).max() <= (1e-9 if mode == _abi.PLAIN_FP64 else 1e-3)
    # the chain state read back through cm3d_nb_get_nhc
    eta, veta = e.nhc_state()
    assert eta.shape == veta.shape == (1, 3)
    for got, key in ((eta, "final_nhc_eta"), (veta, "final_nhc_veta")):
        want = d[key]
        assert np.abs(got.ravel() - want).max() <= (1e-8 if mode == _abi.PLAIN_FP64 else 1e-3) * np.abs(want).max()
    e.close()

"""The CPU oracle against CM3D's own outputs (golden fixtures dumped from the
reference by tests/golden/make_golden.py).  The oracle restates CM3D's
algorithms in CM3D's operation order, so every comparison here is exact."""
import hashlib

import numpy as np
import pytest

from conftest import CASES, golden, xyz
from cm3d_b200.system import System
from oracle import Oracle
from tests.golden.make_golden import pair_key

LISTS = (("t", 0), ("s", 1), ("te", 2), ("se", 3))


def make(name):
    d = golden(name)
    return d, Oracle(System.from_arrays(d))


@pytest.mark.parametrize("name", CASES)
def test_pair_lists_bit_exact(name):
    d, o = make(name)
    o.get_ngbr()
    n = int(d["natoms"][0])
    for tag, w in LISTS:
        i, j = o.pair_list(w)
        assert len(i) == int(d[f"npr{tag}"][0]), tag
        if f"list_{tag}_hash" not in d:     # no charges: CM3D builds no te/se list
            assert len(i) == 0
            continue
        h = hashlib.sha256(pair_key(i, j, n).tobytes()).hexdigest()
        assert h == str(d[f"list_{tag}_hash"]), tag
        if f"list_{tag}_key" in d:
            assert np.array_equal(pair_key(i, j, n), d[f"list_{tag}_key"])


@pytest.mark.parametrize("name", CASES)
def test_force_terms_bit_exact(name):
    d, o = make(name)
    o.get_ngbr()
    terms = [("f_lj_l", "f_lj_s", lambda: o.force_ter(1)),
             ("f_el_l", "f_el_s", lambda: o.force_ter_e(1))]
    if int(d["ncharge"][0]) > 0:
        terms += [("f_k", None, o.fk_ewald), ("f_ecorr", None, o.ecorr)]
    for kl, ks, fn in terms:
        o.zero_forces(0)
        o.zero_forces(1)
        fn()
        assert np.array_equal(o.forces(0), xyz(d, kl)), kl
        if ks and ks in d:
            assert np.array_equal(o.forces(1), xyz(d, ks)), ks
    # RESPA short level (force_ter(...,0) / force_ter_e(...,0))
    for key, fn in (("f_lj_short", lambda: o.force_ter(0)), ("f_el_short", lambda: o.force_ter_e(0))):
        if key in d:
            o.zero_forces(1)
            fn()
            assert np.array_equal(o.forces(1), xyz(d, key)), key
    for key, fn in (("f_bond", o.fbond), ("f_bend", o.fbend)):
        o.zero_forces(2)
        fn()
        assert np.array_equal(o.forces(2), xyz(d, key)), key
    # cross bonds (level 2), torsions and 1-4 pairs (level 3)
    for key, fn, blk in (("f_bondx", o.fbondx, 2), ("f_tors", o.ftors, 3), ("f_onfo", o.fonfo, 3)):
        if key in d:
            o.zero_forces(blk)
            fn()
            assert np.array_equal(o.forces(blk), xyz(d, key)), key



TORS_KEYS = ("vtors", "wtors", "vonfo", "vonfo_e", "wonfo", "wonfo_e", "UI", "WI")


@pytest.mark.parametrize("name", CASES)
def test_level1_forces_and_energies_exact(name):
    d, o = make(name)
    o.get_ngbr()
    o.force(1)
    assert np.array_equal(o.forces(0), xyz(d, "acc_l"))
    e = o.energies()
    for k in ("vinter", "vhinter", "velec", "vewald", "winter", "welec", "wewald", "U", "US", "W"):
        assert e[k] == float(d[f"e0_{k}"][0]), k
    for k in ("wintertensor", "welectensor", "wewaldtensor", "Wtensor"):
        assert np.array_equal(np.array(e[k]), d[f"e0_{k}"]), k
    o.force(2)
    e = o.energies()
    for k in ("prsi", "zke", "tiout", "poter", "potra", "wbend", "vbond", "wbond") + TORS_KEYS:
        assert e[k] == float(d[f"e0_{k}"][0]), k
    assert np.array_equal(np.array(e["prs_tensor"]), d["e0_prs_tensor"])
    assert np.array_equal(np.array(e["WItensor"]), d["e0_WItensor"])
    # the torsion level (torsions + 1-4 pairs), with abutane's frozen atoms
    if "acc_r" in d:                   # not stored for the large fixtures
        o.force(3)
        assert np.array_equal(o.forces(3), xyz(d, "acc_r"))


@pytest.mark.parametrize("name", ["lj2", "lj256", "abutane", "argon864", "water216", "binary256", "water4096"])
def test_trajectory_bit_exact(name):
    """CM3D's step() (RESPA, nrefsh with RESETPOS) for the dumped number of
    steps: per-step energies and final state identical"""
    d, o = make(name)
    o.step_init()
    eng = d["traj_eng"].reshape(-1, 8)
    for k in range(int(d["nsteps"][0])):
        o.step(1 + k, 1)
        e = o.energies()
        got = [e["poter"], e["potra"], e["zke"], e["vinter"], e["velec"], e["vewald"], e["prsi"]]
        assert got == list(eng[k, :7]), f"step {k + 1}"
    assert np.array_equal(o.positions(), np.stack([d["final_px"], d["final_py"], d["final_pz"]]))
    assert np.array_equal(o.velocities(), np.stack([d["final_vx"], d["final_vy"], d["final_vz"]]))
    assert o.rebuilds - 1 == int(eng[-1, 7])
    # getvireal(..., 1) + geteng after the last step, the pressure tensor with
    # the bend virial of md_fbend.c (always compiled with PRESSURE) included
    e = o.energies()
    for k in ("vbond", "vbend", "wbond", "wbend", "W", "U", "US", "prsi", "zke", "poter", "potra") + TORS_KEYS:
        assert e[k] == float(d[f"ef_{k}"][0]), k
    for k in ("wintertensor", "welectensor", "wewaldtensor", "Wtensor", "prs_tensor"):
        assert np.array_equal(np.array(e[k]), d[f"ef_{k}"]), k


def test_lj_regression_known_answers():
    """test/lj/lj.out_nve.t t=0 report: npairs s=2334 t=7851,
    <inter> = -1232.123279 K (CM3D's own regression golden)"""
    d, o = make("lj256")
    o.step_init()
    assert len(o.pair_list(0)[0]) == 7851
    assert len(o.pair_list(1)[0]) == 2334
    assert round(o.energies()["vinter"], 6) == -1232.123279


def test_nvt_trajectory_bit_exact():
    """CM3D's test/lj NVT deck (lj.input_ljnvt: one global Nose-Hoover chain
    of length 3, md_therm.new.c:278): the oracle's step with intnhc in the
    inner loop follows CM3D's per-step energies, final positions and
    velocities and the final chain state bit for bit"""
    d, o = make("lj256nvt")
    assert int(d["ntherm"][0]) == 1 and int(d["nchain"][0]) == 3
    o.step_init()
    eng = d["traj_eng"].reshape(-1, 8)
    for k in range(int(d["nsteps"][0])):
        o.step(1 + k, 1)
        e = o.energies()
        got = [e["poter"], e["potra"], e["zke"], e["vinter"], e["velec"], e["vewald"], e["prsi"]]
        assert got == list(eng[k, :7]), f"step {k + 1}"
    assert np.array_equal(o.positions(), np.stack([d["final_px"], d["final_py"], d["final_pz"]]))
    assert np.array_equal(o.velocities(), np.stack([d["final_vx"], d["final_vy"], d["final_vz"]]))
    eta, veta = o.nhc_state()
    assert np.array_equal(eta.ravel(), d["final_nhc_eta"])
    assert np.array_equal(veta.ravel(), d["final_nhc_veta"])

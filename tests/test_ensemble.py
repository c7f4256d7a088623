"""The uneven ensemble (many small LJ and charged-binary boxes, one batch)
against the CPU oracle, box by box.

A slice of the benchmark's ensemble generator (16 boxes, N <= 600) covers
the small-box paths: boxes narrower than three list radii (one or two cells
per axis, no FP32 prefilter, minimum image per pair in the pair kernel) next
to larger ones, charged boxes with Ewald next to LJ-only ones.

Tolerances: pair lists bit-exact; forces relative RMS <= 1e-5; energies
relative <= 1e-5; virials <= 5e-5 (the mixed engine's stated bounds).
"""
import numpy as np
import pytest

from conftest import rel_rms
from cm3d_b200 import _abi
from cm3d_b200.engine import Engine
from tests.golden.make_golden import pair_key

pytestmark = pytest.mark.gpu

ETOL, VTOL, FTOL = 1e-5, 5e-5, 1e-5
VIRIAL_KEYS = {"winter", "welec", "W", "prsi"}


@pytest.fixture(scope="module")
def boxes():
    from cm3d_b200 import configs, setup
    wls = configs.ensemble(16, seed=7, nmax=600)
    return [setup.build_system(w) for w in wls]


def close(a, b, tol, floor=1e-9):
    return abs(a - b) <= tol * max(abs(b), 1e-300) or abs(a - b) <= floor


def test_ensemble_matches_oracle(engine_lib, boxes):
    """lists, forces and energies at positions the oracle reached after 10
    steps from the FCC start (at the lattice itself every force is a
    near-cancelling sum, which no relative error can be measured against)"""
    from oracle import Oracle
    pos = []
    for sm in boxes:
        o = Oracle(sm, nocell_all=1)
        o.step_init()
        o.step(1, 10)
        pos.append(o.positions())
    e = Engine(boxes, mode=_abi.MIXED)
    e.set_positions(np.concatenate(pos, axis=1))
    e.get_ngbr()
    e.force(1)
    e.force(2)
    f = e.forces(_abi.FXL)
    en = e.all_energies()
    lists = {w: e.pair_list(w) for w in (_abi.LIST_T, _abi.LIST_S, _abi.LIST_TE, _abi.LIST_SE)}
    e.close()
    small = 0
    for s, sm in enumerate(boxes):
        a0, n = e.ranges[s]
        o = Oracle(sm, nocell_all=1)
        o.set_positions(pos[s])
        o.get_ngbr()
        for w, (i, j) in lists.items():
            sel = (i >= a0) & (i < a0 + n)
            oi, oj = o.pair_list(w)
            got = np.sort(pair_key(i[sel] - a0, j[sel] - a0, n))
            want = np.sort(pair_key(oi, oj, n))
            assert got.shape == want.shape and (got == want).all(), (s, w)
        o.force(1)
        o.force(2)
        fo = o.forces(_abi.FXL)
        scale = float(np.sqrt((fo * fo).mean()))
        assert rel_rms(f[:, a0:a0 + n], fo, scale) <= FTOL, s
        eo = o.energies()
        for k in ("vinter", "velec", "vewald", "U", "W", "prsi", "zke"):
            tol = VTOL if k in VIRIAL_KEYS else ETOL
            assert close(en[s][k], eo[k], tol, floor=1e-6 * max(1.0, abs(eo["U"]))), (s, k, en[s][k], eo[k])
        L = float(sm["hmat"][0])
        small += L < 3 * (float(np.sqrt(sm["rmaxl_skin2"].max())))
    assert small > 0, "the slice should contain boxes narrower than three list radii"


@pytest.fixture(scope="module")
def mid_boxes():
    """12 boxes of 589-1373 atoms from the ensemble generator: 3 or 4 cells
    per axis, every one in the compact path of a batch"""
    from cm3d_b200 import configs, setup
    return [setup.build_system(w) for w in configs.ensemble(12, seed=11, nmin=500, nmax=1400)]


@pytest.mark.parametrize("slice_row", [("small", 0), ("mid", 32), ("mid", 8)])
def test_ensemble_steps_like_oracle(engine_lib, boxes, mid_boxes, slice_row, monkeypatch):
    """20 steps of a slice as one batch (graph) against each box's oracle
    trajectory: energies within the mixed engine's trajectory bound, same
    list rebuild and RESETPOS counts -- the small boxes with the default
    kernels, and boxes of 3-4 cells per axis on the 32- and the 8-lane
    compact kernel (their lists converted again, on the device, at each
    box's rebuilds)"""
    from oracle import Oracle
    nsteps = 20
    which, row = slice_row
    boxes = boxes if which == "small" else mid_boxes
    if row:
        monkeypatch.setenv("CM3D_NB_CW_ROW", str(row))
    e = Engine(boxes, mode=_abi.MIXED)
    monkeypatch.delenv("CM3D_NB_CW_ROW", raising=False)
    monkeypatch.delenv("CM3D_NB_PAIR_KERNEL", raising=False)
    e.step_init()
    if row:
        assert e.pair_kernel()[0] == ("compact" if row == 32 else "compact8")
    e.step(1, nsteps)
    en = e.all_energies()
    rb, rs = e.system_counts()
    st = e.status()
    e.close()
    assert st["stage_timeouts"] == 0 and st["overflows"] == 0
    for s, sm in enumerate(boxes):
        o = Oracle(sm, nocell_all=1)
        o.step_init()
        o.step(1, nsteps)
        eo = o.energies()
        for k in ("poter", "zke"):
            assert close(en[s][k], eo[k], 2e-4, floor=1e-6 * max(1.0, abs(eo["poter"]))), (s, k)
        assert rb[s] == o.rebuilds and rs[s] == o.resets, (s, rb[s], o.rebuilds, rs[s], o.resets)


@pytest.fixture(scope="module")
def large_boxes():
    """a slice of the headline ensemble itself (configs.ensemble(1024, seed
    2024)): its two largest LJ boxes and two largest charged boxes (3,900-4,100
    atoms) and the two smallest of each kind"""
    from cm3d_b200 import configs, setup
    wls = configs.ensemble(1024, seed=2024)
    nat = np.array([w.natoms for w in wls])
    ch = np.array(["kmax" in w.keywords for w in wls])
    pick = []
    for kind in (False, True):
        idx = np.flatnonzero(ch == kind)
        order = idx[np.argsort(nat[idx])]
        pick += list(order[-2:]) + list(order[:2])
    return [setup.build_system(wls[k]) for k in sorted(pick)]


def test_headline_kernel_on_large_boxes(engine_lib, large_boxes, monkeypatch):
    """the kernel the headline runs -- the batch gather kernel with 4 lanes
    per atom and the compact LJ table (the autotuner's choice on the
    ensemble) -- on boxes up to 4,096 atoms against each box's oracle, at
    positions the oracle reached after 10 steps"""
    from oracle import Oracle
    pos = []
    for sm in large_boxes:
        o = Oracle(sm, nocell_all=1)
        o.step_init()
        o.step(1, 10)
        pos.append(o.positions())
    monkeypatch.setenv("CM3D_NB_PAIR_KERNEL", "list")
    e = Engine(large_boxes, mode=_abi.MIXED, tpa=4)
    monkeypatch.delenv("CM3D_NB_PAIR_KERNEL")
    e.set_positions(np.concatenate(pos, axis=1))
    e.get_ngbr()
    e.force(1)
    assert e.pair_kernel() == ("gather", 4)
    e.force(2)
    f = e.forces(_abi.FXL)
    en = e.all_energies()
    e.close()
    assert max(sm.natoms for sm in large_boxes) >= 3900
    stats = []
    for s, sm in enumerate(large_boxes):
        a0, n = e.ranges[s]
        o = Oracle(sm, nocell_all=1)
        o.set_positions(pos[s])
        o.get_ngbr()
        o.force(1)
        o.force(2)
        fo = o.forces(_abi.FXL)
        scale = float(np.sqrt((fo * fo).mean()))
        assert rel_rms(f[:, a0:a0 + n], fo, scale) <= FTOL, s
        d = np.sqrt(((f[:, a0:a0 + n] - fo) ** 2).sum(axis=0))
        stats.append({"natoms": n, "charged": bool(sm.get("ncharge", 0)), "rel_rms": rel_rms(f[:, a0:a0 + n], fo),
                      "max_atom_over_rms": float(d.max() / np.sqrt((fo * fo).sum(axis=0).mean()))})
        eo = o.energies()
        for k in ("vinter", "velec", "vewald", "U", "W", "prsi", "zke"):
            tol = VTOL if k in VIRIAL_KEYS else ETOL
            assert close(en[s][k], eo[k], tol, floor=1e-6 * max(1.0, abs(eo["U"]))), (s, k, en[s][k], eo[k])
    import json
    import os
    line = json.dumps({"config": "ensemble_large_boxes_gather", "kernel": "gather, 4 lanes per atom", "boxes": stats})
    print("ERRSTAT", line)
    if os.environ.get("CM3D_NB_ERRLOG"):
        with open(os.environ["CM3D_NB_ERRLOG"], "a") as fh:
            fh.write(line + "\n")


@pytest.mark.parametrize("row", [32, 8])
def test_compact_batch_on_large_boxes(engine_lib, large_boxes, row, monkeypatch):
    """the headline's compact pair paths: the batch's boxes with 3 or more
    cells per axis in the compact kernel (grouped by their tables) with 32
    lanes per atom (k_pair_cw) or 8 (k_pair_cs, the small-cell kernel), the
    others in the gather kernel in the same force call -- on the headline
    ensemble's largest and smallest boxes against each box's oracle, at
    positions the oracle reached after 10 steps; with 32 lanes the compact
    boxes' forces are bit-identical to the same box alone (one system,
    compact kernel); a repeat of the force call gives the same bits"""
    from oracle import Oracle
    pos = []
    for sm in large_boxes:
        o = Oracle(sm, nocell_all=1)
        o.step_init()
        o.step(1, 10)
        pos.append(o.positions())
    monkeypatch.setenv("CM3D_NB_CW_ROW", str(row))
    e = Engine(large_boxes, mode=_abi.MIXED, tpa=4)
    monkeypatch.delenv("CM3D_NB_CW_ROW")
    e.set_positions(np.concatenate(pos, axis=1))
    e.get_ngbr()
    e.force(1)
    assert e.pair_kernel()[0] == ("compact" if row == 32 else "compact8")
    f = e.forces(_abi.FXL)
    e.force(1)
    np.testing.assert_array_equal(e.forces(_abi.FXL), f)
    e.force(2)
    en = e.all_energies()
    grids = [e.grid(s)[0] for s in range(len(large_boxes))]
    assert e.status()["stage_timeouts"] == 0
    e.close()
    ncompact = 0
    stats = []
    for s, sm in enumerate(large_boxes):
        a0, n = e.ranges[s]
        if min(grids[s]) >= 3:
            ncompact += 1
        if min(grids[s]) >= 3 and row == 32:
            one = Engine(sm, mode=_abi.MIXED)
            one.set_positions(pos[s])
            one.get_ngbr()
            one.force(1)
            assert one.pair_kernel()[0] == "compact"
            np.testing.assert_array_equal(f[:, a0:a0 + n], one.forces(_abi.FXL))
            one.close()
        o = Oracle(sm, nocell_all=1)
        o.set_positions(pos[s])
        o.get_ngbr()
        o.force(1)
        o.force(2)
        fo = o.forces(_abi.FXL)
        scale = float(np.sqrt((fo * fo).mean()))
        assert rel_rms(f[:, a0:a0 + n], fo, scale) <= FTOL, s
        d = np.sqrt(((f[:, a0:a0 + n] - fo) ** 2).sum(axis=0))
        stats.append({"natoms": n, "charged": bool(sm.get("ncharge", 0)), "cells": grids[s],
                      "kernel": f"compact{row}" if min(grids[s]) >= 3 else "gather",
                      "rel_rms": rel_rms(f[:, a0:a0 + n], fo),
                      "max_atom_over_rms": float(d.max() / np.sqrt((fo * fo).sum(axis=0).mean()))})
        eo = o.energies()
        for k in ("vinter", "velec", "vewald", "U", "W", "prsi", "zke"):
            tol = VTOL if k in VIRIAL_KEYS else ETOL
            assert close(en[s][k], eo[k], tol, floor=1e-6 * max(1.0, abs(eo["U"]))), (s, k, en[s][k], eo[k])
    assert 0 < ncompact < len(large_boxes), "the slice should hold compact and gather boxes"
    import json
    import os
    line = json.dumps({"config": f"ensemble_large_boxes_compact{row}",
                       "kernel": f"compact batch ({row} lanes per atom) + gather, 4 lanes", "boxes": stats})
    print("ERRSTAT", line)
    if os.environ.get("CM3D_NB_ERRLOG"):
        with open(os.environ["CM3D_NB_ERRLOG"], "a") as fh:
            fh.write(line + "\n")

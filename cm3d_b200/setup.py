"""Build a `System` for a generated workload without CM3D: a restatement of
CM3D's set-up for the terms this engine runs.

    read_parmfile       input/md_readparm.c:110-165   atom order, types, masses
                                                      (amu*MCONV), charges (e*sqrt(CCONV))
    search_ter_base     input/md_searchbase.c:108-128 interaction map, cutoffs
    get_ter_parm        input/md_getparm.c:222-366    LJ tables, long-range correction
                                                      (tables built by the C ABI,
                                                      cm3d_nb_lj_table)
    search_bond_base /  input/md_searchbase.c         bond and bend types in order
    search_bend_base                                  of first appearance; bend
                                                      angles degrees -> radians
    set_exclude         energy/control/md_setexclude.c:38-126 with exclude_bonds
                        (md_fbond.c:60-72) and exclude_bends (md_fbend.c:89-122)
    set_charges         energy/control/elec_ngbr.c:36-136 (erfc table via the C ABI)
    set_ecorr           energy/control/elec_ngbr.c:139-218
    ewald_setup         energy/inter/md_ewald.c:48-142

The arrays come out bit-identical to the state CM3D builds from the same
input deck (tests/test_setup.py checks this against dumps of CM3D).
"""
from __future__ import annotations

import math
import re

import numpy as np

from . import engine
from .configs import CCONV, MCONV, TCONV, Workload
from .system import System

# defaults of set_sim_default (input/md_setsimdef.c:33-138)
DEFAULTS = dict(skin=0.5, rheal_res=0.5, ntable=500, nlen=500, ncell_div=7, alp_ewald=0.15,
                kmax=7, shift=0, rcute_max=10.0, rcute_min=1.0, rcute_resp=7.0, nres_lrf=1,
                nres_intra=1, nres_tors=1)

_KEY = re.compile(r"\\(\w+)\{([^}]*)\}")


def _keys(text: str) -> dict:
    return {k: v.strip() for k, v in _KEY.findall(text)}


def _blocks(text: str, meta: str) -> list[dict]:
    out = []
    for m in re.finditer(r"~" + meta + r"\[(.*?)\]", text, flags=re.S):
        out.append(_keys(m.group(1)))
    return out


def build_system(wl: Workload) -> System:
    kw = dict(DEFAULTS)
    kw.update({k: v for k, v in wl.keywords.items()})
    skin = float(kw["skin"])
    rheal = float(kw["rheal_res"])
    ntable = int(kw["ntable"])
    shift = int(kw["shift"])
    # ---------------------------------------------------- atoms and types
    types: list[str] = []
    itype, mass, charge = [], [], []
    bonds, bends = [], []              # (atom1, atom2[, atom3]) global, topology order
    bond_tt, bend_tt = [], []          # type-name tuples
    off = 0
    for _mol, nmol, top in wl.species:
        atoms = sorted(_blocks(top, "atom_def"), key=lambda a: int(a["atom_ind"]))
        napm = len(atoms)
        names = [a["atom_typ"] for a in atoms]
        for a in atoms:
            if a["atom_typ"].lower() not in [t.lower() for t in types]:
                types.append(a["atom_typ"])
        tidx = [[t.lower() for t in types].index(nm.lower()) for nm in names]
        for m in range(nmol):
            for j, a in enumerate(atoms):
                itype.append(tidx[j])
                mass.append(float(a["mass"]) * MCONV)
                charge.append(float(a["charge"]) * math.sqrt(CCONV) * 1.0)
        for b in _blocks(top, "bond_def"):
            i1, i2 = int(b["atom1"]) - 1, int(b["atom2"]) - 1
            for m in range(nmol):
                bonds.append((off + m * napm + i1, off + m * napm + i2))
                bond_tt.append((names[i1], names[i2]))
        for b in _blocks(top, "bend_def"):
            i1, i2, i3 = int(b["atom1"]) - 1, int(b["atom2"]) - 1, int(b["atom3"]) - 1
            for m in range(nmol):
                bends.append((off + m * napm + i1, off + m * napm + i2, off + m * napm + i3))
                bend_tt.append((names[i1], names[i2], names[i3]))
        off += nmol * napm
    n = off
    assert n == wl.natoms
    ntypes = len(types)
    itype = np.array(itype, np.int32)
    qch = np.array(charge)
    amass = np.array(mass)
    # ------------------------------------------------- interactions (LJ)
    parms = {}
    for p in _blocks(wl.database_text(), "inter_parm"):
        a, b = sorted([p["atom1"].lower(), p["atom2"].lower()])
        parms[(a, b)] = p
    mp = np.full((ntypes, ntypes), -1, np.int32)
    cut = {k: [] for k in ("rmaxs_cut2", "rmins_cut2", "rmaxl_cut2", "rminl_cut2", "rmaxs_skin2",
                           "rmaxl_skin2", "dx2tab")}
    vt, dvt, swt, vl, wl_ = [], [], [], [], []
    k = 0
    for i in range(ntypes):
        for j in range(i, ntypes):
            a, b = sorted([types[i].lower(), types[j].lower()])
            p = parms[(a, b)]
            if p["pot_type"].lower() == "null":
                continue
            if p["pot_type"].lower() != "lennard-jones":
                raise ValueError(f"pot_type {p['pot_type']} is not generated by this set-up")
            eps, sig = float(p["eps"]), float(p["sig"])
            rmin = float(p.get("min_dist", 1.0))
            rmax = float(p.get("max_dist", 10.0))
            rres = float(p.get("res_dist", 7.0))
            # get_ter_parm md_getparm.c:222-235
            if rres < rmax:
                rmins, rmaxs, rminl, rmaxl = rmin, rres, rres - rheal, rmax
            else:
                rmins, rmaxs, rmaxl, rminl = rmin, rmax, rmax, rmax + 2. * skin
            v, dv, sw, dx2 = engine.lj_table(eps, sig, rmin, rmax, rres, rheal, skin, ntable, shift)
            vt.append(v)
            dvt.append(dv)
            swt.append(sw)
            # search_ter_base md_searchbase.c:117-123
            cut["rmaxs_cut2"].append(rmaxs * rmaxs)
            cut["rmins_cut2"].append(rmins * rmins)
            cut["rmaxl_cut2"].append(rmaxl * rmaxl)
            cut["rminl_cut2"].append(rminl * rminl)
            cut["rmaxs_skin2"].append((rmaxs + skin) * (rmaxs + skin))
            cut["rmaxl_skin2"].append((rmaxl + skin) * (rmaxl + skin))
            cut["dx2tab"].append(dx2)
            # long-range correction md_getparm.c:259-266 (scaleeps = 1)
            vl.append(4. * eps * math.pow(sig, 6.) * ((1. / 9.) * math.pow(sig, 6.) * math.pow(1. / rmax, 9.)
                                                      - (1. / 3.) * math.pow(1. / rmax, 3.)) * 1.0)
            wl_.append(8. * eps * math.pow(sig, 6.) * (math.pow(1. / rmax, 3.)
                                                       - (2. / 3.) * math.pow(sig, 6.) * math.pow(1. / rmax, 9.)) * 1.0)
            mp[i, j] = mp[j, i] = k
            k += 1
    ninter = k
    vlrc = wlrc = 0.0
    counts = [int((itype == t).sum()) for t in range(ntypes)]
    for i in range(ntypes):
        for j in range(ntypes):
            l = mp[i, j]
            if l != -1:
                vlrc += counts[i] * counts[j] * math.pi * 2. * vl[l]
                wlrc += counts[i] * counts[j] * math.pi * 2. * wl_[l] / 3.
    # --------------------------------------------------- bonds and bends
    bparm = {}
    for p in _blocks(wl.database_text(), "bond_parm"):
        bparm[tuple(sorted([p["atom1"].lower(), p["atom2"].lower()]))] = p
    eparm = {}
    for p in _blocks(wl.database_text(), "bend_parm"):
        a1, a2, a3 = p["atom1"].lower(), p["atom2"].lower(), p["atom3"].lower()
        eparm[(a1, a2, a3)] = p
        eparm[(a3, a2, a1)] = p
    btypes, idxbond = [], []
    for tt in bond_tt:
        key = tuple(sorted([t.lower() for t in tt]))
        if key not in btypes:
            btypes.append(key)
        idxbond.append(btypes.index(key))
    etypes, idxbend = [], []
    for tt in bend_tt:
        key = tuple(t.lower() for t in tt)
        rkey = key[::-1]
        found = next((e for e in etypes if e in (key, rkey)), None)
        if found is None:
            etypes.append(key)
            found = key
        idxbend.append(etypes.index(found))
    eqbond = [float(bparm[t]["eq"]) for t in btypes]
    fkbond = [float(bparm[t]["fk"]) for t in btypes]
    eqbend = [float(eparm[t]["eq"]) * math.pi / 180.0 for t in etypes]
    fkbend = [float(eparm[t]["fk"]) for t in etypes]
    # ----------------------------------------------------------- exclusions
    excl = [set() for _ in range(n)]
    for a, b in bonds:
        excl[min(a, b)].add(max(a, b))
    for a, b, c in bends:
        for u, v in ((a, b), (a, c), (b, c)):
            excl[min(u, v)].add(max(u, v))
    excl_off = np.zeros(n + 1, np.int32)
    excl_idx = []
    for i in range(n):
        s = sorted(excl[i])
        excl_idx += s
        excl_off[i + 1] = excl_off[i] + len(s)
    charged = qch != 0.0
    cexcl_off = np.zeros(n + 1, np.int32)
    cexcl_idx, iecorr, jecorr = [], [], []
    for i in range(n):
        s = [j for j in sorted(excl[i]) if charged[j]] if charged[i] else []
        cexcl_idx += s
        cexcl_off[i + 1] = cexcl_off[i] + len(s)
        for j in s:
            iecorr.append(i)
            jecorr.append(j)
    # --------------------------------------------------- charges / Ewald
    sysm = System()
    ncharge = int(charged.sum())
    if ncharge > 0:
        alpha = float(kw["alp_ewald"])
        rmin_c, rresp, rmax_c = float(kw["rcute_min"]), float(kw["rcute_resp"]), float(kw["rcute_max"])
        c, dc, swe, dx2c = engine.coul_table(alpha, rmin_c, rresp, rmax_c, rheal, skin, ntable, 3, shift)
        sysm["coultab"], sysm["dcoultab"], sysm["switchse"] = c, dc, swe
        sysm["dx2coul"] = dx2c
        sysm["rmins_coul2"] = rmin_c * rmin_c
        sysm["rmaxs_coul2"] = rresp * rresp
        sysm["rminl_coul2"] = ((rresp - rheal) * (rresp - rheal))
        sysm["rmaxl_coul2"] = rmax_c * rmax_c
        sysm["rmaxs_skin2_e"] = ((rresp + skin) * (rresp + skin))
        sysm["rmaxl_skin2_e"] = ((rmax_c + skin) * (rmax_c + skin))
        ka, kb, kc, _kup = engine.ewald_kvectors(int(kw["kmax"]))
        sysm["ka"], sysm["kb"], sysm["kc"] = ka, kb, kc
        sysm["ktot"] = len(ka)
        # ewald_setup md_ewald.c:56-76
        selfe = back = 0.0
        for j in np.flatnonzero(charged):
            selfe += qch[j] * qch[j]
            back += qch[j]
        sysm["kappa"] = alpha
        sysm["falp2"] = 1. / (4. * (alpha * alpha))
        sysm["ewald_self"] = selfe * (-alpha / math.sqrt(math.pi))
        sysm["ewald_bkg"] = -.5 * back * back * math.pi / (alpha * alpha)
    else:
        sysm["ktot"] = 0
    # ----------------------------------------------------------- the rest
    L = wl.box
    sysm["natoms"] = n
    sysm["iperd"] = int(kw.get("iperd", 3))
    sysm["nres_lrf"] = int(kw["nres_lrf"])
    sysm["nres_intra"] = int(kw["nres_intra"])
    sysm["nres_tors"] = int(kw["nres_tors"])
    sysm["ndof"] = max(3 * n - 3, 1)
    sysm["dt"] = float(kw["dt"]) * TCONV
    sysm["temp"] = float(kw.get("t_ext", wl.temp))
    sysm["vlrc"] = vlrc
    sysm["wlrc"] = wlrc
    sysm["hmat"] = np.array([L, 0, 0, 0, L, 0, 0, 0, L], float)
    p, v = wl.pos, wl.vel
    sysm["px"], sysm["py"], sysm["pz"] = p[:, 0], p[:, 1], p[:, 2]
    sysm["vx"], sysm["vy"], sysm["vz"] = v[:, 0], v[:, 1], v[:, 2]
    sysm["amass"] = amass
    sysm["qch"] = qch
    sysm["itype"] = itype
    sysm["ntypes"] = ntypes
    sysm["map"] = mp.ravel()
    sysm["ninter"] = ninter
    sysm["ntable"] = ntable
    if ninter:
        sysm["vtab"] = np.concatenate(vt)
        sysm["dvtab"] = np.concatenate(dvt)
        sysm["switchs"] = np.concatenate(swt)
        for key, vals in cut.items():
            sysm[key] = np.array(vals)
    sysm["skin"] = skin
    sysm["rheal"] = rheal
    sysm["excl_off"], sysm["excl_idx"] = excl_off, np.array(excl_idx, np.int32)
    sysm["cexcl_off"], sysm["cexcl_idx"] = cexcl_off, np.array(cexcl_idx, np.int32)
    sysm["necorr"] = len(iecorr)
    sysm["iecorr"], sysm["jecorr"] = np.array(iecorr, np.int32), np.array(jecorr, np.int32)
    sysm["nbonds"] = len(bonds)
    if bonds:
        sysm["ibond"] = [b[0] for b in bonds]
        sysm["jbond"] = [b[1] for b in bonds]
        sysm["idxbond"] = idxbond
        sysm["itypbond"] = [0] * len(btypes)
        sysm["eqbond"], sysm["fkbond"] = eqbond, fkbond
    sysm["nbends"] = len(bends)
    if bends:
        sysm["ibend"] = [b[0] for b in bends]
        sysm["jbend"] = [b[1] for b in bends]
        sysm["kbend"] = [b[2] for b in bends]
        sysm["idxbend"] = idxbend
        sysm["itypbend"] = [0] * len(etypes)
        sysm["eqbend"], sysm["fkbend"] = eqbend, fkbend
    sysm["ntors"] = 0
    sysm["n14"] = 0
    sysm["nbondx"] = 0
    sysm["nfreeze"] = 0
    sysm["iensemble"] = 0            # NVE: no thermostat chains
    sysm["ntherm"] = 0
    sysm["nchain"] = 0
    sysm["ncells"] = int(kw["ncell_div"])
    sysm["nocell_all"] = 1
    sysm["nlen"] = int(kw["nlen"])
    return sysm

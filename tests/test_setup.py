"""Host-side set-up and C-ABI checks that need no GPU: the library loads and
exports every entry point of include/cm3d_nb.h, the table/k-vector builders
reproduce CM3D's tables bit for bit, and the standalone set-up of a generated
workload equals the state CM3D itself builds from the same input deck."""
import os
import re

import numpy as np
import pytest

from conftest import ROOT, golden
from cm3d_b200 import configs
from cm3d_b200.system import System

HEADER = os.path.join(ROOT, "include", "cm3d_nb.h")


def header_functions():
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(cm3d_nb_\w+)\s*\(", txt)))


def test_library_exports_every_header_symbol(engine_lib):
    names = header_functions()
    assert len(names) >= 35
    for name in names:
        assert hasattr(engine_lib, name), name


def test_oracle_has_no_product_dependency():
    """the product package never imports the checker"""
    pkg = os.path.join(ROOT, "cm3d_b200")
    for root, _d, files in os.walk(pkg):
        for f in files:
            if f.endswith((".py", ".cu", ".cuh", ".c", ".cpp", ".h")):
                src = open(os.path.join(root, f)).read()
                assert "import oracle" not in src and "from oracle" not in src, f
                assert "cm3d_oracle" not in src, f


@pytest.mark.parametrize("name", ["lj256", "argon864", "water216", "binary256", "water4096"])
def test_lj_tables_bit_exact(engine_lib, name):
    from cm3d_b200 import engine
    d = golden(name)
    if name == "lj256":
        # test/lj/data_base: eps 1 sig 1 min .8 max 2.5 res 1.7; skin .1 rheal .1
        params = [(1.0, 1.0, 0.8, 2.5, 1.7, 0)]
    elif name == "argon864":
        a = configs.ARGON
        rc = 2.5 * a["sig"]
        params = [(a["eps"], a["sig"], 0.55 * a["sig"], rc, rc, 1)]
    elif name == "binary256":
        wl = configs.charged_binary(natoms=256)
        rc = wl.keywords["rcute_max"]
        a = configs.ARGON
        params = [(a["eps"], a["sig"], 0.55 * a["sig"], rc, rc, 1)] * 3
    else:
        w = configs.WATER
        rc = float(np.sqrt(d["rmaxl_cut2"][0]))
        params = [(w["eps_oo"], w["sig_oo"], 1.8, rc, rc, 0)]
    nt = int(d["ntable"][0])
    for k, (eps, sig, rmin, rmax, rres, shift) in enumerate(params):
        v, dv, sw, dx2 = engine.lj_table(eps, sig, rmin, rmax, rres, float(d["rheal"][0]),
                                         float(d["skin"][0]), nt, shift)
        sl = slice(k * nt, (k + 1) * nt)
        assert np.array_equal(v, d["vtab"][sl])
        assert np.array_equal(dv, d["dvtab"][sl])
        assert np.array_equal(sw, d["switchs"][sl])
        assert dx2 == d["dx2tab"][k]


@pytest.mark.parametrize("name,kmax", [("water216", 7), ("water4096", 7), ("binary256", 5), ("abutane", 15)])
def test_coul_table_and_kvectors_bit_exact(engine_lib, name, kmax):
    from cm3d_b200 import engine
    d = golden(name)
    ka, kb, kc, kup = engine.ewald_kvectors(kmax)
    assert np.array_equal(ka, d["ka"]) and np.array_equal(kb, d["kb"]) and np.array_equal(kc, d["kc"])
    if name == "abutane":
        return
    rmin = float(np.sqrt(d["rmins_coul2"][0]))
    rmax = float(np.sqrt(d["rmaxl_coul2"][0]))
    rresp = float(np.sqrt(d["rmaxs_coul2"][0]))
    alpha = float(d["kappa"][0])
    shift = 1 if name == "binary256" else 0          # that deck sets \shift{1}
    c, dc, sw, dx2 = engine.coul_table(alpha, rmin, rresp, rmax, float(d["rheal"][0]),
                                       float(d["skin"][0]), int(d["ntable"][0]), 3, shift)
    assert np.array_equal(c, d["coultab"]) and np.array_equal(dc, d["dcoultab"])
    assert np.array_equal(sw, d["switchse"]) and dx2 == d["dx2coul"][0]


def test_kvector_counts():
    """ktot for kmax 5/7/12/15/21 (CM3D's spherical half-space set)"""
    from cm3d_b200 import engine
    assert [len(engine.ewald_kvectors(k)[0]) for k in (5, 7, 12, 15, 21)] == [257, 709, 3576, 7073, 19455]


CHARGE_ONLY = {"coultab", "dcoultab", "switchse", "dx2coul", "rmins_coul2", "rmaxs_coul2",
               "rminl_coul2", "rmaxl_coul2", "rmaxs_skin2_e", "rmaxl_skin2_e", "kappa", "falp2",
               "ewald_self", "ewald_bkg", "iecorr", "jecorr"}


@pytest.mark.parametrize("name,make", [
    ("argon864", lambda: configs.argon_fcc(ntime=20)),
    ("water216", lambda: configs.water_box(ngrid=6, ntime=20)),
    ("binary256", lambda: configs.charged_binary(natoms=256, ntime=10)),
])
def test_standalone_setup_matches_cm3d(engine_lib, name, make):
    from cm3d_b200.setup import build_system
    s = build_system(make())
    g = System.from_arrays(golden(name))
    charged = int((g["qch"] != 0).sum()) > 0
    for k in set(g.a) | set(s.a):
        if (not charged or k in ("iecorr", "jecorr")) and k in CHARGE_ONLY:
            if k not in g.a or k not in s.a:
                continue
        assert k in s.a and k in g.a, k
        assert np.array_equal(s.a[k], g.a[k]), k
    for k in set(g.s) | set(s.s):
        if not charged and k in CHARGE_ONLY:
            continue
        assert s.s.get(k) == g.s.get(k), k


def test_workloads_are_seeded_and_sized():
    a = configs.argon_fcc()
    assert a.natoms == 864 and abs(a.box - 34.3142) < 1e-3
    w = configs.water_box(ngrid=4, seed=3)
    w2 = configs.water_box(ngrid=4, seed=3)
    assert np.array_equal(w.pos, w2.pos) and np.array_equal(w.vel, w2.vel)
    assert abs(configs.water_box(ngrid=2).box - 2 * 49.66 / 16) < 1e-12
    # MB velocities: zero momentum, exact temperature (ndof = 3N - 3)
    m = a.mass_amu * configs.MCONV
    assert np.allclose((m[:, None] * a.vel).sum(0), 0, atol=1e-9)
    t = float((m[:, None] * a.vel ** 2).sum()) / (3 * a.natoms - 3)
    assert abs(t - 120.0) < 1e-9


def test_system_description_carries_the_torsion_level():
    """CM3D's abutane state (dumped by the reference) packed into the C ABI's
    cm3d_nb_system: torsions, 1-4 pairs, cross bonds and frozen atoms with
    the counts and table sizes CM3D reports, every array present"""
    from cm3d_b200 import _abi
    d = golden("abutane")
    s = System.from_arrays(d)
    desc = s.desc()
    assert (desc.ntors, desc.n14, desc.nbondx, desc.nfreeze) == (27, 27, 3, 2)
    assert desc.ntors_types == int(d["tors_ind_pot"].size)
    # every torsion type of the deck is a cosine power series (form 1)
    assert desc.ntors_harm == 0 and desc.ntors_series == int(d["vphi"].size) // _abi.MAXPOWER_TORS
    assert desc.n14_types == int(d["n14types"][0]) and desc.n14table == int(d["n14table"][0])
    assert desc.nbondx_types == int(d["eq1bondx"].size)
    assert (desc.scale_onefour, desc.scale_onefour_e) == (float(d["scale_onefour"][0]),
                                                         float(d["scale_onefour_e"][0]))
    for name in ("itors", "jtors", "ktors", "ltors", "idxtors", "tors_ind_pot", "tors_ind_pot_num", "vphi",
                 "i14", "j14", "i14dx", "r14min2", "r14max2", "dx214tab", "v14tab", "dv14tab", "ibondx",
                 "jbondx", "kbondx", "idxbondx", "eq1bondx", "eq2bondx", "fkbondx", "ifreeze"):
        assert bool(getattr(desc, name)), name
    assert list(desc.ifreeze[:2]) == list(d["ifreeze"])
    # a system without them (generated argon) leaves the fields empty
    from cm3d_b200.setup import build_system
    a = build_system(configs.argon_fcc(ncell=3, ntime=2)).desc()
    assert (a.ntors, a.n14, a.nbondx, a.nfreeze) == (0, 0, 0, 0)
    assert not bool(a.itors) and not bool(a.ifreeze)


def test_engine_refuses_barostats_on_the_host(engine_lib):
    """the engine integrates NVE or NVT: an NPT system (iensemble 2), or NVT
    without its chain state, is refused by cm3d_nb_create before any device
    work, with the reason"""
    from cm3d_b200 import _abi
    from cm3d_b200.engine import Engine, EngineError
    s = System.from_arrays(golden("lj256nvt"))
    assert s.desc().ntherm == 1 and s.desc().iensemble == 1
    s["iensemble"] = 2
    with pytest.raises(EngineError, match="without barostats"):
        Engine(s, mode=_abi.MIXED)
    s = System.from_arrays(golden("lj256nvt"))
    del s.a["nhc_veta"]
    s._desc = None
    with pytest.raises(EngineError, match="without barostats"):
        Engine(s, mode=_abi.MIXED)

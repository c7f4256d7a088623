"""Host-side description of one CM3D system for the engine.

`System` holds, as numpy arrays, exactly the fields of CM3D's SIMPARMS /
COORDS / INTER / COUL / BONDS / BENDS / TORS / ONFO / BONDXS structs that the
nonbonded path and the intramolecular RESPA levels read
(include/md_typedef.h:59-268), under CM3D's names.
`System.desc()` packs them into the C ABI struct `cm3d_nb_system`
(include/cm3d_nb.h) without copying.

A System is built either from a dict of arrays under those names (a dump of
CM3D's own state, see tests/golden) or by `cm3d_b200.setup.build_system`,
which restates CM3D's set-up (tables, exclusions, k-vectors) for a generated
workload.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _abi

_F64 = ("hmat", "px", "py", "pz", "vx", "vy", "vz", "amass", "qch", "vtab", "dvtab",
        "switchs", "rmaxs_cut2", "rmins_cut2", "rmaxl_cut2", "rminl_cut2",
        "rmaxs_skin2", "rmaxl_skin2", "dx2tab", "coultab", "dcoultab", "switchse",
        "eqbond", "fkbond", "eqbend", "fkbend", "eqtors", "fktors", "vphi", "r14min2",
        "r14max2", "dx214tab", "v14tab", "dv14tab", "eq1bondx", "eq2bondx", "fkbondx", "mnh", "gkt", "nhc_eta", "nhc_veta")
_I32 = ("itype", "map", "excl_off", "excl_idx", "cexcl_off", "cexcl_idx", "ka", "kb",
        "kc", "iecorr", "jecorr", "ibond", "jbond", "idxbond", "itypbond", "ibend",
        "jbend", "kbend", "idxbend", "itypbend", "itors", "jtors", "ktors", "ltors",
        "idxtors", "tors_ind_pot", "tors_ind_pot_num", "i14", "j14", "i14dx", "ibondx",
        "jbondx", "kbondx", "idxbondx", "ifreeze", "ithm")
_SCALARS_F = ("dt", "vlrc", "wlrc", "skin", "rheal", "dx2coul", "rmins_coul2",
              "rmaxs_coul2", "rminl_coul2", "rmaxl_coul2", "rmaxs_skin2_e",
              "rmaxl_skin2_e", "kappa", "falp2", "ewald_self", "ewald_bkg", "temp",
              "scale_onefour", "scale_onefour_e")
_SCALARS_I = ("natoms", "iperd", "nres_lrf", "nres_intra", "nres_tors", "ndof",
              "ntypes", "ninter", "ntable", "ktot", "necorr", "nbonds", "nbends",
              "ntors", "n14", "nbondx", "ncells", "nocell_all", "nlen", "n14table", "n14types",
              "nfreeze", "iensemble", "ntherm", "nchain")


class System:
    """Arrays and scalars of one system, under CM3D's field names."""

    def __init__(self, **kw):
        self.a: dict[str, np.ndarray] = {}
        self.s: dict[str, float | int] = {}
        for k, v in kw.items():
            self[k] = v
        self._desc = None

    # ----------------------------------------------------------- access
    def __setitem__(self, key: str, value) -> None:
        if key in _F64:
            self.a[key] = np.ascontiguousarray(value, dtype=np.float64).ravel()
        elif key in _I32:
            self.a[key] = np.ascontiguousarray(value, dtype=np.int32).ravel()
        elif key in _SCALARS_F:
            self.s[key] = float(np.asarray(value).ravel()[0])
        elif key in _SCALARS_I:
            self.s[key] = int(np.asarray(value).ravel()[0])
        else:
            raise KeyError(key)
        self._desc = None

    def __getitem__(self, key: str):
        if key in self.a:
            return self.a[key]
        return self.s[key]

    def get(self, key: str, default=None):
        try:
            return self[key]
        except KeyError:
            return default

    @property
    def natoms(self) -> int:
        return int(self.s["natoms"])

    @classmethod
    def from_arrays(cls, d: dict) -> "System":
        """Build from a mapping that uses CM3D's field names (e.g. a golden
        fixture).  Unknown keys are ignored."""
        sysm = cls()
        for k in _F64 + _I32 + _SCALARS_F + _SCALARS_I:
            if k in d:
                sysm[k] = d[k]
        for k in ("ntors", "n14", "nbondx", "nbonds", "nbends", "necorr", "ktot"):
            sysm.s.setdefault(k, 0)
        n = sysm.natoms
        for k in ("excl_off", "cexcl_off"):
            if k not in sysm.a:
                sysm.a[k] = np.zeros(n + 1, np.int32)
        for k in ("excl_idx", "cexcl_idx"):
            if k not in sysm.a:
                sysm.a[k] = np.zeros(0, np.int32)
        return sysm

    def copy(self) -> "System":
        out = System()
        out.a = {k: v.copy() for k, v in self.a.items()}
        out.s = dict(self.s)
        return out

    # ------------------------------------------------------------- C ABI
    def _ptr(self, key: str, ctype):
        arr = self.a.get(key)
        if arr is None or arr.size == 0:
            return C.cast(None, C.POINTER(ctype))
        return arr.ctypes.data_as(C.POINTER(ctype))

    def desc(self) -> _abi.SystemDesc:
        """The cm3d_nb_system view of this System (pointers into self.a)."""
        if self._desc is not None:
            return self._desc
        d = _abi.SystemDesc()
        s, a = self.s, self.a
        d.natoms = s["natoms"]
        d.iperd = s.get("iperd", 3)
        d.nres_lrf = s.get("nres_lrf", 1)
        d.nres_intra = s.get("nres_intra", 1)
        d.nres_tors = s.get("nres_tors", 1)
        d.ndof = s.get("ndof", max(3 * s["natoms"] - 3, 1))
        d.dt = s.get("dt", 0.0)
        d.vlrc = s.get("vlrc", 0.0)
        d.wlrc = s.get("wlrc", 0.0)
        for i in range(9):
            d.hmat[i] = a["hmat"][i]
        for k in ("px", "py", "pz", "vx", "vy", "vz", "amass", "qch", "vtab", "dvtab",
                  "switchs", "rmaxs_cut2", "rmins_cut2", "rmaxl_cut2", "rminl_cut2",
                  "rmaxs_skin2", "rmaxl_skin2", "dx2tab", "coultab", "dcoultab",
                  "switchse", "eqbond", "fkbond", "eqbend", "fkbend", "eqtors", "fktors",
                  "vphi", "r14min2", "r14max2", "dx214tab", "v14tab", "dv14tab", "eq1bondx",
                  "eq2bondx", "fkbondx", "mnh", "gkt", "nhc_eta", "nhc_veta"):
            setattr(d, k, self._ptr(k, C.c_double))
        for k in ("itype", "map", "excl_off", "excl_idx", "cexcl_off", "cexcl_idx",
                  "ka", "kb", "kc", "iecorr", "jecorr", "ibond", "jbond", "idxbond",
                  "itypbond", "ibend", "jbend", "kbend", "idxbend", "itypbend", "itors",
                  "jtors", "ktors", "ltors", "idxtors", "tors_ind_pot", "tors_ind_pot_num",
                  "i14", "j14", "i14dx", "ibondx", "jbondx", "kbondx", "idxbondx", "ifreeze",
                  "ithm"):
            setattr(d, k, self._ptr(k, C.c_int))
        d.ntypes = s["ntypes"]
        d.ninter = s["ninter"]
        d.ntable = s["ntable"]
        d.skin_ter = s["skin"]
        d.rheal = s.get("rheal", 0.5)
        for k in ("dx2coul", "rmins_coul2", "rmaxs_coul2", "rminl_coul2", "rmaxl_coul2",
                  "rmaxs_skin2_e", "rmaxl_skin2_e", "kappa", "falp2", "ewald_self",
                  "ewald_bkg"):
            setattr(d, k, s.get(k, 0.0))
        d.ktot = s.get("ktot", 0)
        d.necorr = s.get("necorr", 0)
        d.nbonds = s.get("nbonds", 0)
        d.nbond_types = int(a["eqbond"].size) if "eqbond" in a else 0
        d.nbends = s.get("nbends", 0)
        d.nbend_types = int(a["eqbend"].size) if "eqbend" in a else 0
        d.ntors = s.get("ntors", 0)
        d.n14 = s.get("n14", 0)
        d.nbondx = s.get("nbondx", 0)
        # torsions, 1-4 pairs and cross bonds (TORS / ONFO / BONDXS)
        d.ntors_types = int(a["tors_ind_pot"].size) if "tors_ind_pot" in a else 0
        d.ntors_harm = int(a["eqtors"].size) if "eqtors" in a else 0
        d.ntors_series = int(a["vphi"].size) // _abi.MAXPOWER_TORS if "vphi" in a else 0
        d.n14_types = int(a["r14min2"].size) if "r14min2" in a else 0
        d.n14table = s.get("n14table", 0)
        d.scale_onefour = s.get("scale_onefour", 1.0)
        d.scale_onefour_e = s.get("scale_onefour_e", 1.0)
        d.nbondx_types = int(a["eq1bondx"].size) if "eq1bondx" in a else 0
        d.nfreeze = s.get("nfreeze", 0)
        d.iensemble = s.get("iensemble", 0)
        d.ntherm = s.get("ntherm", 0)
        d.nchain = s.get("nchain", 0)
        self._desc = d
        return d

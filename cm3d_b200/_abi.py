"""ctypes mirror of include/cm3d_nb.h (structs and constants)."""
from __future__ import annotations

import ctypes as C

OK = 0
ERR_ARG, ERR_CUDA, ERR_NOMEM, ERR_STATE, ERR_OVERFLOW, ERR_NODEV = -1, -2, -3, -4, -5, -6

PLAIN_FP64, MIXED = 0, 1
FXL, FXS, FXA, FXR = 0, 1, 2, 3
MAXPOWER_TORS = 7
LIST_T, LIST_S, LIST_TE, LIST_SE = 0, 1, 2, 3

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


class SystemDesc(C.Structure):
    _fields_ = [
        ("natoms", C.c_int), ("iperd", C.c_int), ("nres_lrf", C.c_int),
        ("nres_intra", C.c_int), ("nres_tors", C.c_int), ("ndof", C.c_int),
        ("dt", C.c_double), ("vlrc", C.c_double), ("wlrc", C.c_double),
        ("hmat", C.c_double * 9),
        ("px", _dp), ("py", _dp), ("pz", _dp), ("vx", _dp), ("vy", _dp), ("vz", _dp),
        ("amass", _dp), ("qch", _dp),
        ("ntypes", C.c_int), ("itype", _ip), ("map", _ip),
        ("ninter", C.c_int), ("ntable", C.c_int),
        ("vtab", _dp), ("dvtab", _dp), ("switchs", _dp),
        ("rmaxs_cut2", _dp), ("rmins_cut2", _dp), ("rmaxl_cut2", _dp), ("rminl_cut2", _dp),
        ("rmaxs_skin2", _dp), ("rmaxl_skin2", _dp), ("dx2tab", _dp),
        ("skin_ter", C.c_double), ("rheal", C.c_double),
        ("coultab", _dp), ("dcoultab", _dp), ("switchse", _dp),
        ("dx2coul", C.c_double), ("rmins_coul2", C.c_double), ("rmaxs_coul2", C.c_double),
        ("rminl_coul2", C.c_double), ("rmaxl_coul2", C.c_double),
        ("rmaxs_skin2_e", C.c_double), ("rmaxl_skin2_e", C.c_double),
        ("excl_off", _ip), ("excl_idx", _ip),
        ("cexcl_off", _ip), ("cexcl_idx", _ip),
        ("ktot", C.c_int), ("ka", _ip), ("kb", _ip), ("kc", _ip),
        ("kappa", C.c_double), ("falp2", C.c_double), ("ewald_self", C.c_double),
        ("ewald_bkg", C.c_double),
        ("necorr", C.c_int), ("iecorr", _ip), ("jecorr", _ip),
        ("nbonds", C.c_int), ("nbond_types", C.c_int),
        ("ibond", _ip), ("jbond", _ip), ("idxbond", _ip), ("itypbond", _ip),
        ("eqbond", _dp), ("fkbond", _dp),
        ("nbends", C.c_int), ("nbend_types", C.c_int),
        ("ibend", _ip), ("jbend", _ip), ("kbend", _ip), ("idxbend", _ip), ("itypbend", _ip),
        ("eqbend", _dp), ("fkbend", _dp),
        ("ntors", C.c_int), ("n14", C.c_int), ("nbondx", C.c_int),
        ("ntors_types", C.c_int),
        ("itors", _ip), ("jtors", _ip), ("ktors", _ip), ("ltors", _ip), ("idxtors", _ip),
        ("tors_ind_pot", _ip), ("tors_ind_pot_num", _ip),
        ("ntors_harm", C.c_int), ("eqtors", _dp), ("fktors", _dp),
        ("ntors_series", C.c_int), ("vphi", _dp),
        ("n14_types", C.c_int), ("n14table", C.c_int),
        ("i14", _ip), ("j14", _ip), ("i14dx", _ip),
        ("r14min2", _dp), ("r14max2", _dp), ("dx214tab", _dp),
        ("v14tab", _dp), ("dv14tab", _dp),
        ("scale_onefour", C.c_double), ("scale_onefour_e", C.c_double),
        ("nbondx_types", C.c_int),
        ("ibondx", _ip), ("jbondx", _ip), ("kbondx", _ip), ("idxbondx", _ip),
        ("eq1bondx", _dp), ("eq2bondx", _dp), ("fkbondx", _dp),
        ("nfreeze", C.c_int), ("ifreeze", _ip),
        ("iensemble", C.c_int), ("ntherm", C.c_int), ("nchain", C.c_int), ("ithm", _ip),
        ("mnh", _dp), ("gkt", _dp), ("nhc_eta", _dp), ("nhc_veta", _dp),
    ]


class Options(C.Structure):
    _fields_ = [("device", C.c_int), ("mode", C.c_int), ("need_short", C.c_int),
                ("tpa", C.c_int), ("use_graph", C.c_int), ("cell_scale", C.c_double)]


class Energies(C.Structure):
    _fields_ = [
        ("vinter", C.c_double), ("vhinter", C.c_double), ("winter", C.c_double),
        ("wintertensor", C.c_double * 9),
        ("velec", C.c_double), ("welec", C.c_double), ("welectensor", C.c_double * 9),
        ("vewald", C.c_double), ("wewald", C.c_double), ("wewaldtensor", C.c_double * 9),
        ("vbond", C.c_double), ("vbend", C.c_double), ("wbond", C.c_double),
        ("wbend", C.c_double),
        ("US", C.c_double), ("U", C.c_double), ("W", C.c_double), ("Wtensor", C.c_double * 9),
        ("zke", C.c_double), ("p2m_tensor", C.c_double * 9),
        ("prsi", C.c_double), ("prs_tensor", C.c_double * 9), ("tiout", C.c_double),
        ("poter", C.c_double), ("poth", C.c_double), ("potra", C.c_double),
        ("vtors", C.c_double), ("wtors", C.c_double), ("vonfo", C.c_double),
        ("vonfo_e", C.c_double), ("wonfo", C.c_double), ("wonfo_e", C.c_double),
        ("UI", C.c_double), ("WI", C.c_double), ("WItensor", C.c_double * 9),
    ]

    @classmethod
    def numpy_dtype(cls):
        """numpy structured dtype with the struct's layout (tensors as (9,))"""
        import numpy as np
        return np.dtype([(name, np.float64, (9,)) if issubclass(typ, C.Array) else (name, np.float64)
                         for name, typ in cls._fields_])

    def as_dict(self) -> dict:
        out = {}
        for name, typ in self._fields_:
            v = getattr(self, name)
            out[name] = list(v) if isinstance(v, C.Array) else float(v)
        return out


class Status(C.Structure):
    _fields_ = [("table_underflow", C.c_longlong), ("rebuilds", C.c_longlong),
                ("resets", C.c_longlong), ("overflows", C.c_longlong),
                ("nonfinite", C.c_int), ("last_istep", C.c_int), ("stage_timeouts", C.c_int)]

"""CPU oracle for the CM3D nonbonded path (TEST INFRASTRUCTURE ONLY).

ctypes wrapper over oracle/libcm3d_oracle.so, the C restatement of CM3D's
algorithms (oracle/cm3d_oracle.c).  Only tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg may use it; the product never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from cm3d_b200 import _abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "libcm3d_oracle.so")
REF_DIR = os.path.join(HERE, "_ref")

_lib = None


def build(force: bool = False) -> None:
    if force or not os.path.exists(LIB):
        subprocess.run(["make", "-C", HERE, "libcm3d_oracle.so"], check=True,
                       stdout=subprocess.DEVNULL)


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(LIB)
        vp = C.c_void_p
        dp = C.POINTER(C.c_double)
        ip = C.POINTER(C.c_int)
        L.orc_create.restype = vp
        L.orc_create.argtypes = [C.POINTER(_abi.SystemDesc), C.c_int, C.c_int, C.c_int]
        for name in ("orc_destroy", "orc_get_ngbr", "orc_fk_ewald", "orc_ecorr",
                     "orc_fbond", "orc_fbend", "orc_fbondx", "orc_ftors", "orc_fonfo",
                     "orc_step_init"):
            getattr(L, name).argtypes = [vp]
            getattr(L, name).restype = None
        for name in ("orc_force", "orc_force_ter", "orc_force_ter_e", "orc_rmass",
                     "orc_zero_forces"):
            getattr(L, name).argtypes = [vp, C.c_int]
            getattr(L, name).restype = None
        for name in ("orc_set_positions", "orc_get_positions", "orc_set_velocities",
                     "orc_get_velocities"):
            getattr(L, name).argtypes = [vp, dp, dp, dp]
            getattr(L, name).restype = None
        L.orc_get_forces.argtypes = [vp, C.c_int, dp, dp, dp]
        L.orc_get_forces.restype = None
        L.orc_list_count.argtypes = [vp, C.c_int]
        L.orc_list_count.restype = C.c_longlong
        L.orc_get_list.argtypes = [vp, C.c_int, ip, ip]
        L.orc_get_list.restype = None
        L.orc_get_energies.argtypes = [vp, C.POINTER(_abi.Energies)]
        L.orc_get_energies.restype = None
        L.orc_step.argtypes = [vp, C.c_int, C.c_int]
        L.orc_step.restype = None
        L.orc_get_nhc.argtypes = [vp, dp, dp]
        L.orc_get_nhc.restype = None
        for name in ("orc_rebuilds", "orc_resets", "orc_underflows"):
            getattr(L, name).argtypes = [vp]
            getattr(L, name).restype = C.c_longlong
        _lib = L
    return _lib


def _p(a: np.ndarray, t=C.c_double):
    return a.ctypes.data_as(C.POINTER(t))


class Oracle:
    """CM3D's nonbonded path on the CPU, in CM3D's own operation order."""

    def __init__(self, system, ncells: int | None = None, nocell_all: int | None = None,
                 nlen: int | None = None):
        self.sys = system
        self.n = system.natoms
        ncells = ncells if ncells is not None else int(system.get("ncells", 7))
        nocell_all = nocell_all if nocell_all is not None else int(system.get("nocell_all", 1))
        nlen = nlen if nlen is not None else int(system.get("nlen", 500))
        self._h = lib().orc_create(C.byref(system.desc()), ncells, nocell_all, nlen)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            lib().orc_destroy(h)
            self._h = None

    def _xyz(self, fn, *lead):
        x, y, z = (np.empty(self.n) for _ in range(3))
        fn(self._h, *lead, _p(x), _p(y), _p(z))
        return np.stack([x, y, z])

    def positions(self):
        return self._xyz(lib().orc_get_positions)

    def velocities(self):
        return self._xyz(lib().orc_get_velocities)

    def set_positions(self, p):
        p = np.ascontiguousarray(p, dtype=np.float64)
        lib().orc_set_positions(self._h, _p(p[0].copy()), _p(p[1].copy()), _p(p[2].copy()))

    def set_velocities(self, v):
        v = np.ascontiguousarray(v, dtype=np.float64)
        lib().orc_set_velocities(self._h, _p(v[0].copy()), _p(v[1].copy()), _p(v[2].copy()))

    def forces(self, which: int = _abi.FXL):
        return self._xyz(lib().orc_get_forces, which)

    def zero_forces(self, which: int):
        lib().orc_zero_forces(self._h, which)

    def get_ngbr(self):
        lib().orc_get_ngbr(self._h)

    def pair_list(self, which: int):
        n = lib().orc_list_count(self._h, which)
        i = np.empty(n, np.int32)
        j = np.empty(n, np.int32)
        if n:
            lib().orc_get_list(self._h, which, _p(i, C.c_int), _p(j, C.c_int))
        return i, j

    def force(self, iflg: int):
        lib().orc_force(self._h, iflg)

    def force_ter(self, iflg: int):
        lib().orc_force_ter(self._h, iflg)

    def force_ter_e(self, iflg: int):
        lib().orc_force_ter_e(self._h, iflg)

    def fk_ewald(self):
        lib().orc_fk_ewald(self._h)

    def ecorr(self):
        lib().orc_ecorr(self._h)

    def fbond(self):
        lib().orc_fbond(self._h)

    def nhc_state(self):
        """the Nose-Hoover chains' (eta, veta), each ntherm x nchain"""
        nt, nc = int(self.sys.get("ntherm", 0)), int(self.sys.get("nchain", 0))
        eta, veta = np.zeros(max(nt * nc, 1)), np.zeros(max(nt * nc, 1))
        lib().orc_get_nhc(self._h, _p(eta), _p(veta))
        return eta[:nt * nc].reshape(nt, nc), veta[:nt * nc].reshape(nt, nc)

    def fbondx(self):
        lib().orc_fbondx(self._h)

    def ftors(self):
        lib().orc_ftors(self._h)

    def fonfo(self):
        lib().orc_fonfo(self._h)

    def fbend(self):
        lib().orc_fbend(self._h)

    def rmass(self, which: int):
        lib().orc_rmass(self._h, which)

    def energies(self) -> dict:
        e = _abi.Energies()
        lib().orc_get_energies(self._h, C.byref(e))
        return e.as_dict()

    def step_init(self):
        lib().orc_step_init(self._h)

    def step(self, istep0: int, nsteps: int):
        lib().orc_step(self._h, istep0, nsteps)

    @property
    def rebuilds(self) -> int:
        return lib().orc_rebuilds(self._h)

    @property
    def resets(self) -> int:
        return lib().orc_resets(self._h)

    @property
    def underflows(self) -> int:
        return lib().orc_underflows(self._h)


def load_golden(name: str) -> dict:
    path = os.path.join(os.path.dirname(HERE), "tests", "golden", f"{name}.npz")
    with np.load(path) as z:
        return {k: z[k] for k in z.files}

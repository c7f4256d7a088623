"""Python host mirror of CM3D's nonbonded entry points over the C ABI.

`Engine` wraps one device-resident system (libcm3d_nb.so, include/cm3d_nb.h)
and exposes CM3D's routines under CM3D's names:

    get_ngbr()            energy/control/ngbr_list.c:297
    nrefsh(istep)         energy/control/md_finter.c:43
    force(iflg)           energy/control/md_fcntr.c:44   (levels 0, 1, 2)
    force_ter(iflg)       energy/control/md_finter.c:110
    force_ter_e(iflg)     energy/control/md_finter_e.c:78
    fk_ewald()            energy/inter/md_ewald.c:185
    ecorr()               energy/inter/md_ewald.c:385
    getsvirter()          energy/inter/md_fnopol.c:386
    getsvirter_e()        energy/inter/finter_e.c:410
    getvewald()           energy/inter/md_ewald.c:364
    step_init(), step()   integrate/md_step.c:32, 62

Errors surface as `EngineError` carrying the library's message, where CM3D
would have called md_error().  There is no CPU fallback: without the built
library or a CUDA device the constructor raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import _abi
from .system import System

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libcm3d_nb.so")

_lib = None


class EngineError(RuntimeError):
    pass


def load_library() -> C.CDLL:
    """Load the in-tree engine library (build it first with
    `python -m cm3d_b200.build`); raises when it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise EngineError(f"{LIB_PATH} is missing: run `python -m cm3d_b200.build` "
                          "(the engine has no CPU fallback)")
    L = C.CDLL(LIB_PATH)
    vp, dp, ip = C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int)
    ll = C.c_longlong
    sig = {
        "cm3d_nb_version": (C.c_int, []),
        "cm3d_nb_last_error": (C.c_char_p, []),
        "cm3d_nb_device_count": (C.c_int, [ip]),
        "cm3d_nb_default_options": (None, [C.POINTER(_abi.Options)]),
        "cm3d_nb_create": (C.c_int, [C.POINTER(_abi.SystemDesc), C.POINTER(_abi.Options), C.POINTER(vp)]),
        "cm3d_nb_destroy": (None, [vp]),
        "cm3d_nb_create_batch": (C.c_int, [C.POINTER(_abi.SystemDesc), C.c_int, C.POINTER(_abi.Options),
                                           C.POINTER(vp)]),
        "cm3d_nb_num_systems": (C.c_int, [vp, ip]),
        "cm3d_nb_system_atoms": (C.c_int, [vp, C.c_int, ip, ip]),
        "cm3d_nb_get_system_energies": (C.c_int, [vp, C.c_int, C.POINTER(_abi.Energies)]),
        "cm3d_nb_get_all_energies": (C.c_int, [vp, C.POINTER(_abi.Energies)]),
        "cm3d_nb_system_counts": (C.c_int, [vp, C.POINTER(ll), C.POINTER(ll)]),
        "cm3d_nb_get_nhc": (C.c_int, [vp, C.c_int, dp, dp, ip, ip]),
        "cm3d_nb_set_positions": (C.c_int, [vp, dp, dp, dp]),
        "cm3d_nb_set_box": (C.c_int, [vp, dp]),
        "cm3d_nb_grid": (C.c_int, [vp, C.c_int, C.POINTER(C.c_int), ip, ip]),
        "cm3d_nb_get_positions": (C.c_int, [vp, dp, dp, dp]),
        "cm3d_nb_set_velocities": (C.c_int, [vp, dp, dp, dp]),
        "cm3d_nb_get_velocities": (C.c_int, [vp, dp, dp, dp]),
        "cm3d_nb_get_forces": (C.c_int, [vp, C.c_int, dp, dp, dp]),
        "cm3d_nb_set_forces": (C.c_int, [vp, C.c_int, dp, dp, dp]),
        "cm3d_nb_get_ngbr": (C.c_int, [vp]),
        "cm3d_nb_nrefsh": (C.c_int, [vp, C.c_int, ip]),
        "cm3d_nb_force": (C.c_int, [vp, C.c_int]),
        "cm3d_nb_force_ter": (C.c_int, [vp, C.c_int]),
        "cm3d_nb_force_ter_e": (C.c_int, [vp, C.c_int]),
        "cm3d_nb_fk_ewald": (C.c_int, [vp]),
        "cm3d_nb_ecorr": (C.c_int, [vp]),
        "cm3d_nb_zero_forces": (C.c_int, [vp, C.c_int]),
        "cm3d_nb_rmass": (C.c_int, [vp, C.c_int]),
        "cm3d_nb_getsvirter": (C.c_int, [vp, dp, dp, dp, dp]),
        "cm3d_nb_getsvirter_e": (C.c_int, [vp, dp, dp, dp]),
        "cm3d_nb_getvewald": (C.c_int, [vp, dp, dp, dp]),
        "cm3d_nb_step_init": (C.c_int, [vp]),
        "cm3d_nb_step": (C.c_int, [vp, C.c_int, C.c_int]),
        "cm3d_nb_step_async": (C.c_int, [vp, C.c_int, C.c_int]),
        "cm3d_nb_set_host_outputs": (C.c_int, [vp, dp, dp]),
        "cm3d_nb_step_host": (C.c_int, [vp, C.c_int, dp, dp]),
        "cm3d_nb_step_query": (C.c_int, [vp, ip]),
        "cm3d_nb_step_wait": (C.c_int, [vp]),
        "cm3d_nb_get_energies": (C.c_int, [vp, C.POINTER(_abi.Energies)]),
        "cm3d_nb_list_count": (C.c_int, [vp, C.c_int, C.POINTER(ll)]),
        "cm3d_nb_get_list": (C.c_int, [vp, C.c_int, ip, ip, ll, C.POINTER(ll)]),
        "cm3d_nb_get_status": (C.c_int, [vp, C.POINTER(_abi.Status)]),
        "cm3d_nb_synchronize": (C.c_int, [vp]),
        "cm3d_nb_stream": (vp, [vp]),
        "cm3d_nb_enable_timing": (C.c_int, [vp, C.c_int]),
        "cm3d_nb_kernel_time": (C.c_int, [vp, C.c_int, dp, C.POINTER(ll)]),
        "cm3d_nb_launch_count": (ll, [vp]),
        "cm3d_nb_measure_peaks": (C.c_int, [C.c_int, dp, dp]),
        "cm3d_nb_autotune": (C.c_int, [vp, C.c_int, ip, dp]),
        "cm3d_nb_pair_kernel": (C.c_int, [vp, ip, ip]),
        "cm3d_nb_lj_table": (C.c_int, [C.c_double] * 7 + [C.c_int, C.c_int, dp, dp, dp, dp]),
        "cm3d_nb_coul_table": (C.c_int, [C.c_double] * 6 + [C.c_int, C.c_int, C.c_int, dp, dp, dp, dp]),
        "cm3d_nb_ewald_kvectors": (C.c_int, [C.c_int, ip, ip, ip, ip, ip]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def last_error() -> str:
    return load_library().cm3d_nb_last_error().decode(errors="replace")


def check(rc: int, what: str) -> None:
    if rc != _abi.OK:
        raise EngineError(f"{what}: {last_error()} (code {rc})")


def device_count() -> int:
    n = C.c_int(0)
    load_library().cm3d_nb_device_count(C.byref(n))
    return int(n.value)


def _p(a: np.ndarray, t=C.c_double):
    return a.ctypes.data_as(C.POINTER(t))


def measure_peaks(device: int = 0) -> tuple[float, float]:
    """(FP32, FP64) FMA throughput of the device in TFLOP/s, measured now."""
    f32, f64 = C.c_double(0), C.c_double(0)
    check(load_library().cm3d_nb_measure_peaks(device, C.byref(f32), C.byref(f64)), "measure_peaks")
    return f32.value, f64.value


class Engine:
    """CM3D systems resident on one GPU: one system, or a batch of independent
    systems (a list) that every kernel of a step covers at once.  In a batch
    the per-atom arrays (positions, velocities, forces) hold all systems'
    atoms back to back; `ranges[s]` is system s's (first, natoms)."""

    def __init__(self, system, mode: int = _abi.MIXED, device: int = 0,
                 need_short: bool = False, tpa: int = 0, use_graph: bool = True, cell_scale: float = 1.0):
        L = load_library()
        systems = list(system) if isinstance(system, (list, tuple)) else [system]
        self.systems = systems
        self.sys = systems[0]
        self.nsys = len(systems)
        self.n = sum(s.natoms for s in systems)
        self.mode = mode
        opt = _abi.Options(device=device, mode=mode, need_short=int(need_short), tpa=tpa,
                           use_graph=int(use_graph), cell_scale=float(cell_scale))
        h = C.c_void_p()
        descs = (_abi.SystemDesc * self.nsys)(*[s.desc() for s in systems])
        check(L.cm3d_nb_create_batch(descs, self.nsys, C.byref(opt), C.byref(h)), "cm3d_nb_create_batch")
        self._h = h
        self.ranges = []
        a0 = 0
        for s in systems:
            self.ranges.append((a0, s.natoms))
            a0 += s.natoms

    def close(self) -> None:
        if getattr(self, "_h", None):
            load_library().cm3d_nb_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # --------------------------------------------------------- transfers
    def _get3(self, fn, *lead, out=None) -> np.ndarray:
        """x | y | z blocks into a new (3, n) array, or into `out` (a C-contiguous
        float64 (3, n) array, e.g. in pinned host memory: the copies then go
        straight into it)"""
        if out is None:
            out = np.empty((3, self.n))
        elif out.shape != (3, self.n) or out.dtype != np.float64 or not out.flags.c_contiguous:
            raise ValueError(f"out must be a C-contiguous float64 array of shape (3, {self.n})")
        check(fn(self._h, *lead, _p(out[0]), _p(out[1]), _p(out[2])), fn.__name__)
        return out

    def _set3(self, fn, a, *lead) -> None:
        a = np.asarray(a, dtype=np.float64)
        x, y, z = (np.ascontiguousarray(a[k]) for k in range(3))
        check(fn(self._h, *lead, _p(x), _p(y), _p(z)), fn.__name__)

    def positions(self, out=None) -> np.ndarray:
        return self._get3(load_library().cm3d_nb_get_positions, out=out)

    def set_positions(self, p) -> None:
        self._set3(load_library().cm3d_nb_set_positions, p)

    def set_box(self, hmat) -> None:
        """a new box matrix (row-major 3x3) for a one-system context"""
        h = np.ascontiguousarray(np.asarray(hmat, dtype=np.float64).reshape(9))
        check(load_library().cm3d_nb_set_box(self._h, h.ctypes.data_as(C.POINTER(C.c_double))), "set_box")

    def velocities(self, out=None) -> np.ndarray:
        return self._get3(load_library().cm3d_nb_get_velocities, out=out)

    def set_velocities(self, v) -> None:
        self._set3(load_library().cm3d_nb_set_velocities, v)

    def forces(self, which: int = _abi.FXL, out=None) -> np.ndarray:
        """The stored force block (accelerations after rmass, raw forces after
        force_ter/force_ter_e/fk_ewald/ecorr alone)."""
        return self._get3(load_library().cm3d_nb_get_forces, which, out=out)

    def set_forces(self, f, which: int = _abi.FXL) -> None:
        L = load_library()
        a = np.asarray(f, dtype=np.float64)
        x, y, z = (np.ascontiguousarray(a[k]) for k in range(3))
        check(L.cm3d_nb_set_forces(self._h, which, _p(x), _p(y), _p(z)), "set_forces")

    # ---------------------------------------------------- CM3D routines
    def get_ngbr(self) -> None:
        check(load_library().cm3d_nb_get_ngbr(self._h), "get_ngbr")

    def nrefsh(self, istep: int) -> bool:
        r = C.c_int(0)
        check(load_library().cm3d_nb_nrefsh(self._h, istep, C.byref(r)), "nrefsh")
        return bool(r.value)

    def force(self, iflg: int) -> None:
        check(load_library().cm3d_nb_force(self._h, iflg), f"force({iflg})")

    def force_ter(self, iflg: int) -> None:
        check(load_library().cm3d_nb_force_ter(self._h, iflg), f"force_ter({iflg})")

    def force_ter_e(self, iflg: int) -> None:
        check(load_library().cm3d_nb_force_ter_e(self._h, iflg), f"force_ter_e({iflg})")

    def fk_ewald(self) -> None:
        check(load_library().cm3d_nb_fk_ewald(self._h), "fk_ewald")

    def ecorr(self) -> None:
        check(load_library().cm3d_nb_ecorr(self._h), "ecorr")

    def zero_forces(self, which: int) -> None:
        check(load_library().cm3d_nb_zero_forces(self._h, which), "zero_forces")

    def rmass(self, which: int) -> None:
        check(load_library().cm3d_nb_rmass(self._h, which), "rmass")

    def getsvirter(self) -> dict:
        vh, v, w = C.c_double(0), C.c_double(0), C.c_double(0)
        t = np.zeros(9)
        check(load_library().cm3d_nb_getsvirter(self._h, C.byref(vh), C.byref(v), C.byref(w), _p(t)),
              "getsvirter")
        return {"vhinter": vh.value, "vinter": v.value, "winter": w.value, "wintertensor": t}

    def getsvirter_e(self) -> dict:
        v, w = C.c_double(0), C.c_double(0)
        t = np.zeros(9)
        check(load_library().cm3d_nb_getsvirter_e(self._h, C.byref(v), C.byref(w), _p(t)), "getsvirter_e")
        return {"velec": v.value, "welec": w.value, "welectensor": t}

    def autotune(self, reps: int = 5) -> dict:
        """Pick the pair kernel (gather, or the staged window/system kernel) and its lanes per atom by
        timing 4/8/16/32 on the current lists (cm3d_nb_autotune); returns the
        choice and, per lanes-per-atom choice, the faster kernel's time."""
        t = C.c_int(0)
        ms = np.zeros(4)
        check(load_library().cm3d_nb_autotune(self._h, reps, C.byref(t), _p(ms)), "autotune")
        nc, split, nt = self.grid(0)
        return {"tpa": int(t.value), "kernel": self.pair_kernel()[0], "cells": nc, "compact_split": split,
                "compact_block_threads": nt, "ms_per_launch": {4: ms[0], 8: ms[1], 16: ms[2], 32: ms[3]}}

    def grid(self, sys: int = 0) -> tuple[list, int, int]:
        """(cells per box direction of system `sys`, parts per cell of the compact kernel's work items,
        threads of its blocks (0 without the compact path))"""
        nc = (C.c_int * 3)()
        sp, nt = C.c_int(0), C.c_int(0)
        check(load_library().cm3d_nb_grid(self._h, sys, nc, C.byref(sp), C.byref(nt)), "grid")
        return [int(x) for x in nc], int(sp.value), int(nt.value)

    def pair_kernel(self) -> tuple[str, int]:
        """(kernel of the last pair launch: "gather", "window", "system", "compact" or "compact8" (a
        batch's compact lists with 8 lanes per atom), lanes per atom of the gather kernel)"""
        k, t = C.c_int(0), C.c_int(0)
        check(load_library().cm3d_nb_pair_kernel(self._h, C.byref(k), C.byref(t)), "pair_kernel")
        return {0: "gather", 1: "window", 2: "system", 3: "compact", 4: "compact8"}[k.value], int(t.value)

    def system_energies(self, sys: int) -> dict:
        """getvireal + geteng of one system of a batch"""
        e = _abi.Energies()
        check(load_library().cm3d_nb_get_system_energies(self._h, sys, C.byref(e)), "get_system_energies")
        return e.as_dict()

    def all_energies(self) -> list[dict]:
        arr = (_abi.Energies * self.nsys)()
        check(load_library().cm3d_nb_get_all_energies(self._h, arr), "get_all_energies")
        return [arr[k].as_dict() for k in range(self.nsys)]

    def energies_table(self, out=None) -> np.ndarray:
        """Every system's getvireal + geteng as one numpy structured array
        (fields of cm3d_nb_energies, one row per system), written into `out`
        when given: no per-system Python objects, for a host loop that reads
        all systems every step."""
        dt = _abi.Energies.numpy_dtype()
        assert dt.itemsize == C.sizeof(_abi.Energies)
        if out is None:
            out = np.empty(self.nsys, dtype=dt)
        elif out.dtype != dt or out.shape != (self.nsys,) or not out.flags.c_contiguous:
            raise ValueError("out must be a contiguous energies_table array of this engine")
        check(load_library().cm3d_nb_get_all_energies(self._h, out.ctypes.data_as(C.POINTER(_abi.Energies))),
              "get_all_energies")
        return out

    def nhc_state(self, sys: int = 0) -> tuple[np.ndarray, np.ndarray]:
        """NVT: system `sys`'s Nose-Hoover chain (eta, veta), ntherm x nchain
        each (empty for NVE)"""
        L = load_library()
        nt, nc = C.c_int(0), C.c_int(0)
        check(L.cm3d_nb_get_nhc(self._h, sys, None, None, C.byref(nt), C.byref(nc)), "get_nhc")
        eta, veta = np.zeros(max(nt.value * nc.value, 1)), np.zeros(max(nt.value * nc.value, 1))
        check(L.cm3d_nb_get_nhc(self._h, sys, _p(eta), _p(veta), None, None), "get_nhc")
        k = nt.value * nc.value
        return eta[:k].reshape(nt.value, nc.value), veta[:k].reshape(nt.value, nc.value)

    def system_counts(self) -> tuple[np.ndarray, np.ndarray]:
        """per-system (list rebuilds, RESETPOS events)"""
        rb = np.zeros(self.nsys, np.int64)
        rs = np.zeros(self.nsys, np.int64)
        check(load_library().cm3d_nb_system_counts(self._h, _p(rb, C.c_longlong), _p(rs, C.c_longlong)),
              "system_counts")
        return rb, rs

    def getvewald(self) -> dict:
        p, w = C.c_double(0), C.c_double(0)
        t = np.zeros(9)
        check(load_library().cm3d_nb_getvewald(self._h, C.byref(p), C.byref(w), _p(t)), "getvewald")
        return {"vewald": p.value, "wewald": w.value, "wewaldtensor": t}

    def step_init(self) -> None:
        check(load_library().cm3d_nb_step_init(self._h), "step_init")

    def step(self, istep0: int, nsteps: int = 1) -> None:
        check(load_library().cm3d_nb_step(self._h, istep0, nsteps), "step")

    def step_async(self, istep0: int, nsteps: int = 1) -> None:
        """launch the steps and return (cm3d_nb_step_async)"""
        check(load_library().cm3d_nb_step_async(self._h, istep0, nsteps), "step_async")

    def set_host_outputs(self, pos_out=None, vel_out=None) -> None:
        """register page-locked (3, n) float64 arrays that every later step
        fills with its final positions and velocities (cm3d_nb_set_host_outputs;
        None for both stops it); the arrays must stay alive while registered"""
        self._host_out = (pos_out, vel_out)

        def ptr(a):
            if a is None:
                return None
            if a.dtype != np.float64 or not a.flags.c_contiguous or a.size != 3 * self.n:
                raise EngineError("host outputs: C-contiguous float64 arrays of 3 x natoms")
            return a.ctypes.data_as(C.POINTER(C.c_double))
        check(load_library().cm3d_nb_set_host_outputs(self._h, ptr(pos_out), ptr(vel_out)), "set_host_outputs")

    def step_host(self, istep0: int, pos_in=None, vel_in=None) -> None:
        """copy the (3, n) float64 host arrays in (page-locked for an
        asynchronous copy; None keeps the device's) and run one step
        (cm3d_nb_step_host); registered outputs are complete on return"""
        def ptr(a):
            if a is None:
                return None
            if a.dtype != np.float64 or not a.flags.c_contiguous or a.size != 3 * self.n:
                raise EngineError("step_host: C-contiguous float64 arrays of 3 x natoms")
            return a.ctypes.data_as(C.POINTER(C.c_double))
        check(load_library().cm3d_nb_step_host(self._h, istep0, ptr(pos_in), ptr(vel_in)), "step_host")

    def step_done(self) -> bool:
        """non-blocking: have the launched steps completed?"""
        d = C.c_int(0)
        check(load_library().cm3d_nb_step_query(self._h, C.byref(d)), "step_query")
        return bool(d.value)

    def step_wait(self) -> None:
        check(load_library().cm3d_nb_step_wait(self._h), "step_wait")

    def energies(self) -> dict:
        e = _abi.Energies()
        check(load_library().cm3d_nb_get_energies(self._h, C.byref(e)), "get_energies")
        return e.as_dict()

    def pair_list(self, which: int) -> tuple[np.ndarray, np.ndarray]:
        L = load_library()
        n = C.c_longlong(0)
        check(L.cm3d_nb_list_count(self._h, which, C.byref(n)), "list_count")
        i = np.empty(max(n.value, 1), np.int32)
        j = np.empty(max(n.value, 1), np.int32)
        got = C.c_longlong(0)
        check(L.cm3d_nb_get_list(self._h, which, _p(i, C.c_int), _p(j, C.c_int), n.value, C.byref(got)),
              "get_list")
        return i[:got.value], j[:got.value]

    def status(self) -> dict:
        s = _abi.Status()
        check(load_library().cm3d_nb_get_status(self._h, C.byref(s)), "get_status")
        return {k: getattr(s, k) for k, _ in s._fields_}

    def synchronize(self) -> None:
        check(load_library().cm3d_nb_synchronize(self._h), "synchronize")

    def enable_timing(self, on: bool = True) -> None:
        check(load_library().cm3d_nb_enable_timing(self._h, int(on)), "enable_timing")

    def kernel_time(self, cls: int) -> tuple[float, int]:
        ms, n = C.c_double(0), C.c_longlong(0)
        check(load_library().cm3d_nb_kernel_time(self._h, cls, C.byref(ms), C.byref(n)), "kernel_time")
        return ms.value, n.value

    def launch_count(self) -> int:
        return int(load_library().cm3d_nb_launch_count(self._h))

    def stream(self) -> int:
        return int(load_library().cm3d_nb_stream(self._h) or 0)


# ----------------------------------------------------- host set-up helpers
def tune_cell_scale(systems, device: int = 0, scales=(1.0, 1.25), steps: int = 20, warmup: int = 5,
                    reps: int = 5) -> dict:
    """Cell size by measurement: for each candidate cell width (in list
    radii; cm3d_nb_options.cell_scale) a fresh mixed context of the same
    systems runs step_init, the kernel autotuner (pair kernel, lanes per
    atom, compact tile) and `warmup` + `steps` graph steps; the step time is
    measured with CUDA events around the timed steps.  Returns the fastest
    scale with every candidate's step time and kernel choice; the systems
    themselves are not changed.  Step times within 2% of the fastest count
    as a tie (the timing noise of a short run; a step whose critical path is
    the reciprocal space on its side stream barely sees the pair kernel),
    and the tie goes to the faster pair kernel."""
    import torch
    out = {}
    for s in scales:
        with Engine(systems, mode=_abi.MIXED, device=device, cell_scale=s) as e:
            e.step_init()
            tune = e.autotune(reps)
            e.step(1, warmup)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            st = torch.cuda.ExternalStream(e.stream(), device=device)
            e.synchronize()
            a.record(st)
            e.step_async(1 + warmup, steps)
            b.record(st)
            e.step_wait()
            b.synchronize()
            out[s] = {"ms_per_step": a.elapsed_time(b) / steps, "kernel": tune["kernel"], "tpa": tune["tpa"],
                      "cells": tune["cells"], "compact_split": tune["compact_split"],
                      "compact_block_threads": tune["compact_block_threads"],
                      "pair_ms": float(min(tune["ms_per_launch"].values()))}
    return {"cell_scale": pick_cell_scale(out), "candidates": out}


def pick_cell_scale(candidates: dict, tie: float = 0.02):
    """The cell scale of the fastest step among `candidates` ({scale:
    {"ms_per_step", "pair_ms"}}); steps within `tie` of the fastest count as
    equal and go to the faster pair kernel (then the faster step)."""
    fastest = min(v["ms_per_step"] for v in candidates.values())
    ties = [k for k in candidates if candidates[k]["ms_per_step"] <= (1.0 + tie) * fastest]
    return min(ties, key=lambda k: (candidates[k]["pair_ms"], candidates[k]["ms_per_step"]))


def lj_table(eps, sig, rmin, rmax, rres, rheal, skin, ntable, shift):
    """get_ter_parm's LJ table (input/md_getparm.c:236-366) via the C ABI."""
    L = load_library()
    v, dv, sw = np.empty(ntable), np.empty(ntable), np.empty(ntable)
    dx2 = C.c_double(0)
    check(L.cm3d_nb_lj_table(eps, sig, rmin, rmax, rres, rheal, skin, ntable, int(shift), _p(v), _p(dv),
                             _p(sw), C.byref(dx2)), "lj_table")
    return v, dv, sw, dx2.value


def coul_table(alpha, rmin, rresp, rmax, rheal, skin, ntable, iperd=3, shift=0):
    """set_charges' erfc table (energy/control/elec_ngbr.c:51-103) via the C ABI."""
    L = load_library()
    c, dc, sw = np.empty(ntable), np.empty(ntable), np.empty(ntable)
    dx2 = C.c_double(0)
    check(L.cm3d_nb_coul_table(alpha, rmin, rresp, rmax, rheal, skin, ntable, iperd, int(shift), _p(c),
                               _p(dc), _p(sw), C.byref(dx2)), "coul_table")
    return c, dc, sw, dx2.value


def ewald_kvectors(kmax: int):
    """ewald_setup's half-space spherical k set (energy/inter/md_ewald.c:93-114)."""
    L = load_library()
    n = C.c_int(0)
    null = C.POINTER(C.c_int)()
    check(L.cm3d_nb_ewald_kvectors(kmax, null, null, null, null, C.byref(n)), "ewald_kvectors")
    ka, kb, kc, kup = (np.empty(n.value + 1, np.int32) for _ in range(4))
    check(L.cm3d_nb_ewald_kvectors(kmax, _p(ka, C.c_int), _p(kb, C.c_int), _p(kc, C.c_int),
                                   _p(kup, C.c_int), C.byref(n)), "ewald_kvectors")
    return ka[:n.value], kb[:n.value], kc[:n.value], kup[:n.value + 1]

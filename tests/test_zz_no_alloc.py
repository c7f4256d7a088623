"""cm3d_nb_fk_ewald_noalloc (the reciprocal-space forces and totals computed
on the library's static scratch area, no device allocation) against the
engine's cm3d_nb_fk_ewald on the same system, called through the C ABI.

The file name sorts last so that, in a full run, the entry point is also
exercised after every other test has used the device; it passes alone too.

Tolerances (both paths run the same mixed-precision kernels; only the force
kernel's split, hence the order of its FP64 atomic adds, may differ)
  forces      relative RMS <= 1e-5 (the mixed engine's force bound)
  vk_ewald    relative <= 1e-5
  vp_ewald and the virial tensor   relative <= 5e-5 (of the largest entry)
"""
import ctypes as C

import numpy as np
import pytest

from conftest import force_scale, golden, rel_rms, xyz
from cm3d_b200 import _abi
from cm3d_b200.engine import Engine, ewald_kvectors, last_error
from cm3d_b200.system import System

pytestmark = pytest.mark.gpu

FTOL, ETOL, VTOL = 1e-5, 1e-5, 5e-5
MAX_CHARGES, MAX_KMAX = 32768, 15       # CM3D_NB_NOALLOC_MAX_* of include/cm3d_nb.h


def _fn(lib):
    fn = lib.cm3d_nb_fk_ewald_noalloc
    fn.restype = C.c_int
    fn.argtypes = [C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p,
                   C.POINTER(C.c_double), C.c_int, C.c_double, C.c_double, C.c_double,
                   C.c_void_p, C.c_void_p]
    return fn


class Bufs:
    """the caller's device buffers (allocated here, by the caller)"""

    def __init__(self, d):
        import torch
        self.torch = torch
        dev = torch.device("cuda", 0)
        self.n = int(d["natoms"][0])
        self.pos = torch.tensor(np.concatenate([d["px"], d["py"], d["pz"]]), dtype=torch.float64, device=dev)
        self.q = torch.tensor(d["qch"], dtype=torch.float64, device=dev)
        self.icharge = torch.tensor(d["icharge"], dtype=torch.int32, device=dev)
        self.nq = int(self.icharge.numel())
        self.fxl = torch.zeros(3 * self.n, dtype=torch.float64, device=dev)
        self.out = torch.full((11,), float("nan"), dtype=torch.float64, device=dev)
        self.hmat = (C.c_double * 9)(*[float(x) for x in d["hmat"]])

    def call(self, fn, d, kmax, ncharge=None):
        st = self.torch.cuda.current_stream().cuda_stream
        return fn(0, C.c_void_p(st), self.n, self.pos.data_ptr(), self.q.data_ptr(),
                  self.nq if ncharge is None else ncharge, self.icharge.data_ptr(), self.hmat, kmax,
                  float(d["falp2"][0]), float(d["ewald_self"][0]), float(d["ewald_bkg"][0]),
                  self.fxl.data_ptr(), self.out.data_ptr())


def _kmax(d):
    kmax = int(d["ka"].max())
    ka, kb, kc, _ = ewald_kvectors(kmax)
    n = int(d["ktot"][0])
    assert len(ka) == n
    assert (ka == d["ka"][:n]).all() and (kb == d["kb"][:n]).all() and (kc == d["kc"][:n]).all()
    return kmax


@pytest.mark.parametrize("name", ["water216", "binary256", "water4096"])
def test_noalloc_matches_fk_ewald(engine_lib, name):
    d = golden(name)
    assert (np.flatnonzero(d["qch"] != 0) == d["icharge"]).all()
    kmax = _kmax(d)
    # the existing entry point, through an engine context
    e = Engine(System.from_arrays(d), mode=_abi.MIXED)
    e.zero_forces(_abi.FXL)
    e.fk_ewald()
    f_ref = e.forces(_abi.FXL)
    tot = e.getvewald()
    e.close()
    want = np.concatenate([[tot["vewald"], tot["wewald"]], tot["wewaldtensor"]])

    fn = _fn(engine_lib)
    b = Bufs(d)
    fs = force_scale(d)
    for call in range(2):               # two calls in a row on the same scratch
        b.fxl.zero_()
        b.out.fill_(float("nan"))
        rc = b.call(fn, d, kmax)
        assert rc == _abi.OK, last_error()
        b.torch.cuda.synchronize()
        f = b.fxl.cpu().numpy().reshape(3, -1)
        out = b.out.cpu().numpy()
        assert rel_rms(f, f_ref, fs) <= FTOL, call
        assert rel_rms(f, xyz(d, "f_k"), fs) <= FTOL, call       # CM3D's own fk_ewald forces
        assert abs(out[0] - want[0]) <= ETOL * abs(want[0]), (call, out[0], want[0])
        vscale = np.abs(want[1:]).max()
        assert np.all(np.abs(out[1:] - want[1:]) <= VTOL * vscale), (call, out[1:], want[1:])
        assert abs(out[0] - float(d["vk_ewald"][0])) <= ETOL * abs(float(d["vk_ewald"][0]))


def test_noalloc_adds_to_fxl(engine_lib):
    """forces are added to what fxl holds, as fk_ewald adds to COORDS.fxl"""
    d = golden("water216")
    kmax = _kmax(d)
    fn = _fn(engine_lib)
    b = Bufs(d)
    b.fxl.zero_()
    assert b.call(fn, d, kmax) == _abi.OK, last_error()
    once = b.fxl.clone()
    assert b.call(fn, d, kmax) == _abi.OK, last_error()
    b.torch.cuda.synchronize()
    assert b.torch.allclose(b.fxl, 2 * once, rtol=1e-12, atol=0)


def test_noalloc_rejects_sizes_beyond_its_scratch(engine_lib):
    d = golden("water216")
    fn = _fn(engine_lib)
    b = Bufs(d)
    b.n = MAX_CHARGES + 1               # only the sizes are checked: nothing is launched
    rc = b.call(fn, d, 7, ncharge=MAX_CHARGES + 1)
    assert rc == _abi.ERR_ARG
    assert "CM3D_NB_NOALLOC_MAX_CHARGES" in last_error()
    b.n = int(d["natoms"][0])
    rc = b.call(fn, d, MAX_KMAX + 1)
    assert rc == _abi.ERR_ARG
    assert "CM3D_NB_NOALLOC_MAX_KMAX" in last_error()

"""cm3d_nb_set_box: a context follows a new box matrix (CM3D's barostat,
intbar in integrate/md_step.c, scales the box and the positions between
force calls; route B hands the engine each new box).

The check: a context built on the original box, handed the box scaled by
0.99 (isotropic) or a small shear (a flexible cell) and the positions scaled
with it, gives the level-1 forces, energies and virials of a fresh context
built on the new box and positions -- in the plain FP64 engine to 1e-11, in
the mixed engine to FP32 summation order (1e-6; its cell-relative
coordinates and cell shifts both follow the box).  The lists are rebuilt in
both, so both hold the pairs of the new geometry.  A box that shrinks below
the cell grid is refused.
"""
import numpy as np
import pytest

from conftest import golden, rel_rms
from cm3d_b200 import _abi
from cm3d_b200.engine import Engine, EngineError
from cm3d_b200.system import System

pytestmark = pytest.mark.gpu


def scaled(d: dict, m: np.ndarray) -> dict:
    """the system with box H' = m H and positions x' = m x"""
    out = dict(d)
    h = np.asarray(d["hmat"], float).reshape(3, 3)
    out["hmat"] = (m @ h).reshape(-1)
    p = np.stack([d["px"], d["py"], d["pz"]]).astype(float)
    q = m @ p
    out["px"], out["py"], out["pz"] = q[0].copy(), q[1].copy(), q[2].copy()
    return out


def level1(e: Engine):
    e.get_ngbr()
    e.force(1)
    f = e.forces(_abi.FXL)
    e.force(2)
    return f, e.energies()


@pytest.mark.parametrize("name", ["water4096", "binary256"])
@pytest.mark.parametrize("mode", [_abi.PLAIN_FP64, _abi.MIXED], ids=["plain", "mixed"])
@pytest.mark.parametrize("kind", ["iso", "shear"])
def test_set_box_matches_a_fresh_context(engine_lib, name, mode, kind):
    d = golden(name)
    m = np.eye(3) * 0.99 if kind == "iso" else np.array([[1.0, 0.004, 0.0], [0.0, 1.0, -0.003], [0.0, 0.0, 1.0]])
    d2 = scaled(d, m)
    e = Engine(System.from_arrays(d), mode=mode)
    e.get_ngbr()
    e.force(1)
    e.set_box(np.asarray(d2["hmat"], float))
    e.set_positions(np.stack([d2["px"], d2["py"], d2["pz"]]))
    f1, en1 = level1(e)
    e.close()
    fresh = Engine(System.from_arrays(d2), mode=mode)
    f2, en2 = level1(fresh)
    fresh.close()
    tol = 1e-11 if mode == _abi.PLAIN_FP64 else 1e-6
    assert rel_rms(f1, f2) <= tol
    for k in ("vinter", "velec", "vewald", "U", "W", "prsi", "winter", "welec"):
        assert abs(en1[k] - en2[k]) <= tol * max(abs(en2[k]), 1.0), (k, en1[k], en2[k])
    np.testing.assert_allclose(en1["Wtensor"], en2["Wtensor"], rtol=tol * 10, atol=tol * abs(en2["W"]))


def test_set_box_refuses_a_box_below_the_cell_grid(engine_lib):
    d = golden("water4096")
    e = Engine(System.from_arrays(d), mode=_abi.MIXED)
    e.get_ngbr()
    h = np.asarray(d["hmat"], float) * 0.5
    with pytest.raises(EngineError, match="shrank below the cell grid"):
        e.set_box(h)
    e.close()

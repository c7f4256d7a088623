"""The FP32 decision margin of the staged list build (k_list_win's fast_flags).

In a cell grid of 3 or more cells per axis the staged list build compares
FP32 squared distances with the list radii and falls back to CM3D's FP64 test
only within 4e-5 R^2 + 2e-3 A^2 of a radius.  That is sound only if the FP32
squared distance -- formed the way the kernel forms it -- never errs by more
than that margin.  The kernel's recipe:

- cell-relative coordinates xq = fp32(r - corner);
- the staged j moved by the FP32 cell shift, xs = xq_j - fp32(H k / nc);
- d = xq_i - xs, and r2 = d.d in FP32.

This test builds those numbers in numpy (FP32 arithmetic) on the golden
boxes and on random boxes whose cells are almost two list radii wide (the
widest the grid makes), and bounds the error against the FP64 minimum-image
distance.  The GPU tests check the lists themselves bit-exact against CM3D.
"""
import numpy as np
import pytest

from conftest import golden

MARGIN_REL, MARGIN_ABS = 4e-5, 2e-3          # fast_flags: fabsf(r2f - R2) < 4e-5 R2 + 2e-3


def fp32_r2_errors(pos: np.ndarray, h: np.ndarray, rlist: float, nmax_pairs: int = 400000, seed: int = 0):
    """(FP64 r^2, |FP32 r^2 - FP64 r^2|) for pairs within rlist + 1 A, the
    FP32 value formed as the staged list build forms it (orthorhombic box,
    nc = floor(L / rlist) >= 3 per axis)."""
    L = np.diag(h)
    nc = np.floor(L / rlist).astype(int)
    assert (nc >= 3).all()
    w = L / nc
    n = pos.shape[0]
    s = pos / L
    s -= np.floor(s)
    cell = np.minimum((s * nc).astype(int), nc - 1)
    corner = cell * w
    # atoms are not wrapped: the corner is the cell's origin in the atom's
    # own periodic image, as the engine keeps it
    img = np.floor(pos / L)
    corner = corner + img * L
    xq = (pos - corner).astype(np.float32)
    rng = np.random.default_rng(seed)
    i = rng.integers(0, n, nmax_pairs)
    j = rng.integers(0, n, nmax_pairs)
    keep = i != j
    i, j = i[keep], j[keep]
    # stencil offset of j's cell from i's cell (periodic), and the FP64 shift
    o = cell[j] - cell[i]
    o = np.where(o > nc // 2, o - nc, np.where(o < -(nc // 2), o + nc, o))
    near = (np.abs(o) <= 1).all(axis=1)
    i, j, o = i[near], j[near], o[near]
    k = -o
    # shift so that d = (xq_i - xq_j) + S is the minimum-image displacement:
    # S = corner_i - corner_j + (image shift) = H k / nc + lattice vector
    d64 = pos[i] - pos[j]
    d64 -= L * np.round(d64 / L)
    S64 = d64 - ((pos[i] - corner[i]) - (pos[j] - corner[j]))
    S32 = S64.astype(np.float32)
    xs = (xq[j] - S32).astype(np.float32)
    d32 = (xq[i] - xs).astype(np.float32)
    r2f = (d32[:, 0] * d32[:, 0] + d32[:, 1] * d32[:, 1]).astype(np.float32) + d32[:, 2] * d32[:, 2]
    r2 = (d64 * d64).sum(axis=1)
    sel = r2 < (rlist + 1.0) ** 2
    return r2[sel], np.abs(r2f[sel].astype(np.float64) - r2[sel])


@pytest.mark.parametrize("name", ["argon864", "water4096"])
def test_fp32_distance_error_is_far_inside_the_margin_golden(name):
    d = golden(name)
    pos = np.stack([d["px"], d["py"], d["pz"]], axis=1)
    h = d["hmat"].reshape(3, 3)
    r2l = float(np.max(d["rmaxl_skin2"]))
    if "rmaxl_skin2_e" in d and float(np.asarray(d["rmaxl_skin2_e"]).max()) > 0:
        r2l = max(r2l, float(np.asarray(d["rmaxl_skin2_e"]).max()))
    rlist = float(np.sqrt(r2l))
    r2, err = fp32_r2_errors(pos, h, rlist)
    assert r2.size > 1000
    margin = MARGIN_REL * r2 + MARGIN_ABS
    # the margin is at least 5x the worst error seen
    assert (err * 5 < margin).all(), float((err / margin).max())


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_fp32_distance_error_wide_cells_random(seed):
    """cells of 1.9 list radii (nc = 3, the widest cells the grid makes), atoms
    anywhere in them, including a drift of up to half a skin past the cell"""
    rng = np.random.default_rng(seed)
    rlist = 12.0
    L = 3 * 1.9 * rlist
    pos = rng.uniform(-0.3, L + 0.3, size=(4000, 3))
    r2, err = fp32_r2_errors(pos, np.diag([L, L, L]), rlist, seed=seed)
    assert r2.size > 1000
    margin = MARGIN_REL * r2 + MARGIN_ABS
    assert (err * 5 < margin).all(), float((err / margin).max())

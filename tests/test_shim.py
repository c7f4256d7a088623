"""CM3D itself, relinked with the engine in place of its md_step.o
(cm3d_b200/shim), against the unmodified CM3D on the same input decks.

Both programs are CM3D's own main program, input readers, averaging and
writers (main/md_mdcntr.new.c, output/md_writescreen.c); only step_init() and
step() differ (integrate/md_step.c:32-159 on the host against the B200
engine).  The tests compare what a CM3D user sees: every screen report
(<...> = average ~ instantaneous, the pressure tensor, the pair counts and
<ts/update>) and the final restart coordinates.

Tolerances: the plain FP64 engine sums the same FP64 terms in another order,
so its printed values agree with CM3D to a few units in the last printed
digit (on B200 they are identical, restart file included).  The mixed engine
carries forces to a relative RMS error of 1e-5 per evaluation; after 20 steps
of a liquid its printed energies and pressures differ from CM3D's by up to
8e-5 relative (the scalar pressure, a small difference of large virials), so
the test allows 2e-4 (tensor entries: 2e-4 of the tensor's largest entry).

The CPU tests need no GPU: a deck the engine does not support stops at
step_init with the reason, and a run without a CUDA device stops with the
CUDA error -- neither falls back to CM3D's CPU step.
"""
import os
import re
import subprocess

import numpy as np
import pytest

from cm3d_b200 import configs

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CPU_CM3D = os.path.join(ROOT, "oracle", "_ref", "cm3d")
GPU_CM3D = os.path.join(ROOT, "cm3d_b200", "shim", "_build", "cm3d_gpu")
# route B: CM3D's own step() and host integrator; get_ngbr, nrefsh, force and
# getvireal bound to the engine
GPU_CM3D_B = os.path.join(ROOT, "cm3d_b200", "shim", "_build", "cm3d_gpu_b")

needs_bins = pytest.mark.skipif(
    not (os.path.exists(CPU_CM3D) and os.path.exists(GPU_CM3D)),
    reason="CM3D and its relinked build are made from the CM3D source tree (make -C oracle ref; "
           "make -C cm3d_b200/shim)")

needs_bins_b = pytest.mark.skipif(
    not (os.path.exists(CPU_CM3D) and os.path.exists(GPU_CM3D_B)),
    reason="CM3D and its route-B build are made from the CM3D source tree (make -C oracle ref; "
           "make -C cm3d_b200/shim)")

VAL = re.compile(r"^<([^>]+)>\s*=\s*(\S+)\s*~\s*(\S+)")
NUM = re.compile(r"[-+]?\d+(?:\.\d*)?(?:[eE][-+]?\d+)?")


def deck(kind: str):
    if kind == "argon":
        wl = configs.argon_fcc(ncell=4, ntime=20)
    elif kind == "argon_nvt":
        # CM3D's NVT: one global Nose-Hoover chain of length 3 (the chain
        # state goes to the engine and comes back into COORDS every step)
        wl = configs.argon_fcc(ncell=4, ntime=20, nvt_chain=3)
    elif kind in ("argon_npt_i", "argon_npt_f"):
        # CM3D's barostats (route B: integrated on the host, the engine
        # follows the box)
        wl = configs.argon_fcc(ncell=4, ntime=20, npt=kind[6:])
    else:
        wl = configs.water_box(ngrid=6, ntime=20, seed=7, placement="octant")
    wl.keywords["iwr_screen"] = 10
    return wl


def run(exe, wl, directory, env_extra=None):
    inp = wl.write(str(directory))
    env = dict(os.environ)
    env.update(env_extra or {})
    p = subprocess.run([exe, os.path.basename(inp)], cwd=str(directory), env=env,
                       stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True, timeout=600)
    return p.returncode, p.stdout


def parse_reports(text: str) -> list[dict]:
    """The screen reports of a CM3D run: the initial report and one per
    iwr_screen steps, each with its pair counts, <...> values and pressure
    tensor rows."""
    blocks, cur = [], None
    for ln in text.splitlines():
        s = ln.strip()
        if s.startswith("npairs ="):
            cur = {"ints": [int(x) for x in re.findall(r"=(\d+)", s)], "vals": [], "tensor": [],
                   "update": None}
            blocks.append(cur)
        elif s.startswith("nprs="):
            nums = re.findall(r"=\s*(" + NUM.pattern + ")", s)
            cur = {"ints": [int(x) for x in nums[:4]], "update": float(nums[4]), "vals": [],
                   "tensor": []}
            blocks.append(cur)
        elif cur is None:
            continue
        elif VAL.match(s):
            m = VAL.match(s)
            cur["vals"].append((m.group(1), float(m.group(2)), float(m.group(3))))
        elif re.match(r"^(Temp|Pressure)\s*=", s):
            # the initial report prints these with six significant digits
            v = float(NUM.findall(s)[0])
            cur["vals"].append((s.split()[0] + "%g", v, v))
        elif "~" in s and s.endswith("atm"):
            cur["tensor"].append([float(x) for x in NUM.findall(s)])
    return blocks


def read_restart(path: str):
    with open(path) as fh:
        rows = [ln.split() for ln in fh if ln.strip()]
    n = int(rows[0][0])
    pos = np.array([[float(x) for x in r[:3]] for r in rows[1:1 + n]])
    hmat = np.array([[float(x) for x in r[:3]] for r in rows[1 + n:4 + n]])
    return pos, hmat


def compare(cpu_out: str, gpu_out: str, rtol: float, atol: float, exact_counts: bool, small_rtol: dict | None = None):
    a, b = parse_reports(cpu_out), parse_reports(gpu_out)
    assert len(a) == len(b) and len(a) >= 3, (len(a), len(b))
    for k, (x, y) in enumerate(zip(a, b)):
        if exact_counts or k == 0:
            assert x["ints"] == y["ints"], (k, x["ints"], y["ints"])
            assert x["update"] == y["update"], (k, x["update"], y["update"])
        else:
            assert np.allclose(x["ints"], y["ints"], rtol=1e-3, atol=0), (k, x["ints"], y["ints"])
        assert [v[0] for v in x["vals"]] == [v[0] for v in y["vals"]]
        for (name, c0, c1), (_, g0, g1) in zip(x["vals"], y["vals"]):
            rt = max(rtol, 1e-5) if name.endswith("%g") else rtol
            rt = max(rt, (small_rtol or {}).get(name, 0.0))
            for c, g in ((c0, g0), (c1, g1)):
                assert abs(g - c) <= rt * abs(c) + atol, (k, name, c, g)
        tc, tg = np.array(x["tensor"]), np.array(y["tensor"])
        assert tc.shape == tg.shape and tc.shape in ((0,), (3, 6)), (k, tc.shape, tg.shape)
        if tc.size:
            scale = max(float(np.abs(tc).max()), 1.0)
            assert np.abs(tg - tc).max() <= rtol * scale + atol, (k, tc, tg)


@needs_bins
@pytest.mark.gpu
@pytest.mark.timeout(900)
@pytest.mark.parametrize("kind", ["argon", "water", "argon_nvt"])
@pytest.mark.parametrize("mode", ["plain", "mixed"])
def test_relinked_cm3d_matches_cm3d(tmp_path, kind, mode):
    wl = deck(kind)
    rc, cpu_out = run(CPU_CM3D, wl, tmp_path / "cpu")
    assert rc == 0, cpu_out[-2000:]
    rc, gpu_out = run(GPU_CM3D, wl, tmp_path / "gpu", {"CM3D_NB_MODE": mode, "CM3D_NB_DEVICE": "0"})
    assert rc == 0, gpu_out[-2000:]
    assert "B200 nonbonded engine" in gpu_out
    if mode == "plain":
        compare(cpu_out, gpu_out, rtol=1e-7, atol=3e-6, exact_counts=True)
        pos_tol = 3e-4
    else:
        compare(cpu_out, gpu_out, rtol=2e-4, atol=3e-6, exact_counts=False)
        pos_tol = 2e-3
    pc, hc = read_restart(str(tmp_path / "cpu" / f"{wl.name}.rest_N"))
    pg, hg = read_restart(str(tmp_path / "gpu" / f"{wl.name}.rest_N"))
    assert pc.shape == pg.shape == (wl.natoms, 3)
    np.testing.assert_array_equal(hc, hg)
    assert float(np.abs(pg - pc).max()) <= pos_tol


@needs_bins_b
@pytest.mark.gpu
@pytest.mark.timeout(900)
@pytest.mark.parametrize("kind", ["argon", "water", "argon_nvt", "argon_npt_i", "argon_npt_f"])
@pytest.mark.parametrize("mode", ["plain", "mixed"])
def test_route_b_binding_matches_cm3d(tmp_path, kind, mode):
    """Route B: CM3D's own step() (its RESPA loop and, for NVT, its
    Nose-Hoover chains on the host) with the neighbour lists, the skin test
    and every force level on the engine -- positions in and forces out at
    each call.  Same reports and tolerances as the relinked step."""
    wl = deck(kind)
    rc, cpu_out = run(CPU_CM3D, wl, tmp_path / "cpu")
    assert rc == 0, cpu_out[-2000:]
    rc, gpu_out = run(GPU_CM3D_B, wl, tmp_path / "gpu", {"CM3D_NB_MODE": mode, "CM3D_NB_DEVICE": "0"})
    assert rc == 0, gpu_out[-2000:]
    if mode == "plain":
        compare(cpu_out, gpu_out, rtol=1e-7, atol=3e-6, exact_counts=True)
        pos_tol = 3e-4
    else:
        # under a barostat the volume and its chain integrate the pressure, a
        # small difference of large virials: the mixed engine's virial error
        # (<= 5e-5) becomes about 1e-3 of the pressure, which the barostat
        # carries into the volume, its kinetic energy and the conserved
        # energy (2e-4 of Ham/N after 20 steps of strong compression); the
        # chains' energies (tenths of a K) then differ by up to 0.5%
        chains = {k: 1e-2 for k in ("Ueta/NC", "Keta/NC", "Ubar/NB", "Kbar/NB")} if "npt" in kind else None
        compare(cpu_out, gpu_out, rtol=2e-3 if "npt" in kind else 2e-4, atol=1e-3 if "npt" in kind else 3e-6,
                exact_counts=False, small_rtol=chains)
        pos_tol = 2e-3
    pc, hc = read_restart(str(tmp_path / "cpu" / f"{wl.name}.rest_N"))
    pg, hg = read_restart(str(tmp_path / "gpu" / f"{wl.name}.rest_N"))
    if "npt" in kind:
        # the box moved with the barostat, the same way in both programs
        assert not np.array_equal(hc, np.diag([wl.box] * 3))
        # relative to the box's size: under NPT_F the off-diagonal elements
        # are small (1e-5 of the edge) and carry the diagonal's absolute error
        tol = 1e-9 if mode == "plain" else 1e-6
        np.testing.assert_allclose(hg, hc, rtol=tol, atol=tol * float(np.abs(hc).max()))
    else:
        np.testing.assert_array_equal(hc, hg)
    assert float(np.abs(pg - pc).max()) <= pos_tol


@needs_bins_b
def test_route_b_binding_without_a_device_fails_loudly(tmp_path):
    """the bound get_ngbr (called by CM3D's own step_init) reaches the engine
    and stops there without a device: CM3D's host list and force routines
    are not what runs"""
    wl = configs.argon_fcc(ncell=3, ntime=2)
    rc, out = run(GPU_CM3D_B, wl, tmp_path, {"CUDA_VISIBLE_DEVICES": ""})
    assert rc != 0
    assert "GPU nonbonded engine: cm3d_nb_create" in out
    assert "Begining Molecular Dynamics" not in out


@needs_bins
def test_relinked_cm3d_refuses_unsupported_input(tmp_path):
    wl = configs.argon_fcc(ncell=3, ntime=2)
    wl.keywords["iperd"] = 0
    rc, out = run(GPU_CM3D, wl, tmp_path)
    assert rc != 0
    assert "GPU nonbonded engine: a non-periodic or partially periodic box (iperd != 3) is not supported" in out
    assert "Begining Molecular Dynamics" not in out


@needs_bins
def test_relinked_cm3d_without_a_device_fails_loudly(tmp_path):
    wl = configs.argon_fcc(ncell=3, ntime=2)
    rc, out = run(GPU_CM3D, wl, tmp_path, {"CUDA_VISIBLE_DEVICES": ""})
    assert rc != 0
    assert "GPU nonbonded engine: cm3d_nb_create" in out
    assert "Begining Molecular Dynamics" not in out


@needs_bins
def test_relinked_cm3d_accepts_a_torsion_deck(tmp_path):
    """CM3D's own test/abutane deck (torsions, 1-4 pairs, cross bonds, frozen
    atoms) passes the shim's feature check and reaches the engine; without a
    device it then stops at cm3d_nb_create, not with an "is not supported".
    The deck is read from the reference tree, so this host-only test is
    skipped where that tree is absent."""
    import shutil
    src = os.path.join(os.environ.get("CM3D_REF", ""), "test", "abutane")
    if not os.environ.get("CM3D_REF") or not os.path.isdir(src):
        pytest.skip("the reference tree's test/abutane deck is not on this machine")
    work = tmp_path / "abutane"
    shutil.copytree(src, work)
    for root, _dirs, files in os.walk(work):
        for f in files:
            os.chmod(os.path.join(root, f), 0o644)
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    p = subprocess.run([GPU_CM3D, "abutane.input"], cwd=str(work), env=env, stdout=subprocess.PIPE,
                       stderr=subprocess.STDOUT, text=True, timeout=300)
    assert p.returncode != 0
    assert "is not supported" not in p.stdout, p.stdout[-2000:]
    assert "GPU nonbonded engine: cm3d_nb_create" in p.stdout, p.stdout[-2000:]

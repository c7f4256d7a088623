"""Writes the energy-conservation fixtures: CM3D's own NVE trajectories, as
the per-step conserved energy ham = poth + potra + zke
(integrate/md_averages.new.c:100), and the equilibrated water state they
start from.

  argon864     LJ argon FCC 6^3 x 4, rho* 0.8442, 120 K, dt 5 fs: 1000 NVE
               steps from the FCC start (the generator's own state)
  water12288   4096 flexible waters (the golden fixture's generator), RESPA
               0.5/2 fs.  Its lattice start is far from equilibrium (the
               kinetic energy doubles in 40 steps), so CM3D first runs 1000
               steps with its velocity rescaling to 300 K every 10 steps
               (keyword rescalevel, main/md_mdcntr.new.c:197-199); its
               restart file is the NVE start, kept in water12288_eq.npz,
               and 1000 NVE steps follow.

CM3D runs as oracle/_ref/cm3d and oracle/_ref/ref_bench (built from CM3D's
sources by oracle/Makefile) on decks that cm3d_b200.configs writes in CM3D's
input formats.  Outputs: tests/golden/nve_cm3d.json and
tests/golden/water12288_eq.npz.

    python tests/golden/make_nve.py
"""
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from cm3d_b200 import configs  # noqa: E402

NSTEPS = 1000
EQ_STEPS = 1000
REF = os.path.join(ROOT, "oracle", "_ref")
GOLDEN = os.path.join(ROOT, "tests", "golden")


def trace(wl, nsteps):
    with tempfile.TemporaryDirectory() as tmp:
        inp = wl.write(tmp)
        out = subprocess.run([os.path.join(REF, "ref_bench"), os.path.basename(inp), str(nsteps), "0", "trace"],
                             cwd=tmp, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True,
                             check=True).stdout
    ham = []
    for ln in out.splitlines():
        if ln.startswith("T "):
            _, _, poth, potra, zke = ln.split()
            ham.append(float(poth) + float(potra) + float(zke))
    assert len(ham) == nsteps, len(ham)
    return ham


def equilibrate(wl, nsteps, every):
    """CM3D itself with velocity rescaling every `every` steps; its restart
    file after `nsteps` steps"""
    kw = dict(wl.keywords)
    kw.update({"ntime": nsteps, "rescalevel": every, "iwr_dump": nsteps})
    run = configs.Workload(**{**wl.__dict__, "keywords": kw})
    with tempfile.TemporaryDirectory() as tmp:
        inp = run.write(tmp)
        subprocess.run([os.path.join(REF, "cm3d"), os.path.basename(inp)], cwd=tmp, stdout=subprocess.DEVNULL,
                       stderr=subprocess.DEVNULL, check=True)
        return configs.read_restart(os.path.join(tmp, kw["dpo_file"]))


def main():
    out = {}
    wl = configs.argon_fcc(seed=1, ntime=NSTEPS)
    out["argon864"] = {"natoms": wl.natoms, "dt_ps": wl.dt_fs / 1000.0, "nsteps": NSTEPS,
                       "start": "FCC lattice", "ham": trace(wl, NSTEPS)}
    print("argon864 done", flush=True)
    wl = configs.water_box(ngrid=16, seed=1, ntime=NSTEPS)
    pos, vel = equilibrate(wl, EQ_STEPS, 10)
    np.savez_compressed(os.path.join(GOLDEN, "water12288_eq.npz"), pos=pos, vel=vel)
    out["water12288"] = {"natoms": wl.natoms, "dt_ps": wl.dt_fs / 1000.0, "nsteps": NSTEPS,
                         "start": f"water12288_eq.npz ({EQ_STEPS} steps rescaled to 300 K every 10)",
                         "ham": trace(wl.with_state(pos, vel), NSTEPS)}
    print("water12288 done", flush=True)
    with open(os.path.join(GOLDEN, "nve_cm3d.json"), "w") as fh:
        json.dump(out, fh)


if __name__ == "__main__":
    main()

"""Writes tests/golden/nve_cm3d.json: CM3D's own NVE trajectories of the two
energy-conservation configurations, as the per-step conserved energy
ham = poth + potra + zke (integrate/md_averages.new.c:100).

  argon864     LJ argon FCC 6^3 x 4, rho* 0.8442, 120 K, dt 5 fs, 1000 steps
  water12288   4096 flexible waters (the golden fixture's generator),
               RESPA 0.5/2 fs, 1000 outer steps

CM3D runs through oracle/_ref/ref_bench (built from CM3D's sources by
oracle/Makefile) in its trace mode, from decks that cm3d_b200.configs writes
in CM3D's input formats with the same initial state the engine starts from.

    python tests/golden/make_nve.py
"""
import json
import os
import subprocess
import sys
import tempfile

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from cm3d_b200 import configs  # noqa: E402

NSTEPS = 1000
CASES = {
    "argon864": lambda: configs.argon_fcc(seed=1, ntime=NSTEPS),
    "water12288": lambda: configs.water_box(ngrid=16, seed=1, ntime=NSTEPS),
}


def trace(wl, nsteps):
    exe = os.path.join(ROOT, "oracle", "_ref", "ref_bench")
    with tempfile.TemporaryDirectory() as tmp:
        inp = wl.write(tmp)
        out = subprocess.run([exe, os.path.basename(inp), str(nsteps), "0", "trace"], cwd=tmp,
                             stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True, check=True).stdout
    ham = []
    for ln in out.splitlines():
        if ln.startswith("T "):
            _, _, poth, potra, zke = ln.split()
            ham.append(float(poth) + float(potra) + float(zke))
    assert len(ham) == nsteps, len(ham)
    return ham


def main():
    out = {}
    for name, make in CASES.items():
        wl = make()
        out[name] = {"natoms": wl.natoms, "dt_ps": wl.dt_fs / 1000.0, "nsteps": NSTEPS, "ham": trace(wl, NSTEPS)}
        print(name, "done", flush=True)
    with open(os.path.join(ROOT, "tests", "golden", "nve_cm3d.json"), "w") as fh:
        json.dump(out, fh)


if __name__ == "__main__":
    main()

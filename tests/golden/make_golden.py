"""Regenerate the golden fixtures in this directory from CM3D itself.

Run here (the reference tree must be present; the GPU box never runs this):

    make -C oracle ref
    python tests/golden/make_golden.py

For every case it writes a CM3D input deck (the reference's own test decks for
test/lj -- NVE and NVT -- and test/abutane, copied from the reference tree into a scratch
directory; generated decks for the synthetic workloads), runs
oracle/_ref/ref_dump (CM3D's startup + step_init + step, dumped at full
precision) and stores the result as <case>.npz.  Pair lists of the larger
cases are stored as a count plus a SHA-256 of the sorted (min, max) pairs.
"""
from __future__ import annotations

import hashlib
import os
import shutil
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from cm3d_b200 import configs  # noqa: E402
from oracle.dumpio import read_dump  # noqa: E402

REF = os.environ.get("CM3D_REF", "")   # the CM3D source tree (its test/ decks); main() requires it
DUMP = os.path.join(ROOT, "oracle", "_ref", "ref_dump")

LISTS = (("t", "inpt", "jnpt"), ("s", "inps", "jnps"),
         ("te", "inpte", "jnpte"), ("se", "inpse", "jnpse"))


def pair_key(i: np.ndarray, j: np.ndarray, n: int) -> np.ndarray:
    a = np.minimum(i, j).astype(np.int64)
    b = np.maximum(i, j).astype(np.int64)
    return np.sort(a * n + b)


def pair_hash(i: np.ndarray, j: np.ndarray, n: int) -> str:
    return hashlib.sha256(pair_key(i, j, n).tobytes()).hexdigest()


# big per-atom arrays kept only for the small cases
BULKY = {"f_lj_s", "f_el_s", "f_lj_short", "f_el_short", "acc_s", "acc_a",
         "acc_r", "final_acc_l"}


def convert(d: dict, full_lists: bool, keep_bulky: bool) -> dict:
    out = {}
    n = int(d["natoms"][0])
    for k, v in d.items():
        if k in {"inpt", "jnpt", "inps", "jnps", "inpte", "jnpte", "inpse", "jnpse"}:
            continue
        if k in BULKY and not keep_bulky:
            continue
        out[k] = v
    for tag, ik, jk in LISTS:
        if ik not in d:
            continue
        out[f"list_{tag}_hash"] = np.array(pair_hash(d[ik], d[jk], n))
        if full_lists:
            key = pair_key(d[ik], d[jk], n)
            out[f"list_{tag}_key"] = key
    return out


def run_case(name: str, workdir: str, infile: str, nsteps: int,
             full_lists: bool, keep_bulky: bool) -> None:
    bin_path = os.path.join(workdir, f"{name}.bin")
    with open(os.path.join(workdir, "ref_dump.log"), "w") as log:
        subprocess.run([DUMP, infile, bin_path, str(nsteps)], cwd=workdir,
                       stdout=log, stderr=subprocess.STDOUT, check=True)
    d = read_dump(bin_path)
    out = convert(d, full_lists, keep_bulky)
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
    print(f"{name}: natoms={int(d['natoms'][0])} nprt={int(d['nprt'][0])} "
          f"nprte={int(d['nprte'][0])} -> {name}.npz")


def copy_ref_test(sub: str, dst: str) -> None:
    src = os.path.join(REF, "test", sub)
    shutil.copytree(src, dst)
    for root, _dirs, files in os.walk(dst):
        for f in files:
            os.chmod(os.path.join(root, f), 0o644)


def main() -> None:
    if not REF or not os.path.isdir(REF):
        sys.exit("set CM3D_REF to the CM3D source tree")
    if not os.path.exists(DUMP):
        sys.exit("build the dump harness first: make -C oracle ref")
    with tempfile.TemporaryDirectory() as tmp:
        # CM3D's own regression decks
        d = os.path.join(tmp, "lj")
        copy_ref_test("lj", d)
        run_case("lj256", d, "lj.input_ljnve", 20, True, True)
        run_case("lj2", d, "lj.input_ljnve.2", 10, True, True)
        run_case("lj256nvt", d, "lj.input_ljnvt", 20, True, True)
        d = os.path.join(tmp, "abutane")
        copy_ref_test("abutane", d)
        run_case("abutane", d, "abutane.input", 20, True, True)
        # synthetic workloads in CM3D's formats
        cases = [
            ("argon864", configs.argon_fcc(ntime=20), 20, True, True),
            ("water216", configs.water_box(ngrid=6, ntime=20), 20, True, True),
            ("binary256", configs.charged_binary(natoms=256, ntime=10), 10, True, True),
            ("water4096", configs.water_box(ngrid=16, ntime=2), 2, False, False),
        ]
        for name, wl, nsteps, full, bulky in cases:
            d = os.path.join(tmp, name)
            infile = wl.write(d)
            run_case(name, d, os.path.basename(infile), nsteps, full, bulky)


if __name__ == "__main__":
    main()

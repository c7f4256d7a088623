"""Synthetic workloads written in CM3D's own input formats.

Every workload the engine is measured on is generated here, seeded, and can be
written out as a complete CM3D input deck (keyword file, ``~mol_def`` set file,
``~mol_name_def`` topology, ``~inter_parm``/``~bond_parm``/``~bend_parm``
parameter base and an ``istart{2}`` restart file holding positions *and*
velocities), so that CM3D itself and this engine start from bit-identical
initial conditions.

Formats follow CM3D's readers:
  keyword file      input/md_readsim.c, input/md_setsimkey.c
  set file          input/md_readset.c:46-48        (~mol_def)
  topology          input/md_getmols.c:48-51,162-165 (~mol_name_def, ~atom_def,
                                                     ~bond_def, ~bend_def)
  parameter base    input/md_getparm.c:73-143        (~inter_parm) and
                    input/md_searchbase.c            (~bond_parm, ~bend_parm)
  restart (istart 2) input/md_readpos.c:137-227

Units are CM3D's (include/md_numbers.h): energy in K, length in Angstrom,
time in ps, mass in amu*MCONV, charge in e*sqrt(CCONV).  Bond force constants
follow the 1/2 k (x - x0)^2 convention (energy/intra/md_fbond.c) and bend
equilibrium angles are given in degrees (input/md_searchbase.c:571).
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass, field

import numpy as np

# include/md_numbers.h
KCAL = 503.22289                      # K per kcal/mol
BOLTS = 1.38065812e-23
DCONV = BOLTS * 1.0e23
MCONV = 10.0 / (6.022045 * DCONV)     # g/mol -> K ps^2 / A^2
CCONV = 167102.4                      # e^2 -> K A
TCONV = 1.0e-3                        # fs -> ps (input/md_readsim.c:474)

# water model shared by the water configurations (flexible 3-site)
WATER = dict(q_o=-0.8476, q_h=0.4238, sig_oo=3.166, eps_oo=0.1553 * KCAL,
             m_o=15.9994, m_h=1.008, r0=1.0, k_bond=1059.0 * KCAL,
             theta0=109.47, k_bend=75.9 * KCAL)
WATER_SPACING = 49.66 / 16.0          # 1.0 g/cm^3 on a cubic molecular grid

ARGON = dict(sig=3.405, eps=0.2381 * KCAL, mass=39.948)


@dataclass
class Workload:
    """A complete, seeded simulation set-up in CM3D's vocabulary."""
    name: str
    keywords: dict                       # \keyword{value} pairs of the input file
    species: list                        # [(mol_name, nmol, topology text)]
    inter_parms: list                    # ~inter_parm texts
    bond_parms: list = field(default_factory=list)
    bend_parms: list = field(default_factory=list)
    pos: np.ndarray = None               # (N, 3) Angstrom
    vel: np.ndarray = None               # (N, 3) Angstrom / ps
    mass_amu: np.ndarray = None          # (N,)
    box: float = 0.0                     # cubic edge, Angstrom
    temp: float = 0.0
    dt_fs: float = 1.0
    therm_opt: str = "none"              # each species' \mol_therm_opt (nvt: "global")

    @property
    def natoms(self) -> int:
        return int(self.pos.shape[0])

    # ------------------------------------------------------------- writers
    def input_text(self) -> str:
        lines = [f"\\{k}{{{v}}}" for k, v in self.keywords.items()]
        return "\n".join(lines) + "\n"

    def set_text(self) -> str:
        out = []
        for idx, (mol, nmol, _top) in enumerate(self.species, start=1):
            out.append(f"~mol_def[\\mol_parm_file{{{mol}.top}} "
                       f"\\mol_therm_opt{{{self.therm_opt}}} \\nmol{{{nmol}}} "
                       f"\\mol_index{{{idx}}}]")
        return "\n".join(out) + "\n"

    def database_text(self) -> str:
        return "\n".join(self.inter_parms + self.bond_parms + self.bend_parms) + "\n"

    def restart_text(self) -> str:
        """istart{2} restart: header, averages, x v per atom, hmat, vvol9."""
        n = self.natoms
        dt_ps = self.dt_fs * TCONV
        rows = [f"0 {n} 0 0 0 {self.temp!r} 0 {dt_ps!r}",
                " ".join(["0"] * 8), " ".join(["0"] * 10), " ".join(["0"] * 5),
                " ".join(["0"] * 9)]
        fmt = "%.17g %.17g %.17g %.17g %.17g %.17g"
        for i in range(n):
            rows.append(fmt % (*self.pos[i], *self.vel[i]))
        L = self.box
        rows += [f"{L!r} 0 0", f"0 {L!r} 0", f"0 0 {L!r}"]
        rows += ["0 0 0"] * 3
        return "\n".join(rows) + "\n"

    def with_state(self, pos: np.ndarray, vel: np.ndarray) -> "Workload":
        """the same workload started from other positions and velocities"""
        import dataclasses
        return dataclasses.replace(self, pos=np.array(pos, dtype=float), vel=np.array(vel, dtype=float))

    def write(self, directory: str) -> str:
        """Write the full input deck; returns the keyword-file path."""
        os.makedirs(directory, exist_ok=True)
        for mol, _n, top in self.species:
            with open(os.path.join(directory, f"{mol}.top"), "w") as fh:
                fh.write(top)
        files = {f"{self.name}.input": self.input_text(),
                 f"{self.name}.set": self.set_text(),
                 "data_base": self.database_text(),
                 f"{self.name}.rest": self.restart_text()}
        for fn, txt in files.items():
            with open(os.path.join(directory, fn), "w") as fh:
                fh.write(txt)
        return os.path.join(directory, f"{self.name}.input")


def _base_keywords(name: str, dt_fs: float, temp: float, ntime: int) -> dict:
    return {
        "calculation": "md", "ensemble": "nve", "istart": 2, "ntime": ntime,
        "iperd": 3, "dt": dt_fs, "t_ext": temp,
        "iwr_screen": max(ntime, 1), "iwr_dump": 0, "iwr_inst": 0,
        "iwr_confp": 0, "iwr_confv": 0,
        "dpi_file": f"{name}.rest", "dpo_file": f"{name}.save",
        "ham_file": f"{name}.ham", "eng_file": f"{name}.eng",
        "eval_file": f"{name}.eval", "pos_file": f"{name}.conf",
        "vel_file": f"{name}.vel", "mol_set_file": f"{name}.set",
        "inter_file": "data_base", "bond_file": "data_base",
        "bend_file": "data_base", "torsion_file": "data_base",
        "onefour_file": "data_base",
    }


def maxwell_boltzmann(mass_amu: np.ndarray, temp: float, rng) -> np.ndarray:
    """Gaussian velocities, net momentum removed, rescaled to exactly `temp`
    with ndof = 3N - 3 (CM3D's samvel/zerotm/scale, integrate/md_zeroam.c:33-47)."""
    n = mass_amu.shape[0]
    m = mass_amu * MCONV
    v = rng.standard_normal((n, 3)) * np.sqrt(temp / m)[:, None]
    v -= (m[:, None] * v).sum(0) / m.sum()
    ndof = max(3 * n - 3, 1)
    t_now = float((m[:, None] * v * v).sum()) / ndof
    if t_now > 0:
        v *= math.sqrt(temp / t_now)
    return v


def _lj_parm(a: str, b: str, eps: float, sig: float, rmin: float,
             rmax: float, rres: float) -> str:
    return (f"~inter_parm[\\atom1{{{a}}}\\atom2{{{b}}}\\pot_type{{lennard-jones}}"
            f"\\eps{{{eps!r}}}\\sig{{{sig!r}}}\\min_dist{{{rmin!r}}}"
            f"\\max_dist{{{rmax!r}}}\\res_dist{{{rres!r}}}]")


def _null_parm(a: str, b: str) -> str:
    return f"~inter_parm[\\atom1{{{a}}}\\atom2{{{b}}}\\pot_type{{null}}]"


# ----------------------------------------------------------------- argon
def argon_fcc(ncell: int = 6, density: float = 0.8442, temp: float = 120.0,
              seed: int = 1, rc_sigma: float = 2.5, skin_sigma: float = 0.3,
              dt_fs: float = 5.0, ntime: int = 1000, name: str = "argon",
              nvt_chain: int = 0, npt: str = "", p_ext: float = 1.0) -> Workload:
    """LJ argon on an FCC lattice, reduced density `density`; cut and shifted
    LJ at `rc_sigma` sigma; Verlet list with a `skin_sigma` sigma skin.
    nvt_chain > 0: CM3D's NVT with one global Nose-Hoover chain of that
    length at `temp` (keywords ensemble nvt and len_nhc, each species'
    mol_therm_opt global).  npt "npt_i" or "npt_f": CM3D's barostat at
    `p_ext` (keyword p_ext) with a chain of 3 on the volume (nbar) next to
    the thermostat chain (length nvt_chain, 3 if not given)."""
    sig, eps, mass = ARGON["sig"], ARGON["eps"], ARGON["mass"]
    n = 4 * ncell ** 3
    L = (n / density) ** (1.0 / 3.0) * sig
    a = L / ncell
    basis = np.array([[0, 0, 0], [0.5, 0.5, 0], [0.5, 0, 0.5], [0, 0.5, 0.5]])
    cells = np.array([(i, j, k) for i in range(ncell) for j in range(ncell)
                      for k in range(ncell)], dtype=float)
    pos = ((cells[:, None, :] + basis[None, :, :] + 0.25) * a).reshape(-1, 3)
    rng = np.random.default_rng(seed)
    m = np.full(n, mass)
    vel = maxwell_boltzmann(m, temp, rng)
    rc = rc_sigma * sig
    kw = _base_keywords(name, dt_fs, temp, ntime)
    kw.update({"skin": skin_sigma * sig, "shift": 1, "nres_lrf": 1,
               "nres_intra": 1, "nres_tors": 1, "neighbor_list": "verlist"})
    if npt:
        nvt_chain = nvt_chain or 3
        kw.update({"ensemble": npt, "len_nhc": nvt_chain, "nbar": 3, "p_ext": p_ext})
    elif nvt_chain > 0:
        kw.update({"ensemble": "nvt", "len_nhc": nvt_chain})
    top = (f"~mol_name_def[\\mol_name{{argon}}\\natom{{1}}\\nbond{{0}}]\n"
           f"~atom_def[\\atom_typ{{ar}}\\atom_ind{{1}}\\mass{{{mass!r}}}\\charge{{0}}]\n")
    return Workload(name=name, keywords=kw, species=[("argon", n, top)],
                    therm_opt="global" if nvt_chain > 0 else "none",
                    inter_parms=[_lj_parm("ar", "ar", eps, sig, 0.55 * sig, rc, rc)],
                    pos=pos, vel=vel, mass_amu=m, box=L, temp=temp, dt_fs=dt_fs)


# ----------------------------------------------------------------- water
def _random_rotations(n: int, rng) -> np.ndarray:
    q = rng.standard_normal((n, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    w, x, y, z = q.T
    return np.stack([
        np.stack([1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)], -1),
        np.stack([2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)], -1),
        np.stack([2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)], -1),
    ], 1)


def water_box(ngrid: int = 16, temp: float = 300.0, seed: int = 1,
              rc: float | None = None, alpha: float = 0.31, kmax: int = 7,
              skin: float = 0.5, dt_fs: float = 2.0, nres_intra: int = 4,
              ntime: int = 1000, ntable: int = 500, name: str = "water",
              placement: str = "checkerboard") -> Workload:
    """Flexible 3-site water: ngrid^3 molecules on a cubic grid at 1.0 g/cm^3
    with seeded random orientations.  Ewald with `alpha` and a spherical
    k-space cutoff `kmax` (CM3D's kmax keyword, md_ewald.c:93-114).
    `placement` is how orientations with close intermolecular contacts are
    re-drawn: "checkerboard" (half of the clashing molecules per sweep, at
    most 200 sweeps; the decks of the test fixtures) or "octant" (one parity
    class at a time until clear; converges in a few rounds, used for large
    grids)."""
    w = WATER
    nmol = ngrid ** 3
    L = ngrid * WATER_SPACING
    if rc is None:
        rc = min(10.0, 0.45 * L)
    rng = np.random.default_rng(seed)
    grid = np.array([(i, j, k) for i in range(ngrid) for j in range(ngrid)
                     for k in range(ngrid)], dtype=float)
    o = (grid + 0.5) * WATER_SPACING
    half = math.radians(w["theta0"]) / 2.0
    h1 = np.array([math.sin(half), 0.0, math.cos(half)]) * w["r0"]
    h2 = np.array([-math.sin(half), 0.0, math.cos(half)]) * w["r0"]
    R = _random_rotations(nmol, rng)
    pos = np.empty((nmol, 3, 3))
    pos[:, 0] = o
    pos[:, 1] = o + R @ h1
    pos[:, 2] = o + R @ h2
    # re-draw the orientation of any molecule with an intermolecular contact
    # closer than `min_contact` to a grid neighbour, so the start is not a
    # high-energy overlap (random orientations on a 3.1 A grid otherwise put
    # some H atoms within 1 A of each other)
    min_contact = 1.9
    g = pos.reshape(ngrid, ngrid, ngrid, 3, 3)
    offs = np.array([(dx, dy, dz) for dx in (-1, 0, 1) for dy in (-1, 0, 1) for dz in (-1, 0, 1)
                     if (dx, dy, dz) != (0, 0, 0)])

    def clashes(cells: np.ndarray) -> np.ndarray:
        # closest intermolecular contact of the molecules at grid `cells`
        # (k, 3) with their 26 grid neighbours, below min_contact?
        out = np.zeros(cells.shape[0], dtype=bool)
        for k0 in range(0, cells.shape[0], 65536):
            c = cells[k0:k0 + 65536]
            mine = g[c[:, 0], c[:, 1], c[:, 2]]                   # (k, 3, 3)
            r = np.full(c.shape[0], np.inf)
            for o in offs:
                nb = (c + o) % ngrid
                d = mine[:, :, None, :] - g[nb[:, 0], nb[:, 1], nb[:, 2]][:, None, :, :]
                d -= L * np.round(d / L)
                r = np.minimum(r, np.sqrt((d * d).sum(-1)).min(axis=(-1, -2)))
            out[k0:k0 + 65536] = r < min_contact
        return out

    stencil = np.vstack([np.zeros((1, 3), int), offs])

    def redraw(sel: np.ndarray) -> None:
        Rn = _random_rotations(sel.shape[0], rng)
        oo = g[sel[:, 0], sel[:, 1], sel[:, 2], 0]
        g[sel[:, 0], sel[:, 1], sel[:, 2], 1] = oo + Rn @ h1
        g[sel[:, 0], sel[:, 1], sel[:, 2], 2] = oo + Rn @ h2

    def around(sel: np.ndarray) -> np.ndarray:
        # the molecules at `sel` and their grid neighbours, each once
        near = ((sel[:, None, :] + stencil[None, :, :]) % ngrid).reshape(-1, 3)
        key = np.unique((near[:, 0] * ngrid + near[:, 1]) * ngrid + near[:, 2])
        return np.stack([key // (ngrid * ngrid), (key // ngrid) % ngrid, key % ngrid], axis=1)

    every = np.argwhere(np.ones((ngrid, ngrid, ngrid), dtype=bool))
    bad = clashes(every).reshape(ngrid, ngrid, ngrid)
    if placement == "octant":
        # Grid neighbours differ in the class of at least one coordinate --
        # its parity, with the last layer of an odd grid a class of its own
        # (it touches layer 0 through the periodic boundary) -- so the
        # molecules of one class can be re-drawn together against fixed
        # neighbours; each class is re-drawn until it is clear, then the
        # next, for a few rounds.
        nv = 2 if ngrid % 2 == 0 else 3
        coord_cls = np.arange(ngrid) % 2
        if nv == 3:
            coord_cls[ngrid - 1] = 2
        for _round in range(20):
            if not bad.any():
                break
            for cls in range(nv ** 3):
                par = np.array([cls // (nv * nv), (cls // nv) % nv, cls % nv])
                moved = []
                for _try in range(50):
                    idx = np.argwhere(bad)
                    sel = idx[(coord_cls[idx] == par).all(axis=1)]
                    if sel.shape[0] == 0:
                        break
                    redraw(sel)
                    moved.append(sel)
                    bad[sel[:, 0], sel[:, 1], sel[:, 2]] = clashes(sel)
                if moved:
                    near = around(np.concatenate(moved))
                    bad[near[:, 0], near[:, 1], near[:, 2]] = clashes(near)
    else:
        for _sweep in range(200):
            if not bad.any():
                break
            idx = np.argwhere(bad)
            # re-draw only a checkerboard subset per sweep so neighbours that
            # clash with each other do not both move at once
            sel = idx[(idx.sum(1) + _sweep) % 2 == 0]
            if sel.shape[0] == 0:
                sel = idx[:1]
            redraw(sel)
            # only the re-drawn molecules and their neighbours can change state
            near = around(sel)
            bad[near[:, 0], near[:, 1], near[:, 2]] = clashes(near)
    pos = g.reshape(-1, 3)
    m = np.tile([w["m_o"], w["m_h"], w["m_h"]], nmol)
    vel = maxwell_boltzmann(m, temp, rng)
    kw = _base_keywords(name, dt_fs, temp, ntime)
    kw.update({"skin": skin, "nres_lrf": 1, "nres_intra": nres_intra,
               "nres_tors": 1, "alp_ewald": alpha, "kmax": kmax,
               "rcute_max": rc, "rcute_resp": rc, "rcute_min": 1.0,
               "ntable": ntable, "neighbor_list": "verlist"})
    top = ("~mol_name_def[\\mol_name{water}\\natom{3}\\nbond{2}\\nbend{1}]\n"
           f"~atom_def[\\atom_typ{{ow}}\\atom_ind{{1}}\\mass{{{w['m_o']!r}}}"
           f"\\charge{{{w['q_o']!r}}}]\n"
           f"~atom_def[\\atom_typ{{hw}}\\atom_ind{{2}}\\mass{{{w['m_h']!r}}}"
           f"\\charge{{{w['q_h']!r}}}]\n"
           f"~atom_def[\\atom_typ{{hw}}\\atom_ind{{3}}\\mass{{{w['m_h']!r}}}"
           f"\\charge{{{w['q_h']!r}}}]\n"
           "~bond_def[\\atom1{1}\\atom2{2}]\n~bond_def[\\atom1{1}\\atom2{3}]\n"
           "~bend_def[\\atom1{2}\\atom2{1}\\atom3{3}]\n")
    inter = [_lj_parm("ow", "ow", w["eps_oo"], w["sig_oo"], 1.8, rc, rc),
             _null_parm("ow", "hw"), _null_parm("hw", "hw")]
    bonds = [f"~bond_parm[\\atom1{{ow}}\\atom2{{hw}}\\pot_type{{harm}}"
             f"\\fk{{{w['k_bond']!r}}}\\eq{{{w['r0']!r}}}]"]
    bends = [f"~bend_parm[\\atom1{{hw}}\\atom2{{ow}}\\atom3{{hw}}\\pot_type{{harm}}"
             f"\\fk{{{w['k_bend']!r}}}\\eq{{{w['theta0']!r}}}]"]
    return Workload(name=name, keywords=kw, species=[("water", nmol, top)],
                    inter_parms=inter, bond_parms=bonds, bend_parms=bends,
                    pos=pos, vel=vel, mass_amu=m, box=L, temp=temp, dt_fs=dt_fs)


# ------------------------------------------------------ charged LJ binary
def charged_binary(natoms: int = 256, density: float = 0.75, tstar: float = 1.0,
                   seed: int = 1, charge: float = 0.5, kmax: int = 5,
                   dt_fs: float = 5.0, ntime: int = 2000,
                   name: str = "binary") -> Workload:
    """Equimolar charged LJ binary mixture (argon LJ parameters, charges
    +/- `charge` e) on an FCC start; rc = min(2.5 sigma, 0.45 L),
    Ewald alpha = 3.2 / rc, spherical kmax."""
    sig, eps, mass = ARGON["sig"], ARGON["eps"], ARGON["mass"]
    ncell = max(1, int(round((natoms / 4) ** (1.0 / 3.0))))
    n = 4 * ncell ** 3
    L = (n / density) ** (1.0 / 3.0) * sig
    a = L / ncell
    basis = np.array([[0, 0, 0], [0.5, 0.5, 0], [0.5, 0, 0.5], [0, 0.5, 0.5]])
    cells = np.array([(i, j, k) for i in range(ncell) for j in range(ncell)
                      for k in range(ncell)], dtype=float)
    pos = ((cells[:, None, :] + basis[None, :, :] + 0.25) * a).reshape(-1, 3)
    temp = tstar * eps
    rng = np.random.default_rng(seed)
    m = np.full(n, mass)
    vel = maxwell_boltzmann(m, temp, rng)
    rc = min(2.5 * sig, 0.45 * L)
    alpha = 3.2 / rc
    skin = 0.3 * sig
    kw = _base_keywords(name, dt_fs, temp, ntime)
    kw.update({"skin": skin, "nres_lrf": 1, "nres_intra": 1, "nres_tors": 1,
               "alp_ewald": alpha, "kmax": kmax, "rcute_max": rc,
               "rcute_resp": rc, "rcute_min": 1.0, "shift": 1,
               "neighbor_list": "verlist"})
    # one "molecule" per atom; the two species alternate so that the
    # mixture is equimolar and both species sit on every sublattice
    topa = (f"~mol_name_def[\\mol_name{{cat}}\\natom{{1}}\\nbond{{0}}]\n"
            f"~atom_def[\\atom_typ{{ca}}\\atom_ind{{1}}\\mass{{{mass!r}}}"
            f"\\charge{{{charge!r}}}]\n")
    topb = (f"~mol_name_def[\\mol_name{{ani}}\\natom{{1}}\\nbond{{0}}]\n"
            f"~atom_def[\\atom_typ{{an}}\\atom_ind{{1}}\\mass{{{mass!r}}}"
            f"\\charge{{{-charge!r}}}]\n")
    perm = rng.permutation(n)
    pos = pos[perm]
    inter = [_lj_parm("ca", "ca", eps, sig, 0.55 * sig, rc, rc),
             _lj_parm("an", "an", eps, sig, 0.55 * sig, rc, rc),
             _lj_parm("an", "ca", eps, sig, 0.55 * sig, rc, rc)]
    return Workload(name=name, keywords=kw,
                    species=[("cat", n // 2, topa), ("ani", n - n // 2, topb)],
                    inter_parms=inter, pos=pos, vel=vel, mass_amu=m, box=L,
                    temp=temp, dt_fs=dt_fs)


# ------------------------------------------- uneven ensemble of small boxes
def _fcc_sites(natoms: int, rng) -> tuple[np.ndarray, int]:
    """`natoms` sites of the smallest FCC lattice (4 ncell^3 sites) that holds
    them, as fractional coordinates; a seeded choice of sites when the lattice
    has more than needed (vacancies spread through the box)."""
    ncell = max(1, int(math.ceil((natoms / 4.0) ** (1.0 / 3.0) - 1e-9)))
    basis = np.array([[0, 0, 0], [0.5, 0.5, 0], [0.5, 0, 0.5], [0, 0.5, 0.5]])
    cells = np.array([(i, j, k) for i in range(ncell) for j in range(ncell)
                      for k in range(ncell)], dtype=float)
    sites = ((cells[:, None, :] + basis[None, :, :] + 0.25) / ncell).reshape(-1, 3)
    if sites.shape[0] > natoms:
        keep = np.sort(rng.choice(sites.shape[0], natoms, replace=False))
        sites = sites[keep]
    return sites, ncell


def lj_box(natoms: int, density: float, tstar: float, seed: int, charged: bool = False,
           charge: float = 0.5, kmax: int = 5, dt_fs: float = 5.0, ntime: int = 2000,
           name: str = "ljbox") -> Workload:
    """One box of the uneven ensemble: `natoms` argon-parameter LJ atoms at
    reduced density `density` and reduced temperature `tstar` on an FCC start,
    rc = min(2.5 sigma, 0.45 L) with a 0.3 sigma skin.  `charged`: an
    equimolar binary mixture with charges +/- `charge` e (natoms rounded down
    to even), Ewald alpha = 3.2 / rc and a spherical kmax."""
    sig, eps, mass = ARGON["sig"], ARGON["eps"], ARGON["mass"]
    if charged and natoms % 2:
        natoms -= 1
    rng = np.random.default_rng(seed)
    L = (natoms / density) ** (1.0 / 3.0) * sig
    frac, _ = _fcc_sites(natoms, rng)
    pos = frac * L
    temp = tstar * eps
    m = np.full(natoms, mass)
    vel = maxwell_boltzmann(m, temp, rng)
    rc = min(2.5 * sig, 0.45 * L)
    skin = 0.3 * sig
    kw = _base_keywords(name, dt_fs, temp, ntime)
    kw.update({"skin": skin, "shift": 1, "nres_lrf": 1, "nres_intra": 1,
               "nres_tors": 1, "neighbor_list": "verlist"})
    if not charged:
        top = (f"~mol_name_def[\\mol_name{{argon}}\\natom{{1}}\\nbond{{0}}]\n"
               f"~atom_def[\\atom_typ{{ar}}\\atom_ind{{1}}\\mass{{{mass!r}}}\\charge{{0}}]\n")
        return Workload(name=name, keywords=kw, species=[("argon", natoms, top)],
                        inter_parms=[_lj_parm("ar", "ar", eps, sig, 0.55 * sig, rc, rc)],
                        pos=pos, vel=vel, mass_amu=m, box=L, temp=temp, dt_fs=dt_fs)
    kw.update({"alp_ewald": 3.2 / rc, "kmax": kmax, "rcute_max": rc, "rcute_resp": rc,
               "rcute_min": 1.0})
    topa = (f"~mol_name_def[\\mol_name{{cat}}\\natom{{1}}\\nbond{{0}}]\n"
            f"~atom_def[\\atom_typ{{ca}}\\atom_ind{{1}}\\mass{{{mass!r}}}"
            f"\\charge{{{charge!r}}}]\n")
    topb = (f"~mol_name_def[\\mol_name{{ani}}\\natom{{1}}\\nbond{{0}}]\n"
            f"~atom_def[\\atom_typ{{an}}\\atom_ind{{1}}\\mass{{{mass!r}}}"
            f"\\charge{{{-charge!r}}}]\n")
    pos = pos[rng.permutation(natoms)]
    inter = [_lj_parm("ca", "ca", eps, sig, 0.55 * sig, rc, rc),
             _lj_parm("an", "an", eps, sig, 0.55 * sig, rc, rc),
             _lj_parm("an", "ca", eps, sig, 0.55 * sig, rc, rc)]
    return Workload(name=name, keywords=kw,
                    species=[("cat", natoms // 2, topa), ("ani", natoms // 2, topb)],
                    inter_parms=inter, pos=pos, vel=vel, mass_amu=m, box=L, temp=temp,
                    dt_fs=dt_fs)


@dataclass
class EnsembleMember:
    """One box of an ensemble, with the draws it was generated from."""
    index: int
    natoms: int
    density: float
    tstar: float
    charged: bool
    seed: int


def ensemble_plan(nsys: int = 1024, seed: int = 2024, nmin: int = 64, nmax: int = 4096,
                  frac_charged: float = 0.25) -> list[EnsembleMember]:
    """The draws of the uneven ensemble: N log-uniform in [nmin, nmax],
    reduced density U(0.6, 0.9), reduced temperature U(0.7, 1.5), a per-box
    seed, and exactly round(frac_charged * nsys) charged binary boxes."""
    rng = np.random.default_rng(seed)
    ncharged = int(round(frac_charged * nsys))
    charged = np.zeros(nsys, bool)
    charged[rng.permutation(nsys)[:ncharged]] = True
    out = []
    for k in range(nsys):
        n = int(round(math.exp(rng.uniform(math.log(nmin), math.log(nmax)))))
        rho = float(rng.uniform(0.6, 0.9))
        ts = float(rng.uniform(0.7, 1.5))
        sd = int(rng.integers(1, 2 ** 31 - 1))
        out.append(EnsembleMember(k, n, rho, ts, bool(charged[k]), sd))
    return out


def ensemble(nsys: int = 1024, seed: int = 2024, ntime: int = 2000, **kw) -> list[Workload]:
    """The uneven ensemble as Workloads (argon-parameter LJ and charged binary
    boxes, FCC start, dt 5 fs, kmax 5 for the charged ones)."""
    return [lj_box(m.natoms, m.density, m.tstar, m.seed, charged=m.charged, ntime=ntime,
                   name=f"box{m.index:04d}")
            for m in ensemble_plan(nsys, seed, **kw)]


# ------------------------------------------------------ serving job stream
@dataclass
class ServingRequest:
    """One water-box MD request of the serving workload."""
    index: int
    arrival: float          # seconds
    ngrid: int              # ngrid^3 molecules
    nsteps: int
    seed: int


def serving_plan(rate: float, duration: float, seed: int = 11, mol_min: int = 256, mol_max: int = 16384,
                 steps_min: int = 500, steps_max: int = 5000) -> list[ServingRequest]:
    """Poisson arrivals at `rate` jobs/s over `duration` s; molecule count
    log-uniform in [mol_min, mol_max] (rounded to a cubic grid), step count
    uniform in [steps_min, steps_max]."""
    rng = np.random.default_rng(seed)
    out, t = [], 0.0
    while True:
        t += float(rng.exponential(1.0 / rate))
        if t > duration:
            break
        nmol = math.exp(rng.uniform(math.log(mol_min), math.log(mol_max)))
        ngrid = max(2, int(round(nmol ** (1.0 / 3.0))))
        out.append(ServingRequest(len(out), t, ngrid, int(rng.integers(steps_min, steps_max + 1)),
                                  int(rng.integers(1, 2 ** 31 - 1))))
    return out


def serving_workload(req: ServingRequest) -> Workload:
    """The water box of a request: 1.0 g/cm^3, rc = min(10 A, 0.45 L),
    Ewald alpha = 3.1 / rc, kmax = ceil(7 L / 49.66), RESPA 0.5/2 fs."""
    L = req.ngrid * WATER_SPACING
    rc = min(10.0, 0.45 * L)
    return water_box(ngrid=req.ngrid, seed=req.seed, rc=rc, alpha=3.1 / rc,
                     kmax=int(math.ceil(7.0 * L / 49.66)), ntime=req.nsteps, placement="octant",
                     name=f"job{req.index:04d}")


def read_restart(path: str) -> tuple[np.ndarray, np.ndarray]:
    """positions and velocities (N, 3) from a CM3D restart file
    (output/md_writestart.c:31-80: five header lines, then x y z vx vy vz
    per atom)"""
    with open(path) as fh:
        lines = fh.read().splitlines()
    n = int(lines[0].split()[1])
    rows = np.array([[float(v) for v in ln.split()[:6]] for ln in lines[5:5 + n]])
    return rows[:, :3].copy(), rows[:, 3:].copy()

"""NVE energy conservation: the drift of CM3D's conserved energy.

CM3D's conserved quantity of an NVE run is ham = poth + potra + zke
(integrate/md_averages.new.c:100, the NVE terms): the shifted intermolecular
energy (the LJ sum shifted at the cut-off, electrostatics, reciprocal space
and the long-range correction), the intramolecular energy and the kinetic
energy.  CM3D itself reports <dE> = std(ham) / |mean(ham)| over a run
(output/md_writescreen.c:384-387); the drift here is the least-squares slope
of ham against simulated time, per atom and per nanosecond, in CM3D's energy
unit (K).
"""
from __future__ import annotations

import numpy as np


def conserved(en: dict) -> float:
    """ham of one energies record (NVE: no thermostat or barostat terms)"""
    return float(en["poth"] + en["potra"] + en["zke"])


def drift_stats(ham, dt_ps: float, natoms: int) -> dict:
    """slope of ham(t) per atom per ns (least squares over the steps, with
    its standard error), and CM3D's <dE> fluctuation measure"""
    ham = np.asarray(ham, dtype=float)
    t = np.arange(1, ham.size + 1) * dt_ps
    A = np.stack([t, np.ones_like(t)], axis=1)
    coef, res, *_ = np.linalg.lstsq(A, ham, rcond=None)
    slope = float(coef[0])
    n = ham.size
    resid = ham - A @ coef
    s2 = float(resid @ resid) / max(n - 2, 1)
    se = float(np.sqrt(s2 / max(((t - t.mean()) ** 2).sum(), 1e-300)))
    mean = float(ham.mean())
    return {"steps": int(n), "dt_ps": dt_ps, "natoms": natoms,
            "drift_per_atom_per_ns": slope * 1e3 / natoms,
            "drift_se_per_atom_per_ns": se * 1e3 / natoms,
            "dE_cm3d": float(ham.std(ddof=1) / abs(mean)) if n > 1 and mean != 0 else None,
            "ham_first": float(ham[0]), "ham_last": float(ham[-1]), "ham_mean": mean,
            "unit": "K per atom per ns (CM3D's energy unit)"}


def engine_series(system, mode: int, nsteps: int, device: int = 0, use_graph: bool = True) -> list:
    """ham after each of `nsteps` outer steps of the engine from the
    system's initial state (step_init, then one step at a time)"""
    from .engine import Engine
    e = Engine(system, mode=mode, device=device, use_graph=use_graph)
    try:
        e.step_init()
        out = []
        for k in range(nsteps):
            e.step(1 + k, 1)
            out.append(conserved(e.energies()))
        return out
    finally:
        e.close()

"""Sharding independent systems over ranks (one GPU per rank).

The systems of a batch or the jobs of a serving stream never interact, so a
multi-GPU run gives every rank a subset of whole systems and no collective
touches the step path: each rank steps its own batch; results and timings
are gathered once at the end (torch.distributed over NCCL, or gloo on CPU).

The subsets come from a greedy longest-processing-time packing on a cost
model of one outer step of a system: its pair work (the atoms' list sphere
populations, ~ N * rho * 4/3 pi r_list^3 / 2 unique pairs) plus its
reciprocal-space work (K k-vectors times its N_q charged atoms, weighted by
the relative cost of a phase step against a pair).
"""
from __future__ import annotations

import heapq
import math

import numpy as np

PAIR_COST = 1.0            # one unique listed pair
KSPACE_COST = 0.35         # one (k-vector, charged atom) phase step


def system_cost(system) -> float:
    """Work of one outer step of `system` (cm3d_b200.system.System) in
    pair units."""
    n = int(system.natoms)
    h = np.asarray(system["hmat"], float).reshape(3, 3)
    vol = abs(float(np.linalg.det(h)))
    r2 = float(np.max(system["rmaxl_skin2"])) if system["ninter"] > 0 else 0.0
    ktot = int(system.get("ktot", 0))
    nq = int(np.count_nonzero(np.asarray(system["qch"]))) if ktot else 0
    if nq:
        r2 = max(r2, float(system.get("rmaxl_skin2_e", 0.0)))
    pairs = 0.5 * n * min(n - 1, n / vol * 4.0 / 3.0 * math.pi * r2 ** 1.5)
    return PAIR_COST * pairs + KSPACE_COST * ktot * nq + 1.0


def partition(costs, nranks: int) -> list[list[int]]:
    """Greedy LPT packing of items with `costs` into `nranks` bins: items in
    decreasing cost, each to the currently lightest bin (ties: lowest rank).
    Returns each rank's item indices in increasing order.  Deterministic, so
    every rank computes the same plan without communicating."""
    if nranks < 1:
        raise ValueError("nranks must be >= 1")
    order = sorted(range(len(costs)), key=lambda k: (-float(costs[k]), k))
    heap = [(0.0, r) for r in range(nranks)]
    out = [[] for _ in range(nranks)]
    for k in order:
        load, r = heapq.heappop(heap)
        out[r].append(k)
        heapq.heappush(heap, (load + float(costs[k]), r))
    return [sorted(v) for v in out]


def imbalance(costs, parts) -> float:
    """max rank load / mean rank load (1.0 = perfect)"""
    loads = [sum(float(costs[k]) for k in p) for p in parts]
    mean = sum(loads) / len(loads)
    return max(loads) / mean if mean > 0 else 1.0

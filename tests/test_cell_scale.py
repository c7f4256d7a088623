"""The cell-size choice of cm3d_b200.engine.tune_cell_scale (host logic, no
GPU): the fastest step wins; steps within 2% of it count as a tie, broken by
the faster pair kernel and then the faster step."""
from cm3d_b200.engine import pick_cell_scale


def cand(step, pair):
    return {"ms_per_step": step, "pair_ms": pair}


def test_fastest_step_wins_outside_the_tie():
    c = {1.0: cand(7.58, 0.64), 1.25: cand(7.30, 1.16)}
    assert pick_cell_scale(c) == 1.25


def test_tie_goes_to_the_faster_pair_kernel():
    c = {1.0: cand(7.62, 0.64), 1.25: cand(7.59, 1.16)}
    assert pick_cell_scale(c) == 1.0


def test_tie_on_pair_time_goes_to_the_faster_step():
    c = {1.0: cand(1.610, 0.656), 1.25: cand(1.600, 0.656)}
    assert pick_cell_scale(c) == 1.25


def test_single_candidate_and_tie_width():
    assert pick_cell_scale({1.0: cand(2.0, 1.0)}) == 1.0
    c = {1.0: cand(1.00, 0.5), 1.25: cand(1.04, 0.1)}
    assert pick_cell_scale(c) == 1.0
    assert pick_cell_scale(c, tie=0.05) == 1.25

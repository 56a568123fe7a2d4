"""The batch schedule tuner (psipm_b200.batch.autotune) without a GPU.

A timing model stands in for the device: an LP of m rows takes m * 1e-6 s
when it has the whole grid and longer on a smaller share, and LPs in flight
overlap up to a saturation point, so the model has one best schedule; the
tuner must find it, time every candidate on the same spread-out sample, and
break ties towards fewer LPs in flight.
"""

import pytest

from psipm_b200.batch import BatchResult, autotune, schedule_candidates


class _LP:
    def __init__(self, m):
        self.m = m


def _model(best_workers, sms=148):
    full = 4 * sms

    def run(sub, workers, grid_blocks):
        blocks = full if grid_blocks == 0 else grid_blocks
        slow = max(1.0, full / (blocks * workers))  # a smaller share runs longer
        overlap = min(workers, best_workers) - 0.1 * max(0, workers - best_workers)
        work = sum(lp.m for lp in sub) * 1e-6 * slow * workers / max(0.5, overlap) / workers
        secs = work / max(1.0, min(workers, best_workers))
        return BatchResult(secs, [secs] * len(sub), ["optimal"] * len(sub), [0.0] * len(sub), [0] * len(sub),
                           workers)
    return run


def test_candidates_cover_powers_of_two_with_grid_shares():
    c = schedule_candidates(148, max_workers=8)
    assert (1, 0) in c
    assert [w for w, _ in c] == sorted(w for w, _ in c)
    assert {w for w, _ in c} == {1, 2, 4, 8}
    for w, g in c:
        assert w == 1 or 8 <= g <= 4 * 148 // w


@pytest.mark.parametrize("best", [1, 4, 8])
def test_tuner_finds_the_model_optimum(best):
    lps = [_LP(500 + 37 * k) for k in range(64)]
    seen = []

    def run(sub, workers, grid_blocks):
        seen.append([lp.m for lp in sub])
        return _model(best)(sub, workers, grid_blocks)

    sched = autotune(lps, sample=16, candidates=schedule_candidates(148, max_workers=8), run=run)
    assert sched.workers == best
    assert len(sched.trials) == len(schedule_candidates(148, max_workers=8))
    assert all(s == seen[0] for s in seen)  # every candidate timed on the same sample
    assert len(seen[0]) == 16 and seen[0][0] == 500 and seen[0][-1] > 500 + 37 * 48


def test_tie_goes_to_fewer_workers():
    lps = [_LP(1000)] * 8

    def flat(sub, workers, grid_blocks):
        return BatchResult(1.0, [1.0] * len(sub), ["optimal"] * len(sub), [0.0] * len(sub), [0] * len(sub),
                           workers)

    assert autotune(lps, candidates=[(1, 0), (2, 296), (4, 148)], run=flat).workers == 1


def test_empty_batch_is_an_error():
    with pytest.raises(ValueError):
        autotune([], candidates=[(1, 0)], run=lambda *a: None)

"""Straddling ties in the core selection, on the device.

At the start of a network LP the reference factors with theta = 1
(psipm_active_pool.py:4166, 4186), so every arc's leverage score depends only
on the degrees of its two end nodes and long runs of equal scores are
certain.  The reference picks with np.argpartition
(psipm_stable_preconditioner.py:97-110), whose choice among equal scores that
straddle the cut depends on NumPy's build; this library takes the equal
scores by ascending candidate index and counts every selection whose cut
fell inside such a run (psipm_tie_info).  These tests build that case on the
20 x 25 grid network and check that the device detects it and that its core
is exactly the documented (score descending, index ascending) rule applied
to the device's own, bit-exact scores.
"""

import numpy as np
import pytest

from _helpers import OPTIONS, lp_from

pytestmark = pytest.mark.gpu


def _rule_top(scores, allowed, count):
    """Indices (into scores) of the `count` best allowed entries by
    (score desc, index asc)."""
    idx = np.flatnonzero(allowed & np.isfinite(scores))
    order = np.lexsort((idx, -scores[idx]))
    return idx[order[:count]]


def test_first_refresh_of_a_network_straddles_a_tie_and_follows_the_index_rule(golden):
    from oracle import stable as OS
    from psipm_b200.kkt import GpuSpectralStableColumnPreconditioner

    lp = lp_from(golden("grid_20x25"))
    gpu = GpuSpectralStableColumnPreconditioner(lp.A, protected=~lp.pos, **OPTIONS)
    orc = OS.SpectralOracle(lp.A, protected=~lp.pos, **OPTIONS)
    try:
        ones = np.ones(lp.A.shape[1])
        gpu.factorize(ones, 1.0)  # the starting point's factorisation
        info = gpu.dev.tie_info()
        assert info["straddles"] >= 1, f"no straddling tie detected: {info}"
        assert info["tied"] > info["slots"] > 0
        assert gpu.tie_straddles == info["straddles"]
        # the device scores are the oracle's, bit for bit
        scores = gpu._scores()
        assert np.array_equal(scores, orc._scores(1.0 / ones, 1.0))
        values, counts = np.unique(scores, return_counts=True)
        assert counts.max() > 1
        # documented rule on the first refresh: mandatory columns, then the best of the rest
        cand = gpu.candidates
        mandatory_local = np.searchsorted(cand, gpu.mandatory)
        target = min(gpu.core_target, cand.size)
        allowed = np.ones(cand.size, dtype=bool)
        allowed[mandatory_local] = False
        picked = _rule_top(scores, allowed, target - mandatory_local.size)
        expected = np.sort(cand[np.concatenate([mandatory_local, picked])])
        assert np.array_equal(gpu.core, expected)
    finally:
        gpu.close()


def test_top_k_takes_tied_scores_by_index_and_reports_the_straddle():
    from psipm_b200 import synthetic
    from psipm_b200.device import NormalEquationsDevice

    lp = synthetic.random_lp(60, 180, seed=1)
    dev = NormalEquationsDevice(lp.A)
    try:
        rng = np.random.default_rng(9)
        scores = rng.choice([0.5, 1.0, 2.0, 3.0], size=5000)
        scores[rng.integers(0, 5000, 40)] = np.nan  # not finite: never selected
        mask = (rng.random(5000) < 0.8).astype(np.uint8)
        before = dev.tie_info()["straddles"]
        for count in (1, 7, 1000, 2500):
            got = dev.top_k(scores, count, mask)
            want = np.sort(_rule_top(scores, mask.astype(bool), count))
            assert np.array_equal(got, want), f"count {count}"
        after = dev.tie_info()
        assert after["straddles"] - before == 4  # four values only: every cut splits a run
        assert after["selections"] >= 4
        # distinct scores: no straddle
        distinct = rng.permutation(5000).astype(float)
        dev.top_k(distinct, 123)
        assert dev.tie_info()["straddles"] == after["straddles"]
    finally:
        dev.close()

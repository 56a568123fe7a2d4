"""HSD pricing over all columns on the device against the oracle
(psipm_v3_1_hsd.py:2101-2158): the violation vector bit-identical to
``A' y - c tau``; the candidate set equal to the oracle's (the batch cut
below the number of eligible columns, above it, and zero); a set-cover LP
with a million columns at the reference's default pricing_batch."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("family", ["random", "cover"])
def test_pricing_matches_the_oracle(family):
    from oracle import hsd as OH
    from psipm_b200 import synthetic
    from psipm_b200.pricing import DevicePricing

    lp = (synthetic.random_lp(1600, 4800, seed=8) if family == "random"
          else synthetic.set_cover(4000, 1_000_000, seed=2000))
    m, n = lp.A.shape
    rng = np.random.default_rng(3)
    pr = DevicePricing(lp.A, lp.c)
    try:
        for round_, (tau, frac, batch) in enumerate(((0.7, 0.2, 50), (1.3, 0.5, 10**9), (1e-13, 0.1, 250_000),
                                                     (0.9, 0.3, 0))):
            y = rng.standard_normal(m) * (0.02 if family == "cover" else 1.0)
            active = rng.random(n) < frac
            v, cand = pr.price(y, tau, active, 1e-7, batch)
            v_ref, cand_ref = OH.pricing_round(lp.A, lp.c, y, tau, active, 1e-7, batch)
            assert np.array_equal(v, v_ref), round_
            assert np.array_equal(cand, cand_ref), round_
            print(f"{family} round {round_}: {cand.size} candidates of {n}")
    finally:
        pr.close()

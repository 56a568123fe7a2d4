"""Serving many small LPs at once (psipm_b200.batch): a batch of uneven
random LPs (the batched configuration's generator, scaled down) solved with
several LPs in flight, each on its own handle, stream and share of the GPU,
against the same LPs solved one after another: every LP optimal in both, the
same objective to 1e-8 relative, and the batch's throughput reported next to
the sequential one."""

import pytest

pytestmark = pytest.mark.gpu


def test_batch_matches_sequential_solves():
    from psipm_b200 import synthetic
    from psipm_b200.batch import solve_batch, solve_sequential

    lps = synthetic.random_lp_batch(count=12, mmin=500, mmax=1500, seed=4100)
    seq = solve_sequential(lps)
    bat = solve_batch(lps, workers=4)
    print(f"sequential: {seq.lps_per_second:.2f} LP/s, p50 {seq.percentile(50):.3f} s; batched (4 in flight): "
          f"{bat.lps_per_second:.2f} LP/s, p50 {bat.percentile(50):.3f} s, p99 {bat.percentile(99):.3f} s")
    assert not seq.errors and not bat.errors, (seq.errors, bat.errors)
    assert all(s == "optimal" for s in seq.status) and all(s == "optimal" for s in bat.status)
    for a, b in zip(seq.objectives, bat.objectives):
        assert abs(a - b) <= 1e-8 * max(1.0, abs(a))

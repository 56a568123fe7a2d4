"""The learned column selector on the device.

* kernels against the FP64 NumPy oracle (oracle/mlp.py): the forward pass
  (1e-5 relative), the loss and the gradient of every parameter (1e-4
  relative in norm, FP32 accumulation), one Adam step (1e-5), and the
  repeatability of the gradient (block partials added in block order: the
  same bits on every call);
* the per-column inputs that the solver feeds the network against the
  oracle's features of the same weights, scores and core;
* training on traces that the device solver writes (20 x 25-column-block
  grid networks, true leverage by Hutchinson probes on an exact factor), then
  held-out solves with and without the selector: both optimal at the same
  objective (1e-8 relative); the PCG iteration totals are reported and the
  selector's, thanks to its fallback to the plain rule, stay within 1.5x.
"""

import numpy as np
import pytest

from oracle import mlp as OM

pytestmark = pytest.mark.gpu


def _data(seed, count):
    rng = np.random.default_rng(seed)
    p = np.concatenate([rng.normal(0, 0.3, OM.N_WEIGHTS), rng.normal(0, 0.1, OM.N_BIASES)]).astype(np.float32)
    x = rng.normal(size=(count, 6)).astype(np.float32)
    y = rng.normal(size=(count, 2)).astype(np.float32)
    return p, x, y


def test_kernels_match_the_oracle_and_repeat():
    import torch

    from psipm_b200.learned import DeviceTrainer, SelectorModel

    p, x, y = _data(0, 3001)  # not a multiple of the 128-sample tile
    tr = DeviceTrainer(SelectorModel(p), blocks=7)
    xd, yd = torch.tensor(x, device="cuda"), torch.tensor(y, device="cuda")
    out = tr.forward(xd).cpu().numpy()
    ref = OM.forward(p, x)
    assert np.linalg.norm(out - ref) <= 1e-5 * np.linalg.norm(ref)
    loss, grad = tr.gradient(xd, yd, 1.0, 0.3, scale=1.0 / 3001)
    g = grad.cpu().numpy().copy()
    l_ref, g_ref = OM.loss_and_grad(p, x, y, 1.0, 0.3, scale=1.0 / 3001)
    assert abs(float(loss.item()) - l_ref) <= 1e-5 * l_ref
    for lo, hi in ((0, OM.W1), (OM.W1, OM.W1 + OM.W2), (OM.W1 + OM.W2, OM.N_WEIGHTS), (OM.N_WEIGHTS, OM.N_PARAMS)):
        assert np.linalg.norm(g[lo:hi] - g_ref[lo:hi]) <= 1e-4 * np.linalg.norm(g_ref[lo:hi]), (lo, hi)
    _, grad2 = tr.gradient(xd, yd, 1.0, 0.3, scale=1.0 / 3001)
    assert np.array_equal(grad2.cpu().numpy(), g)  # same bits
    tr.step(xd, yd, 1.0, 0.3)
    master, _, _ = OM.adam(p, np.zeros(OM.N_PARAMS), np.zeros(OM.N_PARAMS), g.astype(np.float64), 1, lr=tr.lr)
    got = tr.master.cpu().numpy()
    assert np.max(np.abs(got - master)) <= 1e-5 * max(1.0, np.max(np.abs(master)))
    assert np.array_equal(tr.w.cpu().numpy().view(np.uint16), OM.bf16_bits(got[:OM.N_WEIGHTS]))


def test_solver_features_match_the_oracle():
    from psipm_b200 import synthetic
    from psipm_b200.device import NormalEquationsDevice

    lp = synthetic.grid_network(rows=15, cols=20, seed=4)
    dev = NormalEquationsDevice(lp.A)
    try:
        rng = np.random.default_rng(5)
        theta = np.exp(rng.uniform(-8, 8, lp.A.shape[1]))
        dev.set_theta(theta, 1e-8)
        core = np.sort(rng.choice(dev.candidates, lp.A.shape[0], replace=False))
        dev.set_core(core)
        scores, _ = dev.scores(0.2)
        x = dev.mlp_features(3.5e-4)
        flags = np.isin(dev.candidates, core).astype(float)
        ref = OM.features(lp.A, dev.candidates, theta, scores, flags, 3.5e-4)
        assert np.allclose(x, ref, rtol=1e-6, atol=1e-6)
        # the network's scores replace the rule's and drive the same refresh step
        from psipm_b200.learned import SelectorModel

        model = SelectorModel(seed=3)
        vote = dev.mlp_scores(model.weights_bf16, model.biases, 3.5e-4)
        out = OM.forward(model.params, ref)
        assert abs(vote - out[:, 1].mean()) <= 1e-5 * max(1.0, abs(out[:, 1].mean()))
        k = lp.A.shape[0]
        new_core, _ = dev.refresh_core(k, 0.9, False, np.empty(0, dtype=np.int64))
        expected = np.sort(dev.candidates[np.argsort(-out[:, 0], kind="stable")[:k]])
        assert new_core.size == k
        # FP32 kernel scores against FP64 oracle scores: only near-ties at the cut may differ
        assert np.intersect1d(new_core, expected).size >= 0.99 * k
    finally:
        dev.close()


def test_training_on_traces_and_held_out_solves():
    from psipm_b200 import synthetic
    from psipm_b200.learned import collect_traces, compare, train_selector

    traces = [collect_traces(synthetic.grid_network(40, 50, seed=1100 + s), samples_per_refresh=4000, probes=32,
                             seed=s) for s in range(3)]
    assert all(t.refreshes > 0 for t in traces)
    assert all(t.solve["status"] == "optimal" for t in traces)
    result = train_selector(traces, epochs=8, batch=8192)
    hist = result["history"]
    print(f"samples {result['samples']}, loss by epoch {hist}")
    assert hist[-1] < hist[0]
    res = compare(synthetic.grid_network(40, 50, seed=1500), result["model"])
    rule, learned = res["rule"], res["learned"]
    print(f"held-out: rule {rule}\nlearned {learned}")
    assert rule["status"] == "optimal" and learned["status"] == "optimal"
    assert abs(learned["obj"] - rule["obj"]) <= 1e-8 * abs(rule["obj"])
    assert learned["learned_refreshes"] >= 1
    assert learned["pcg"] <= 1.5 * rule["pcg"]

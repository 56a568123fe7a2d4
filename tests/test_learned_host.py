"""The learned column selector without a GPU.

* the NumPy oracle of the network (oracle/mlp.py): its analytic gradient
  against central differences in FP64, for weights (at their BF16 values)
  and biases of every layer; its BF16 rounding against PyTorch's;
* the product's parameter packing (psipm_b200.learned.SelectorModel) against
  the oracle's BF16 bit patterns;
* the solver policy (psipm_b200.kkt): a learned core that the rule's own
  signals call poor (psipm_spectral_preconditioner.py:420-467) makes the next
  factorisation refresh with the plain rule and suspends the network for
  `selector_patience` refreshes; a full solve with a selector on the CPU
  stand-in device ends optimal at the plain rule's objective.
"""

import numpy as np
import pytest
import torch

from fake_device import FakeDevice
from oracle import ipm as OI
from oracle import mlp as OM
from psipm_b200 import synthetic
from psipm_b200.kkt import GpuSpectralStableColumnPreconditioner
from psipm_b200.learned import SelectorModel

OPTS = dict(full_preconditioner_row_threshold=10)


def random_params(seed):
    rng = np.random.default_rng(seed)
    return np.concatenate([rng.normal(0, 0.3, OM.N_WEIGHTS), rng.normal(0, 0.1, OM.N_BIASES)]).astype(np.float32)


@pytest.mark.parametrize("index", [0, 5, 383, 384, 2000, 4479, 4480, 4607, 4608, 4671, 4700, 4736, 4737])
def test_oracle_gradient_matches_central_differences(index):
    rng = np.random.default_rng(1)
    p = random_params(2)
    x = rng.normal(size=(40, 6))
    y = rng.normal(size=(40, 2))
    _, g = OM.loss_and_grad(p, x, y, 1.0, 0.3)
    fd = OM.finite_difference(p, x, y, index, 1.0, 0.3)
    assert abs(g[index] - fd) <= 1e-7 * max(1.0, abs(fd))


def test_bf16_rounding_matches_torch():
    x = np.random.default_rng(3).normal(0, 10, 10000).astype(np.float32)
    x[:4] = [1.00390625, 1.01171875, -3.0e-39, 65504.0]  # ties and a subnormal
    ours = OM.bf16_bits(x)
    ref = torch.tensor(x).to(torch.bfloat16).view(torch.int16).numpy().view(np.uint16)
    assert np.array_equal(ours, ref)


def test_model_packing_matches_the_oracle():
    model = SelectorModel(seed=4)
    assert np.array_equal(model.weights_bf16, OM.bf16_bits(model.params[:OM.N_WEIGHTS]))
    assert np.array_equal(model.biases, model.params[OM.N_WEIGHTS:])


def test_poor_learned_core_falls_back_to_the_rule():
    lp = synthetic.random_lp(120, 360, seed=9)
    dev = FakeDevice(lp.A)
    solver = GpuSpectralStableColumnPreconditioner(lp.A, protected=~lp.pos, dev=dev, selector=SelectorModel(seed=1),
                                                   selector_patience=2, **OPTS)
    theta = np.exp(np.random.default_rng(0).uniform(-2, 2, lp.A.shape[1]))
    solver.observe(None, None, None, None, 0.1)
    solver.factorize(theta, 1e-6)
    assert solver.learned_refreshes == 1 and solver._core_learned
    solver._last_cg = solver.refresh_cg  # the learned core's last solve was poor
    refreshes = solver.refreshes
    solver.factorize(theta, 1e-6)
    assert solver.selector_fallbacks == 1
    assert solver.refreshes == refreshes + 1 and not solver._core_learned
    assert solver.learned_refreshes == 1
    solver._last_cg = 1
    for _ in range(2):  # the next refresh still uses the rule, then the network again
        solver.core_age = solver.core_max_age
        solver.factorize(theta, 1e-6)
    assert solver.learned_refreshes == 2 and solver._core_learned


def test_full_solve_with_a_selector_on_the_cpu_stand_in():
    lp = synthetic.grid_network(rows=6, cols=7, seed=3)
    plain = OI.psipm_solve(lp, GpuSpectralStableColumnPreconditioner(lp.A, protected=~lp.pos,
                                                                      dev=FakeDevice(lp.A), **OPTS), tol=1e-8)
    solver = GpuSpectralStableColumnPreconditioner(lp.A, protected=~lp.pos, dev=FakeDevice(lp.A),
                                                   selector=SelectorModel(seed=2), **OPTS)
    sol = OI.psipm_solve(lp, solver, tol=1e-8)
    assert sol.status == "optimal" and plain.status == "optimal"
    assert abs(sol.obj - plain.obj) <= 1e-7 * max(1.0, abs(plain.obj))
    assert solver.learned_refreshes >= 1

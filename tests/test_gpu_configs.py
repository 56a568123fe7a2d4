"""Device parity at the sizes of the benchmark configurations.

* Random LP, m = 2,000, n = 6,000 (fixture ``random_m2000``, written by the
  unmodified reference with its default options): per call, scores
  bit-identical, refreshed cores identical, the device Newton direction
  (with the reference's lagged factor where it reused one) within 1e-6
  relative of the reference's own FP64 PCG direction at the reference's
  tolerance, with the same PCG iteration count up to one; the
  complete device PS-IPM solve optimal at the reference's objective to 1e-8.
* Grid min-cost-flow LP, 200 x 250 (the benchmark's LP, seed 1000): the
  complete device-resident solve optimal, objective within 1e-8 relative of
  the reference's complete solve (``grid_200x250_result.json``), KKT
  residuals under 1e-8, outer iteration count within two of the reference's.
* Set cover, m = 4,000, n = 1,004,000: FP32 PCG inside FP64 refinement
  against the FP64 solve, per Newton system of the first outer iterations of
  a device solve: relative direction error (reported) under 1e-6 and the
  FP64 relative residual of the refined direction at its tolerance.
"""

import json
import os

import numpy as np
import pytest

from _helpers import lp_from, normal_matrix, rel

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))


def test_random_m2000_per_call_parity(golden):
    from psipm_b200.device import NormalEquationsDevice

    g = golden("random_m2000")
    lp = lp_from(g)
    dev = NormalEquationsDevice(lp.A)
    try:
        assert np.array_equal(dev.candidates, g["candidates"])
        mandatory = np.union1d(dev.candidates[(~lp.pos)[dev.candidates]], g["matching_columns"])
        mand = np.searchsorted(dev.candidates, mandatory)
        scored = 0
        for i in range(int(g["n_factor_calls"])):
            if f"f{i}_scores" not in g:
                continue
            before = g[f"f{i}_core_before"]
            dev.set_core(before)
            dev.set_theta(g[f"f{i}_theta"], float(g[f"f{i}_delta"]))
            scores, _ = dev.scores(0.2)
            assert np.array_equal(scores, g[f"f{i}_scores"]), f"scores, call {i}"
            core, _ = dev.refresh_core(int(g[f"f{i}_core_target"]), 0.9, before.size > 0, mand)
            assert np.array_equal(core, g[f"f{i}_core"]), f"core, call {i}"
            scored += 1
        assert scored
        nf = int(g["n_factor_calls"])
        for i in range(int(g["n_solve_calls"])):
            theta, delta, tol = g[f"s{i}_theta"], float(g[f"s{i}_delta"]), float(g[f"s{i}_tolerance"])
            # the preconditioner of this solve: the factor of the last factorize call that
            # refactored (factor_age 0) -- a lagged factor keeps an older theta
            k = max(j for j in range(nf) if np.array_equal(g[f"f{j}_theta"], theta))
            k = max(j for j in range(k + 1) if int(g[f"f{j}_factor_age"]) == 0)
            dev.set_core(g[f"s{i}_core"])
            dev.set_theta(g[f"f{k}_theta"], float(g[f"f{k}_delta"]))
            dev.factor(float(g[f"f{k}_delta"]), 0)
            dev.set_theta(theta, delta)  # the operator's weights; the factor stays
            dx, res = dev.solve(g[f"s{i}_r1"], g[f"s{i}_r2"], tol, 200, 0, 100, 0.1)
            err_y, err_x = rel(res.x, g[f"s{i}_dy"]), rel(dx, g[f"s{i}_dx"])
            print(f"call {i}: tol {tol:.0e}, iterations {res.iterations} (reference "
                  f"{int(g[f's{i}_iterations'])}), dy error {err_y:.2e}, dx error {err_x:.2e}")
            assert err_y <= 1e-6 and err_x <= 1e-6, (i, err_y, err_x)
            assert abs(res.iterations - int(g[f"s{i}_iterations"])) <= 1, i
    finally:
        dev.close()


def test_random_m2000_full_device_solve(golden):
    from psipm_b200 import synthetic
    from psipm_b200.ipm_device import solve_standard

    g = golden("random_m2000")
    lp = synthetic.random_lp(2000, 6000, seed=0)
    assert np.array_equal(lp.A.data, g["A_data"]) and np.array_equal(lp.b, g["b"])
    sol, solver = solve_standard(lp, tol=1e-8)
    try:
        assert sol.status == "optimal"
        ref = float(g["obj"])
        print(f"objective {sol.obj!r} (reference {ref!r}), outer {sol.outer_iter}, PCG {sol.pcg_iterations} "
              f"(reference {int(g['pcg_iterations'])})")
        assert abs(sol.obj - ref) <= 1e-8 * abs(ref)
        assert sol.res_p < 1e-8 and sol.res_d < 1e-8 and sol.gap < 1e-8
    finally:
        solver.close()


def test_grid_200x250_full_device_solve_matches_the_reference_result():
    from psipm_b200 import synthetic
    from psipm_b200.ipm_device import solve_standard

    path = os.path.join(HERE, "golden", "grid_200x250_result.json")
    if not os.path.exists(path):
        pytest.skip("grid_200x250_result.json not generated (tests/golden/make_golden.py)")
    with open(path) as f:
        ref = json.load(f)
    lp = synthetic.grid_network(**ref["kwargs"])
    fp = ref["fingerprint"]
    assert list(lp.A.shape) == fp["shape"] and lp.A.nnz == fp["nnz"]
    assert float(lp.c.sum()) == fp["c_sum"] and float(np.abs(lp.b).sum()) == fp["b_abs_sum"]
    sol, solver = solve_standard(lp, tol=1e-8)
    try:
        print(f"objective {sol.obj!r} (reference {ref['obj']!r}), outer {sol.outer_iter} (reference "
              f"{ref['outer_iter']}), inner {sol.inner_iter} (reference {ref['inner_iter']}), PCG "
              f"{sol.pcg_iterations} (reference {ref['pcg_iterations']})")
        assert sol.status == "optimal" and ref["status"] == "optimal"
        assert abs(sol.obj - ref["obj"]) <= 1e-8 * abs(ref["obj"])
        assert sol.res_p < 1e-8 and sol.res_d < 1e-8 and sol.gap < 1e-8
        assert abs(sol.outer_iter - ref["outer_iter"]) <= 2
    finally:
        solver.close()


def test_set_cover_fp32_refined_directions_against_fp64():
    from oracle import ipm as OI
    from psipm_b200 import _lib, synthetic
    from psipm_b200.device import NormalEquationsDevice
    from psipm_b200.kkt import GpuSpectralStableColumnPreconditioner

    lp = synthetic.set_cover(4000, 1_000_000, seed=2000)
    m, n = lp.A.shape

    class Recording(GpuSpectralStableColumnPreconditioner):
        systems = []

        def solve(self, r1, r2):
            self.systems.append((self.theta.copy(), self.delta, self.core.copy(), r1.copy(), r2.copy()))
            return super().solve(r1, r2)

    rec = Recording(lp.A, protected=~lp.pos)
    try:
        OI.psipm_solve(lp, rec, tol=1e-8, max_outer=2)
    finally:
        rec.close()
    systems = Recording.systems[::3][:6]  # a spread of the recorded Newton systems
    d64 = NormalEquationsDevice(lp.A, precision=_lib.FP64)
    d32 = NormalEquationsDevice(lp.A, precision=_lib.FP32_REFINED)
    try:
        for k, (theta, delta, core, r1, r2) in enumerate(systems):
            out = {}
            for name, dev in (("fp64", d64), ("fp32", d32)):
                dev.set_theta(theta, delta)
                dev.set_core(core)
                dev.factor(delta, 0)
                out[name] = dev.solve(r1, r2, 1e-10, 2000, 0, 100, 0.1)
            dx64, r64 = out["fp64"]
            dx32, r32 = out["fp32"]
            H = normal_matrix(lp.A, theta, delta)
            rhs = r2 - lp.A @ (r1 / theta)
            res32 = np.linalg.norm(rhs - H @ r32.x) / max(1.0, np.linalg.norm(rhs))
            err = rel(r32.x, r64.x)
            print(f"system {k}: FP32-refined dy error vs FP64 {err:.2e}, dx error {rel(dx32, dx64):.2e}, "
                  f"FP64 residual {res32:.2e}, refinement sweeps {r32.refinements}, iterations "
                  f"{r32.iterations} (FP64 {r64.iterations})")
            assert r64.info == 0 and r32.ok
            assert res32 <= 2e-10
            assert err <= 1e-6
    finally:
        d64.close()
        d32.close()

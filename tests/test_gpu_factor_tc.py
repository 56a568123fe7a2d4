"""Tensor-core trailing updates of the FP32 factor (factor_tc.cu).

The update kernel alone (psipm_debug_syrk_tc) is checked against an FP64
NumPy product on fronts of uneven sizes, panel offsets, column limits and K
values that are not multiples of the 32-wide stage; entries outside the
updated lower triangle must come back bit for bit.  3xTF32 products must meet
the FP32 dot-product bound, (kb + 8) 2^-23 of sum |P_ik P_jk| + |result|; TF32
ones that bound plus 2^-10.  The factor as a whole
is checked through the preconditioner: an FP32 handle factored on the tensor
cores gives the same apply as the CUDA-core FP32 factor (to FP32 rounding
amplified by the conditioning) and as the FP64 factor, and a full FP32 solve
reaches the FP64 solve's objective.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def syrk_tc(F, k0, kb, jend, passes):
    from psipm_b200 import _lib

    lib = _lib.load()
    r = F.shape[0]
    fin = np.asfortranarray(F, dtype=np.float32)
    out = np.empty_like(fin)
    status = lib.psipm_debug_syrk_tc(0, r, k0, kb, jend, passes, fin.ctypes.data, out.ctypes.data)
    assert status == _lib.OK, status
    return out


@pytest.mark.parametrize("r,k0,kb,jend", [
    (200, 0, 64, 200), (300, 37, 64, 300), (517, 0, 256, 517), (517, 64, 100, 400),
    (700, 128, 256, 700), (390, 10, 7, 390), (1100, 0, 256, 1100), (1100, 256, 64, 512)])
@pytest.mark.parametrize("passes", [3, 1])
def test_update_matches_fp64_product(r, k0, kb, jend, passes):
    rng = np.random.default_rng(r + k0 + kb + passes)
    F = rng.standard_normal((r, r)).astype(np.float32)
    F[:, k0:k0 + kb] *= np.exp(rng.uniform(-3, 3, (r, kb))).astype(np.float32)
    out = syrk_tc(F, k0, kb, jend, passes)
    base = k0 + kb
    P = F[:, k0:k0 + kb].astype(np.float64)
    exact = F.astype(np.float64) - P @ P.T
    bound = np.abs(P) @ np.abs(P).T
    i, j = np.indices((r, r))
    region = (j >= base) & (j < jend) & (i >= j)
    # FP32 dot-product bound (kb + 8) 2^-23 of sum |P_ik P_jk| (3xTF32); TF32 heads add 2^-10
    tol = (kb + 8) * 2.0 ** -23 + (0.0 if passes == 3 else 2.0 ** -10)
    err = np.abs(out.astype(np.float64) - exact)
    ratio = err[region] / (bound[region] + np.abs(exact[region]) + 1e-30)
    assert ratio.max() <= tol, (float(ratio.max()), tol)
    assert np.array_equal(out[~region], F[~region])


def _cover_handles(precision_list, m, n, seed):
    from psipm_b200 import synthetic
    from psipm_b200.device import NormalEquationsDevice

    lp = synthetic.set_cover(m, n, seed=seed)
    devs = [NormalEquationsDevice(lp.A, precision=p) for p in precision_list]
    return lp, devs


@pytest.mark.parametrize("m,n", [(400, 20_000), (1500, 60_000)])
def test_fp32_factor_on_tensor_cores_matches_cuda_cores(m, n):
    from psipm_b200 import _lib

    lp, (d64, d32) = _cover_handles([_lib.FP64, _lib.FP32_PRECOND], m, n, seed=2001 + m)
    try:
        rng = np.random.default_rng(5)
        theta = np.exp(rng.uniform(-2, 2, lp.A.shape[1]))
        delta = 1e-6
        core = np.sort(rng.choice(d64.candidates, min(d64.candidates.size, 2 * m), replace=False))
        for d in (d64, d32):
            d.set_theta(theta, delta)
            d.set_core(core)
        r = rng.standard_normal(m)
        d64.factor(delta, 0)
        z64 = d64.apply(r)
        z = {}
        for passes in (0, 3, 1):
            d32.set_factor_tc(passes)
            d32.factor(delta, 0)
            z[passes] = d32.apply(r)
        scale = np.linalg.norm(z64)
        assert np.linalg.norm(z[0] - z64) <= 1e-3 * scale
        assert np.linalg.norm(z[3] - z64) <= 1e-3 * scale
        assert np.linalg.norm(z[3] - z[0]) <= 1e-3 * scale
        assert np.isfinite(z[1]).all() and np.linalg.norm(z[1] - z64) <= 0.5 * scale
    finally:
        d64.close()
        d32.close()


def test_fp32_solve_with_tensor_core_factor_reaches_the_fp64_objective():
    from psipm_b200 import _lib, synthetic
    from psipm_b200.ipm_device import solve_standard

    lp = synthetic.set_cover(400, 20_000, seed=2001)
    ref, s64 = solve_standard(lp, tol=1e-8, precision=_lib.FP64)
    s64.close()
    sol, s32 = solve_standard(lp, tol=1e-8, precision=_lib.FP32_PRECOND)
    launches = s32.dev.kernel_launches
    s32.close()
    assert ref.status == "optimal" and sol.status == "optimal"
    assert abs(sol.obj - ref.obj) <= 1e-7 * max(1.0, abs(ref.obj))
    assert launches > 0

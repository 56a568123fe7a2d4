"""The allocation-free operator product against the handle-based one.

psipm_normal_matvec_static exists for callers that cannot allocate device
memory (a host framework that owns the device pool, code that may not call
cudaMalloc because it synchronises the device, a fixed-footprint solver): the
caller passes every buffer and the library's intermediate vector lives in a
fixed array inside the library.  This file is collected last on purpose, so
a run that stops at the first failure has run every other test before it.
"""

import ctypes

import numpy as np
import pytest
import scipy.sparse as sp

pytestmark = pytest.mark.gpu


def _device_arrays(torch, A, theta):
    A = sp.csc_matrix(A)
    A.sort_indices()
    csr = A.tocsr()
    csr.sort_indices()
    dev = torch.device("cuda", 0)
    return dict(
        at_ptr=torch.tensor(A.indptr.astype(np.int32), device=dev),
        at_idx=torch.tensor(A.indices.astype(np.int32), device=dev),
        at_val=torch.tensor(A.data, dtype=torch.float64, device=dev),
        a_ptr=torch.tensor(csr.indptr.astype(np.int32), device=dev),
        a_idx=torch.tensor(csr.indices.astype(np.int32), device=dev),
        a_val=torch.tensor(csr.data, dtype=torch.float64, device=dev),
        w=torch.tensor(1.0 / theta, dtype=torch.float64, device=dev),
    )


def test_static_matvec_matches_handle_matvec_twice():
    import torch

    from psipm_b200 import _lib, synthetic
    from psipm_b200.device import NormalEquationsDevice

    lib = _lib.load()
    lp = synthetic.random_lp(400, 1200, seed=3)
    m, n = lp.A.shape
    rng = np.random.default_rng(11)
    theta = np.exp(rng.uniform(-4.0, 4.0, n))
    delta = 1e-6
    handle = NormalEquationsDevice(lp.A)
    handle.set_theta(theta, delta)
    d = _device_arrays(torch, lp.A, theta)
    stream = torch.cuda.current_stream().cuda_stream
    p = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
    for call in range(2):
        v = rng.standard_normal(m)
        expected = handle.matvec(v)  # the existing entry point (host buffers)
        v_dev = torch.tensor(v, dtype=torch.float64, device="cuda")
        y_dev = torch.full((m,), float("nan"), dtype=torch.float64, device="cuda")
        status = lib.psipm_normal_matvec_static(
            m, n, p(d["at_ptr"]), p(d["at_idx"]), p(d["at_val"]), p(d["a_ptr"]), p(d["a_idx"]),
            p(d["a_val"]), p(d["w"]), delta, p(v_dev), p(y_dev), ctypes.c_void_p(stream))
        assert status == _lib.OK, f"call {call}: status {status}"
        torch.cuda.synchronize()
        y = y_dev.cpu().numpy()
        err = np.linalg.norm(y - expected) / np.linalg.norm(expected)
        assert err <= 1e-13, f"call {call}: relative difference {err:.2e}"
    handle.close()


def test_static_matvec_rejects_too_many_columns():
    import torch

    from psipm_b200 import _lib

    lib = _lib.load()
    x = torch.zeros(4, dtype=torch.float64, device="cuda")
    i = torch.zeros(4, dtype=torch.int32, device="cuda")
    p = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
    status = lib.psipm_normal_matvec_static(
        2, _lib.STATIC_SCRATCH_MAX + 1, p(i), p(i), p(x), p(i), p(i), p(x), p(x), 0.0, p(x), p(x), None)
    assert status == _lib.ERR_ARGUMENT


def test_static_matvec_at_the_column_limit_on_the_null_stream_leaves_inputs_unchanged():
    """n exactly at the limit (one nonzero per column keeps it small), the NULL
    stream, and a check that the call writes only y."""
    import torch

    from psipm_b200 import _lib

    lib = _lib.load()
    m, n = 64, _lib.STATIC_SCRATCH_MAX
    rng = np.random.default_rng(5)
    rows = rng.integers(0, m, n)
    A = sp.csc_matrix((rng.standard_normal(n), (rows, np.arange(n))), shape=(m, n))
    theta = np.exp(rng.uniform(-2.0, 2.0, n))
    delta = 1e-3
    d = _device_arrays(torch, A, theta)
    v = rng.standard_normal(m)
    v_dev = torch.tensor(v, dtype=torch.float64, device="cuda")
    y_dev = torch.full((m,), float("nan"), dtype=torch.float64, device="cuda")
    before = {k: t.clone() for k, t in d.items()}
    v_before = v_dev.clone()
    torch.cuda.synchronize()
    p = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
    for call in range(2):
        status = lib.psipm_normal_matvec_static(
            m, n, p(d["at_ptr"]), p(d["at_idx"]), p(d["at_val"]), p(d["a_ptr"]), p(d["a_idx"]),
            p(d["a_val"]), p(d["w"]), delta, p(v_dev), p(y_dev), None)
        assert status == _lib.OK, f"call {call}: status {status}"
        torch.cuda.synchronize()
        expected = A @ ((A.T @ v) / theta) + delta * v
        y = y_dev.cpu().numpy()
        err = np.linalg.norm(y - expected) / np.linalg.norm(expected)
        assert err <= 1e-13, f"call {call}: relative difference {err:.2e}"
    for k, t in d.items():
        assert torch.equal(t, before[k]), f"{k} was modified"
    assert torch.equal(v_dev, v_before), "v was modified"

"""Argument checks at the C ABI that run before any CUDA call (no GPU needed).

Every entry point rejects a null handle and null or out-of-range arguments
with PSIPM_ERR_ARGUMENT instead of touching memory, and psipm_create
validates the CSC pattern (sizes, column pointers, sorted in-range row
indices, precision) on the host.  The error contract mirrors the reference's
exceptions (psipm_active_pool.py:2033-2040, 2046-2049): the Python layer turns
every nonzero status into an exception.
"""

import ctypes

import numpy as np
import pytest

from psipm_b200 import _lib

P = ctypes.c_void_p


def zero_args(argtypes):
    return [None if t is P or t is None or isinstance(t, type(ctypes.POINTER(P))) else t(0) for t in argtypes]


@pytest.fixture(scope="module")
def lib():
    return _lib.load()


def test_null_handle_is_rejected_by_every_entry_point(lib):
    skip = {"psipm_create", "psipm_normal_matvec_static", "psipm_mlp_forward_dev", "psipm_mlp_grad_dev",
            "psipm_mlp_adam_dev", "psipm_debug_syrk_tc"}
    checked = 0
    for name, (restype, argtypes) in _lib.SIGNATURES.items():
        if name in skip or not argtypes or argtypes[0] is not P:
            continue
        out = getattr(lib, name)(*zero_args(argtypes))
        if name == "psipm_destroy":
            assert out is None
        elif name == "psipm_last_error":
            assert out == b"null handle"
        elif restype is ctypes.c_int64:  # counts: -1 without a handle
            assert out == -1, name
        else:
            assert out == _lib.ERR_ARGUMENT, name
        checked += 1
    assert checked == len(_lib.SIGNATURES) - len(skip)


def test_tensor_core_hooks_reject_bad_arguments(lib):
    f = lib.psipm_debug_syrk_tc
    buf = (ctypes.c_float * 16)()
    p = ctypes.cast(buf, P)
    good = [0, 4, 0, 2, 4, 3, p, p]
    for k, bad in ((1, 0), (2, -1), (3, 0), (3, 5), (4, 5), (5, 2), (6, None), (7, None)):
        args = list(good)
        args[k] = bad
        assert f(*args) == _lib.ERR_ARGUMENT, (k, bad)
    assert lib.psipm_set_factor_tc(None, 3) == _lib.ERR_ARGUMENT


def test_static_matvec_rejects_null_and_oversized_arguments(lib):
    f = lib.psipm_normal_matvec_static
    buf = (ctypes.c_double * 4)()
    ib = (ctypes.c_int32 * 4)()
    p = ctypes.cast(buf, P)
    q = ctypes.cast(ib, P)
    good = [2, 2, q, q, p, q, q, p, p, 0.0, p, p, None]
    for k in (2, 3, 4, 5, 6, 7, 8, 10, 11):
        args = list(good)
        args[k] = None
        assert f(*args) == _lib.ERR_ARGUMENT, k
    for m, n in ((0, 2), (2, 0), (2, _lib.STATIC_SCRATCH_MAX + 1)):
        args = list(good)
        args[0], args[1] = m, n
        assert f(*args) == _lib.ERR_ARGUMENT, (m, n)


def create(lib, m, n, colptr, rowidx, values, precision=_lib.FP64):
    colptr = np.ascontiguousarray(colptr, dtype=np.int64)
    rowidx = np.ascontiguousarray(rowidx, dtype=np.int32)
    values = np.ascontiguousarray(values, dtype=np.float64)
    handle = P()
    status = lib.psipm_create(m, n, int(values.size), colptr.ctypes.data, rowidx.ctypes.data, values.ctypes.data,
                              0, precision, ctypes.byref(handle))
    assert not handle.value
    return status


@pytest.mark.parametrize("case", [
    "rows", "columns", "colptr_start", "colptr_end", "colptr_decreasing", "row_negative", "row_too_large",
    "rows_unsorted", "rows_duplicate", "precision",
])
def test_create_validates_the_pattern_on_the_host(lib, case):
    # a valid 3 x 3 pattern, then one defect
    m, n = 3, 3
    colptr = [0, 2, 3, 5]
    rowidx = [0, 2, 1, 0, 1]
    values = [1.0, 2.0, 3.0, 4.0, 5.0]
    precision = _lib.FP64
    if case == "rows":
        m = 0
    elif case == "columns":
        n = -1
    elif case == "colptr_start":
        colptr = [1, 2, 3, 5]
    elif case == "colptr_end":
        colptr = [0, 2, 3, 4]
    elif case == "colptr_decreasing":
        colptr = [0, 3, 2, 5]
    elif case == "row_negative":
        rowidx = [0, -1, 1, 0, 1]
    elif case == "row_too_large":
        rowidx = [0, 3, 1, 0, 1]
    elif case == "rows_unsorted":
        rowidx = [2, 0, 1, 0, 1]
    elif case == "rows_duplicate":
        rowidx = [0, 0, 1, 0, 1]
    elif case == "precision":
        precision = 7
    assert create(lib, m, n, colptr, rowidx, values, precision) == _lib.ERR_ARGUMENT


def test_create_rejects_a_null_output_and_oversized_problems(lib):
    colptr = np.zeros(2, dtype=np.int64)
    assert lib.psipm_create(1, 1, 0, colptr.ctypes.data, None, None, 0, _lib.FP64, None) == _lib.ERR_ARGUMENT
    handle = P()
    assert lib.psipm_create(1 << 31, 1, 0, colptr.ctypes.data, None, None, 0, _lib.FP64,
                            ctypes.byref(handle)) == _lib.ERR_UNSUPPORTED


def test_selector_training_kernels_reject_null_arguments(lib):
    """The device-pointer training entry points check their pointers and sizes
    before any CUDA call."""
    buf = (ctypes.c_float * 8)()
    p = ctypes.cast(buf, P)
    f = ctypes.c_float
    assert lib.psipm_mlp_forward_dev(-1, p, p, p, p, None) == _lib.ERR_ARGUMENT
    assert lib.psipm_mlp_forward_dev(4, None, p, p, p, None) == _lib.ERR_ARGUMENT
    assert lib.psipm_mlp_forward_dev(0, None, p, p, None, None) == _lib.OK  # nothing to do
    good = [4, p, p, f(1.0), f(0.0), p, p, 2, p, p, f(1.0), p, p, None]
    for k in (1, 2, 5, 6, 8, 9, 11, 12):
        args = list(good)
        args[k] = None
        assert lib.psipm_mlp_grad_dev(*args) == _lib.ERR_ARGUMENT, k
    for k, bad in ((0, 0), (7, 0)):
        args = list(good)
        args[k] = bad
        assert lib.psipm_mlp_grad_dev(*args) == _lib.ERR_ARGUMENT, k
    adam = [p, p, p, p, f(1e-3), f(0.9), f(0.999), f(1e-8), 1, f(0.0), p, p, None]
    for k in (0, 1, 2, 3, 10, 11):
        args = list(adam)
        args[k] = None
        assert lib.psipm_mlp_adam_dev(*args) == _lib.ERR_ARGUMENT, k
    args = list(adam)
    args[8] = 0
    assert lib.psipm_mlp_adam_dev(*args) == _lib.ERR_ARGUMENT

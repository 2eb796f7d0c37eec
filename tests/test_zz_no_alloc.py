"""The allocation-free entry point fc_sum_sumsq_static.

Some callers cannot allocate device memory at all: code running where a
cudaMalloc would synchronise the whole device in the middle of other work,
or a plugin inside a host application that has reserved the GPU's memory for
its own allocator.  fc_sum_sumsq_static gives them the grid sum and sum of
squares (array_ops sum/sumsq) using only a fixed scratch array compiled into
the library.  This test calls it through the C ABI, twice in a row, and
compares it with the allocating fc_grid_sum within the tolerance the other
tests use for FP64 reductions (1e-12 relative).  The buffers the test itself
needs are allocated by the test, not by the entry point under test.
"""
import ctypes

import numpy as np
import pytest

from fftcorr_b200 import _lib

pytestmark = pytest.mark.gpu

RTOL = 1e-12


def _device_grid(values):
    shape = np.array(values.shape, dtype=np.intc)
    h = ctypes.c_void_p()
    _lib.call("fc_grid_create", _lib.iptr(shape), _lib.dptr(np.zeros(3)), 1.0,
              ctypes.byref(h))
    _lib.call("fc_grid_upload", h, _lib.dptr(np.ascontiguousarray(values)))
    ptr = ctypes.c_void_p()
    _lib.call("fc_grid_device_ptr", h, ctypes.byref(ptr))
    return h, ptr


def test_static_sum_matches_allocating_sum_on_two_calls():
    rng = np.random.default_rng(12)
    values = rng.normal(size=(96, 80, 70)) + 0.25
    h, ptr = _device_grid(values)
    try:
        s_ref, q_ref = ctypes.c_double(), ctypes.c_double()
        _lib.call("fc_grid_sum", h, ctypes.byref(s_ref), ctypes.byref(q_ref))
        for _ in range(2):
            s, q = ctypes.c_double(), ctypes.c_double()
            _lib.call("fc_sum_sumsq_static", ptr, values.size, ctypes.byref(s),
                      ctypes.byref(q))
            assert s.value == pytest.approx(s_ref.value, rel=RTOL)
            assert q.value == pytest.approx(q_ref.value, rel=RTOL)
            assert q.value == pytest.approx(float(np.sum(values * values)), rel=RTOL)
    finally:
        _lib.load().fc_grid_destroy(h)


@pytest.mark.parametrize("n", [0, (1 << 18) - 1, (1 << 18) + 1])
def test_static_sum_edge_sizes(n):
    """No values (the result slots are cleared, not summed), and one value
    short of and past the size one block sums, whose last block then ends
    part way."""
    rng = np.random.default_rng(n + 1)
    values = rng.normal(size=(1, 1, max(n, 1))) - 0.5
    h, ptr = _device_grid(values)
    try:
        # A call on other data first, so a stale result would show.
        s, q = ctypes.c_double(), ctypes.c_double()
        _lib.call("fc_sum_sumsq_static", ptr, values.size, ctypes.byref(s),
                  ctypes.byref(q))
        _lib.call("fc_sum_sumsq_static", ptr, n, ctypes.byref(s), ctypes.byref(q))
        v = values.reshape(-1)[:n]
        if n == 0:
            assert s.value == 0.0 and q.value == 0.0
        else:
            assert s.value == pytest.approx(float(np.sum(v)), rel=RTOL)
            assert q.value == pytest.approx(float(np.sum(v * v)), rel=RTOL)
    finally:
        _lib.load().fc_grid_destroy(h)


def test_static_sum_rejects_sizes_beyond_its_scratch():
    values = np.ones((4, 4, 4))
    h, ptr = _device_grid(values)
    try:
        s, q = ctypes.c_double(), ctypes.c_double()
        rc = _lib.load().fc_sum_sumsq_static(ptr, (1 << 30) + 1, ctypes.byref(s),
                                             ctypes.byref(q))
        assert rc == _lib.FC_ERR_RANGE
        # A valid call right after the rejected one still works.
        _lib.call("fc_sum_sumsq_static", ptr, values.size, ctypes.byref(s),
                  ctypes.byref(q))
        assert s.value == 64.0 and q.value == 64.0
    finally:
        _lib.load().fc_grid_destroy(h)

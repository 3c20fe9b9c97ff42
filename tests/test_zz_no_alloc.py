"""The split product for callers that can't allocate device memory.

``einfold_split_gemm_static`` serves an engine that has handed all of HBM to
its own pool, or code that runs where allocating is forbidden (inside an
allocator's callback, or under a budget that allows no memory outside the
pool). Its scratch is one fixed 64 MiB array in the library's device memory,
shared by every call. These tests call it through the C ABI and compare it
with ``einfold_split_gemm``, which allocates its scratch per call, on two
calls in a row with different shapes, so that a stale byte left in the shared
array by the first call would show in the second. This file is collected
last, and passes alone in a fresh process as well as after the other tests.
"""
import ctypes

import numpy as np
import pytest

from einfold_b200 import _lib
from tests.tables import split_bound

pytestmark = pytest.mark.gpu


def _product(static, a, b, batches, m, n, k, transposed):
    import torch

    lib = _lib.load()
    ta = torch.from_numpy(a).cuda()
    tb = torch.from_numpy(b).cuda()
    tc = torch.full((batches, m, n), float("nan"), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    if static:
        msg = ctypes.create_string_buffer(480)
        st = lib.einfold_split_gemm_static(ta.data_ptr(), tb.data_ptr(), tc.data_ptr(), batches, m, n, k, transposed,
                                           6, None, msg, 480)
        assert st == _lib.OK, msg.value.decode()
    else:
        st = lib.einfold_split_gemm(_lib.context(0), ta.data_ptr(), tb.data_ptr(), tc.data_ptr(), batches, m, n, k,
                                    transposed, 6, None)
        assert st == _lib.OK, lib.einfold_last_error()
    torch.cuda.synchronize()
    return tc.cpu().numpy()


def test_static_scratch_matches_the_allocating_entry_point_twice():
    rng = np.random.default_rng(21)
    cases = [(1, 300, 200, 1000, 0), (2, 129, 65, 257, 1)]
    for batches, m, n, k, transposed in cases:
        a = rng.uniform(-1, 1, (batches, m, k))
        b = rng.standard_normal((batches, k, n)) * 1e3
        bb = np.ascontiguousarray(b.transpose(0, 2, 1)) if transposed else b
        want = _product(False, a, bb, batches, m, n, k, transposed)
        got = _product(True, a, bb, batches, m, n, k, transposed)
        for w in range(batches):
            tol = split_bound(k, np.abs(a[w]).max(1), np.abs(b[w]).max(0)) + \
                2 * k * 2.0 ** -53 * (np.abs(a[w]) @ np.abs(b[w]))
            assert (np.abs(got[w] - want[w]) <= tol).all()
            assert (np.abs(got[w] - a[w] @ b[w]) <= 2 * tol).all()


def test_static_scratch_refuses_a_product_too_large_for_it():
    import torch

    lib = _lib.load()
    m = n = k = 4096  # 6 x (4096 + 4096) x 4096 bytes of digits: more than 64 MiB
    ta = torch.zeros((m, k), dtype=torch.float64, device="cuda")
    tb = torch.zeros((k, n), dtype=torch.float64, device="cuda")
    tc = torch.zeros((m, n), dtype=torch.float64, device="cuda")
    msg = ctypes.create_string_buffer(480)
    st = lib.einfold_split_gemm_static(ta.data_ptr(), tb.data_ptr(), tc.data_ptr(), 1, m, n, k, 0, 6, None, msg, 480)
    assert st == _lib.INVALID
    assert b"einfold_split_gemm" in msg.value

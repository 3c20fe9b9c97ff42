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
import os
import subprocess
import sys
import textwrap

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


def test_static_scratch_refuses_sizes_whose_scratch_would_overflow():
    # A k so large that the digits' byte count wraps 64 bits must still be
    # refused, not wrapped to a small size that passes the check.
    import torch

    lib = _lib.load()
    t = torch.zeros(8, dtype=torch.float64, device="cuda")
    msg = ctypes.create_string_buffer(480)
    for k in (2 ** 61, 2 ** 62 - 1, 2 ** 40):
        st = lib.einfold_split_gemm_static(t.data_ptr(), t.data_ptr(), t.data_ptr(), 1, 1, 1, k, 0, 6, None, msg, 480)
        assert st == _lib.INVALID, (k, msg.value)


def test_static_calls_take_no_device_memory():
    # Once warm (both layouts of b, so every kernel is loaded), a call of a
    # new shape leaves the device's free memory as it was.
    import torch

    rng = np.random.default_rng(5)
    for transposed in (0, 1):
        a = rng.uniform(-1, 1, (1, 100, 300))
        b = rng.uniform(-1, 1, (1, 300, 90))
        bb = np.ascontiguousarray(b.transpose(0, 2, 1)) if transposed else b
        _product(True, a, bb, 1, 100, 90, 300, transposed)
    lib = _lib.load()
    m, n, k = 257, 190, 700
    ta = torch.from_numpy(rng.uniform(-1, 1, (m, k))).cuda()
    tb = torch.from_numpy(rng.uniform(-1, 1, (k, n))).cuda()
    tc = torch.zeros((m, n), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    msg = ctypes.create_string_buffer(480)
    st = lib.einfold_split_gemm_static(ta.data_ptr(), tb.data_ptr(), tc.data_ptr(), 1, m, n, k, 0, 6, None, msg, 480)
    assert st == _lib.OK, msg.value.decode()
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
    want = ta.cpu().numpy() @ tb.cpu().numpy()
    tol = split_bound(k, np.abs(ta.cpu().numpy()).max(1), np.abs(tb.cpu().numpy()).max(0)) + \
        2 * k * 2.0 ** -53 * (np.abs(ta.cpu().numpy()) @ np.abs(tb.cpu().numpy()))
    assert (np.abs(tc.cpu().numpy() - want) <= 2 * tol).all()


def test_static_call_before_any_other_in_a_fresh_process():
    # The static entry point as a process's first call into the library
    # (no context, no einfold_split_gemm before it), then the allocating
    # entry point on the same operands: the same values within the bound.
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    code = textwrap.dedent("""
        import ctypes, sys
        import numpy as np, torch
        sys.path.insert(0, %r)
        from einfold_b200 import _lib
        from tests.tables import split_bound
        lib = _lib.load()
        rng = np.random.default_rng(9)
        m, n, k = 130, 70, 515
        a = rng.uniform(-1, 1, (m, k)); b = rng.uniform(-1, 1, (k, n))
        ta, tb = torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda()
        c1 = torch.full((m, n), float("nan"), dtype=torch.float64, device="cuda")
        c2 = torch.full((m, n), float("nan"), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        msg = ctypes.create_string_buffer(480)
        st = lib.einfold_split_gemm_static(ta.data_ptr(), tb.data_ptr(), c1.data_ptr(), 1, m, n, k, 0, 6, None, msg, 480)
        assert st == 0, msg.value
        st = lib.einfold_split_gemm(_lib.context(0), ta.data_ptr(), tb.data_ptr(), c2.data_ptr(), 1, m, n, k, 0, 6, None)
        assert st == 0, lib.einfold_last_error()
        torch.cuda.synchronize()
        tol = split_bound(k, np.abs(a).max(1), np.abs(b).max(0)) + 2 * k * 2.0 ** -53 * (np.abs(a) @ np.abs(b))
        g1, g2 = c1.cpu().numpy(), c2.cpu().numpy()
        assert (np.abs(g1 - g2) <= tol).all() and (np.abs(g1 - a @ b) <= 2 * tol).all()
        print("ok")
    """) % root
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600, cwd=root)
    assert r.returncode == 0 and "ok" in r.stdout, r.stdout[-2000:] + r.stderr[-4000:]

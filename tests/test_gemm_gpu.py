"""The dense products through the C ABI's device entry points."""
import ctypes

import numpy as np
import pytest

from einfold_b200 import _lib
from tests.tables import split_bound

pytestmark = pytest.mark.gpu


def _run(name, a, b, batches, m, n, k, b_transposed, slices=None):
    import torch

    lib = _lib.load()
    ta = torch.from_numpy(a).cuda()
    tb = torch.from_numpy(b).cuda()
    tc = torch.full((batches, m, n), float("nan"), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    ctx = _lib.context(0)
    if name == "split":
        st = lib.einfold_split_gemm(ctx, ta.data_ptr(), tb.data_ptr(), tc.data_ptr(), batches, m, n, k, b_transposed,
                                    slices or 0, None)
    else:
        st = lib.einfold_fp64_gemm(ctx, ta.data_ptr(), tb.data_ptr(), tc.data_ptr(), batches, m, n, k, b_transposed,
                                   None)
    assert st == _lib.OK, lib.einfold_last_error()
    return tc.cpu().numpy()


@pytest.mark.parametrize("shape", [(1, 128, 64, 64), (1, 300, 200, 1000), (3, 129, 65, 257), (1, 1024, 1024, 4096)])
@pytest.mark.parametrize("transposed", [0, 1])
def test_split_product_within_its_bound(shape, transposed):
    batches, m, n, k = shape
    rng = np.random.default_rng(7)
    a = rng.uniform(-1, 1, (batches, m, k))
    b = rng.uniform(-1, 1, (batches, k, n))
    bb = np.ascontiguousarray(b.transpose(0, 2, 1)) if transposed else b
    c = _run("split", a, bb, batches, m, n, k, transposed)
    for w in range(batches):
        ref = a[w] @ b[w]
        err = np.abs(c[w] - ref)
        tol = split_bound(k, np.abs(a[w]).max(1), np.abs(b[w]).max(0)) + 2 * k * 2.0 ** -53 * (np.abs(a[w]) @ np.abs(b[w]))
        assert (err <= tol).all(), (err.max(), (err > tol).sum())
        assert err.max() / np.abs(ref).max() <= 1e-12


def test_split_product_on_wide_ranges_and_zero_rows():
    rng = np.random.default_rng(8)
    m, n, k = 200, 100, 333
    a = rng.standard_normal((1, m, k)) * np.exp(rng.uniform(-30, 30, (1, m, 1)))
    b = rng.standard_normal((1, k, n)) * np.exp(rng.uniform(-30, 30, (1, 1, n)))
    a[0, 5, :] = 0.0
    b[0, :, 7] = 0.0
    c = _run("split", a, b, 1, m, n, k, 0)
    ref = a[0] @ b[0]
    tol = split_bound(k, np.abs(a[0]).max(1), np.abs(b[0]).max(0)) + 2 * k * 2.0 ** -53 * (np.abs(a[0]) @ np.abs(b[0]))
    assert (np.abs(c[0] - ref) <= tol).all()
    assert (c[0, 5, :] == 0).all() and (c[0, :, 7] == 0).all()


@pytest.mark.parametrize("slices", [3, 4, 5, 7])
def test_more_slices_less_error(slices):
    rng = np.random.default_rng(9)
    m, n, k = 256, 128, 512
    a = rng.uniform(-1, 1, (1, m, k))
    b = rng.uniform(-1, 1, (1, k, n))
    c = _run("split", a, b, 1, m, n, k, 0, slices=slices)
    ref = a[0] @ b[0]
    tol = split_bound(k, np.abs(a[0]).max(1), np.abs(b[0]).max(0), slices) + 2 * k * 2.0 ** -53 * (np.abs(a[0]) @ np.abs(b[0]))
    assert (np.abs(c[0] - ref) <= tol).all()


def test_split_product_same_bits_twice():
    rng = np.random.default_rng(10)
    a = rng.uniform(-1, 1, (1, 384, 700))
    b = rng.uniform(-1, 1, (1, 700, 320))
    c1 = _run("split", a, b, 1, 384, 320, 700, 0)
    c2 = _run("split", a, b, 1, 384, 320, 700, 0)
    assert np.array_equal(c1.view(np.uint64), c2.view(np.uint64))


def test_fp64_product_is_in_k_order():
    rng = np.random.default_rng(11)
    m, n, k = 70, 50, 90
    a = rng.uniform(-1, 1, (1, m, k))
    b = rng.uniform(-1, 1, (1, k, n))
    c = _run("fp64", a, b, 1, m, n, k, 0)
    ref = np.zeros((m, n))
    for z in range(k):
        ref = ref + a[0, :, z:z + 1] * b[0, z:z + 1, :]
    assert np.array_equal(c[0].view(np.uint64), ref.view(np.uint64))

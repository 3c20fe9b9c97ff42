"""The dense backend entry points (DenseBackend::run, backend.rs:124-143)
on the GPU: products and attention from operands packed in host memory, as
the trait hands them, and from operands already in HBM, against numpy and
torch float64; ranges that no conditions give are declined (Ok(None))."""
import ctypes

import numpy as np
import pytest

from einfold_b200 import _lib
from tests.tables import split_bound

pytestmark = pytest.mark.gpu


def _run(work, out):
    lib = _lib.load()
    info = _lib.Result()
    return lib.einfold_backend_run(_lib.context(0), ctypes.byref(work), out, ctypes.byref(info)), info


def _product_work(a, b, device, precision=0):
    w, x, z = a.shape
    y = b.shape[2]
    work = _lib.DenseWork()
    work.shape = _lib.DenseShape(0, 0, w, x, z, y, 0)
    work.precision = precision
    work.device = device
    return work


@pytest.mark.parametrize("precision", [0, 1])
def test_products_from_host_memory(precision):
    rng = np.random.default_rng(1)
    a = rng.uniform(-1, 1, (3, 70, 130))
    b = rng.uniform(-1, 1, (3, 130, 45))
    out = np.full((3, 70, 45), np.nan)
    work = _product_work(a, b, -1, precision)
    work.a, work.b = a.ctypes.data, b.ctypes.data
    st, info = _run(work, out.ctypes.data)
    assert st == _lib.OK, info.message
    want = a @ b
    for i in range(3):
        tol = split_bound(130, np.abs(a[i]).max(1), np.abs(b[i]).max(0)) + 2 * 130 * 2.0 ** -53 * (np.abs(a[i]) @ np.abs(b[i]))
        assert (np.abs(out[i] - want[i]) <= tol).all()


def test_products_from_device_memory():
    import torch

    rng = np.random.default_rng(2)
    a = torch.from_numpy(rng.uniform(-1, 1, (2, 64, 96))).cuda()
    b = torch.from_numpy(rng.uniform(-1, 1, (2, 96, 33))).cuda()
    out = torch.full((2, 64, 33), float("nan"), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    work = _product_work(a, b, 0)
    work.a, work.b = a.data_ptr(), b.data_ptr()
    st, info = _run(work, out.data_ptr())
    assert st == _lib.OK, info.message
    assert torch.allclose(out, a @ b, rtol=0, atol=1e-12)


def _attention_work(q, kt, v, ranges, scale_kind=0, scale_c=1.0):
    w, x, e = q.shape
    j, y = v.shape[1], v.shape[2]
    work = _lib.DenseWork()
    work.shape = _lib.DenseShape(1, 0, w, x, e, y, j)
    work.q, work.kt, work.v = q.ctypes.data, kt.ctypes.data, v.ctypes.data
    work.scale_kind, work.scale_c = scale_kind, scale_c
    work.allowed = ranges.ctypes.data
    work.device = -1
    return work


def _torch_attention(q, kt, v, ranges, scale):
    import torch

    q, kt, v = (torch.from_numpy(t) for t in (q, kt, v))
    s = scale * (q @ kt)
    j = torch.arange(s.shape[-1])[None, :]
    lo, hi = torch.from_numpy(ranges[:, 0])[:, None], torch.from_numpy(ranges[:, 1])[:, None]
    allowed = (j >= lo) & (j < hi)
    out = torch.softmax(s.masked_fill(~allowed, float("-inf")), -1) @ v
    return torch.where(allowed.any(-1)[:, None], out, torch.zeros_like(out)).numpy()


@pytest.mark.parametrize("shape", ["causal", "window", "late_start", "full"])
def test_attention_from_host_memory(shape):
    rng = np.random.default_rng(3)
    w, x, e, j, y = 2, 150, 32, 150, 24
    q = rng.normal(0, 0.3, (w, x, e))
    kt = rng.normal(0, 0.3, (w, e, j))
    v = rng.normal(0, 1, (w, j, y))
    xs = np.arange(x)
    lo, hi = {"causal": (np.zeros(x), xs + 1), "window": (xs - 10, xs + 11), "late_start": (np.zeros(x), xs - 19),
              "full": (np.zeros(x), np.full(x, j))}[shape]
    ranges = np.ascontiguousarray(np.stack([np.clip(lo, 0, j), np.clip(hi, 0, j)], 1).astype(np.int64))
    scale_kind, scale = (1, 0.5) if shape == "window" else (0, 1.0)
    out = np.full((w, x, y), np.nan)
    st, info = _run(_attention_work(q, kt, v, ranges, scale_kind, scale), out.ctypes.data)
    assert st == _lib.OK, info.message
    want = _torch_attention(q, kt, v, ranges, scale)
    assert np.abs(out - want).max() <= 1e-12 * np.abs(v).max()


def test_ranges_no_conditions_give_are_declined():
    rng = np.random.default_rng(4)
    w, x, e, j, y = 1, 20, 8, 20, 4
    q, kt, v = rng.normal(0, 1, (w, x, e)), rng.normal(0, 1, (w, e, j)), rng.normal(0, 1, (w, j, y))
    ranges = np.stack([np.zeros(x), np.where(np.arange(x) % 2 == 0, 5, 9)], 1).astype(np.int64)
    out = np.zeros((w, x, y))
    st, _ = _run(_attention_work(q, kt, v, np.ascontiguousarray(ranges)), out.ctypes.data)
    assert st == _lib.DECLINED

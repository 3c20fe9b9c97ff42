"""Radix ranking on the GPU against the oracle's restatement of `radix` and
`ranks_of_words` (discriminate.rs:103-156, 280-292): bit-exact ranks and
first rows."""
import ctypes

import numpy as np
import pytest

from einfold_b200 import _lib
from oracle import oracle

pytestmark = pytest.mark.gpu


def _rank(words: np.ndarray):
    import torch

    lib = _lib.load()
    n = len(words)
    w = torch.from_numpy(words.view(np.int64)).cuda() if n else torch.zeros(1, dtype=torch.int64, device="cuda")
    rank = torch.zeros(max(n, 1), dtype=torch.int32, device="cuda")
    first = torch.zeros(max(n, 1), dtype=torch.int32, device="cuda")
    k = ctypes.c_int64(-1)
    torch.cuda.synchronize()
    st = lib.einfold_rank_words(_lib.context(0), w.data_ptr(), n, rank.data_ptr(), first.data_ptr(), ctypes.byref(k),
                                None)
    assert st == _lib.OK, lib.einfold_last_error()
    return rank.cpu().numpy()[:n].view(np.uint32), first.cpu().numpy()[: k.value].view(np.uint32), k.value


def _check(words):
    got_rank, got_first, k = _rank(words)
    want = oracle.ranks_of_words(words)
    assert k == len(want.first)
    assert np.array_equal(got_rank, want.rank)
    assert np.array_equal(got_first, want.first)
    # And what the ranks mean, independently of both implementations.
    u, first_idx, inv = np.unique(words, return_index=True, return_inverse=True)
    assert np.array_equal(got_rank, inv.astype(np.uint32))
    assert np.array_equal(got_first, first_idx.astype(np.uint32))


@pytest.mark.parametrize("n", [1, 2, 31, 4095, 4096, 4097, 100_003])
def test_random_words_with_duplicates(n):
    rng = oracle.Rng.seeded(n, 1)
    pool = rng.u64s(max(n // 3, 1))
    words = pool[(rng.u64s(n) % np.uint64(len(pool))).astype(np.int64)]
    _check(words)


def test_signed_keys_order_by_their_value():
    rng = oracle.Rng.seeded(5, 2)
    keys = (rng.u64s(50_000) % np.uint64(2001)).astype(np.int64) - 1000
    words = keys.view(np.uint64) ^ np.uint64(1 << 63)
    _check(words)
    got_rank, got_first, k = _rank(words)
    assert k == len(np.unique(keys))
    order = np.argsort(got_rank, kind="stable")
    assert np.all(np.diff(keys[order]) >= 0)


def test_all_equal_and_few_varying_bytes():
    _check(np.full(10_000, 0xDEADBEEF00000000, dtype=np.uint64))
    rng = oracle.Rng.seeded(6, 3)
    low = rng.u64s(70_000) & np.uint64(0xFF)
    _check((low << np.uint64(40)) | np.uint64(0x1234))


def test_zipf_hashes_at_the_sorting_paths_size():
    # 4M keys over a 200k pool of 63-bit hashes with Zipf(1.1) frequencies.
    rng = oracle.Rng.seeded(0, 7)
    pool = rng.u64s(200_000) >> np.uint64(1)
    ranks = np.arange(1, len(pool) + 1, dtype=np.float64)
    p = ranks ** -1.1
    cdf = np.cumsum(p / p.sum())
    pick = np.searchsorted(cdf, rng.units(4_000_000), side="right").clip(0, len(pool) - 1)
    keys = pool[pick].view(np.int64)
    words = keys.view(np.uint64) ^ np.uint64(1 << 63)
    _check(words)


def test_more_than_4m_rows():
    # Rank and first arrays beyond L2, chunks of many tiles.
    n = (1 << 22) + 12_345
    rng = oracle.Rng.seeded(9, 4)
    pool = rng.u64s(n // 2)
    words = pool[(rng.u64s(n) % np.uint64(len(pool))).astype(np.int64)]
    _check(words)


@pytest.mark.parametrize("order", ["ascending", "descending", "three_values"])
def test_ordered_and_heavily_repeated_keys(order):
    # Every tile of a pass holding one digit only, or the same few: the
    # look-back across tiles carries whole runs.
    n = 3_000_017
    rng = oracle.Rng.seeded(10, 5)
    if order == "three_values":
        words = np.array([7, 1 << 40, (1 << 63) + 5], dtype=np.uint64)[(rng.u64s(n) % np.uint64(3)).astype(np.int64)]
    else:
        words = np.sort(rng.u64s(n))
        if order == "descending":
            words = words[::-1].copy()
    _check(words)


def test_keys_not_16_byte_aligned():
    # The passes read keys by TMA bulk copies, which want 16-byte aligned
    # sources: keys starting 8 bytes past an alignment are copied first.
    import torch

    rng = oracle.Rng.seeded(12, 6)
    n = 50_001
    words = rng.u64s(n + 1) % np.uint64(7919)
    lib = _lib.load()
    w = torch.from_numpy(words.view(np.int64)).cuda()
    rank = torch.zeros(n, dtype=torch.int32, device="cuda")
    first = torch.zeros(n, dtype=torch.int32, device="cuda")
    k = ctypes.c_int64(-1)
    torch.cuda.synchronize()
    st = lib.einfold_rank_words(_lib.context(0), w.data_ptr() + 8, n, rank.data_ptr(), first.data_ptr(),
                                ctypes.byref(k), None)
    assert st == _lib.OK, lib.einfold_last_error()
    want = oracle.ranks_of_words(words[1:])
    assert np.array_equal(rank.cpu().numpy().view(np.uint32), want.rank)
    assert np.array_equal(first.cpu().numpy()[: k.value].view(np.uint32), want.first)

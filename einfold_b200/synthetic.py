"""Seeded synthetic tables for the benchmarks, generated on the device.

Values come from SplitMix64 as einfold's test kit draws them
(``crates/einfold-testkit/src/rng.rs:17-43``): ``Rng::seeded(seed, salt)``
then one ``next_u64`` per value, so draw ``i`` is the mix of
``state0 + (i + 1)·γ``. Computed here in parallel with torch int64
arithmetic (wrapping), with logical shifts made by masking.
"""
from __future__ import annotations

import torch

_GAMMA = 0x9E3779B97F4A7C15
_M1 = 0xBF58476D1CE4E5B9
_M2 = 0x94D049BB133111EB
_MASK64 = (1 << 64) - 1


def _signed(x: int) -> int:
    x &= _MASK64
    return x - (1 << 64) if x >= 1 << 63 else x


def _srl(z: torch.Tensor, k: int) -> torch.Tensor:
    """Logical right shift of int64 bit patterns."""
    return (z >> k) & ((1 << (64 - k)) - 1)


def state(seed: int, salt: int) -> int:
    return ((seed * 0x2545F4914F6CDD1D) & _MASK64) ^ salt


def u64(seed: int, salt: int, n: int, start: int = 0, device="cuda") -> torch.Tensor:
    """Draws start .. start+n of Rng::seeded(seed, salt), as int64 bit patterns."""
    s0 = state(seed, salt)
    i = torch.arange(start + 1, start + n + 1, dtype=torch.int64, device=device)
    z = i * _signed(_GAMMA) + _signed(s0)
    z = (z ^ _srl(z, 30)) * _signed(_M1)
    z = (z ^ _srl(z, 27)) * _signed(_M2)
    return z ^ _srl(z, 31)


def units(seed: int, salt: int, n: int, start: int = 0, device="cuda") -> torch.Tensor:
    """``Rng::unit`` draws: 53 random bits in [0, 1), as float64."""
    z = u64(seed, salt, n, start, device)
    return _srl(z, 11).to(torch.float64) * (1.0 / float(1 << 53))


def uniform(seed: int, salt: int, n: int, lo: float = -1.0, hi: float = 1.0, device="cuda") -> torch.Tensor:
    return units(seed, salt, n, 0, device) * (hi - lo) + lo


def normal(seed: int, salt: int, n: int, std: float = 1.0, device="cuda") -> torch.Tensor:
    """Normal draws by Box-Muller over pairs of unit draws."""
    m = (n + 1) // 2
    u = units(seed, salt, 2 * m, 0, device)
    u1 = 1.0 - u[0::2]  # (0, 1]
    u2 = u[1::2]
    r = torch.sqrt(-2.0 * torch.log(u1))
    t = 2.0 * torch.pi * u2
    out = torch.empty(2 * m, dtype=torch.float64, device=device)
    out[0::2] = r * torch.cos(t)
    out[1::2] = r * torch.sin(t)
    return out[:n] * std


def grid_keys(extents, device="cuda"):
    """Every key tuple of the extents, first dimension slowest, one int64 tensor per dimension."""
    n = 1
    for e in extents:
        n *= e
    idx = torch.arange(n, dtype=torch.int64, device=device)
    out = []
    stride = n
    for e in extents:
        stride //= e
        out.append((idx // stride) % e)
    return out


# ---- The sorting path's tables (string and hash keys, Zipf joins) --------


def _np_units(seed: int, salt: int, n: int):
    import numpy as np

    return units(seed, salt, n, device="cpu").numpy().astype(np.float64)


def hex_strings(words):
    """16 lower-case hex digits of each 64-bit word, as an Arrow string array
    built from one buffer (no Python loop over the rows)."""
    import numpy as np
    import pyarrow as pa

    w = np.ascontiguousarray(words, dtype=np.uint64)
    nib = np.empty((len(w), 16), dtype=np.uint8)
    for d in range(16):
        nib[:, d] = ((w >> np.uint64(4 * (15 - d))) & np.uint64(15)).astype(np.uint8)
    digits = np.frombuffer(b"0123456789abcdef", dtype=np.uint8)[nib]
    offsets = np.arange(0, 16 * (len(w) + 1), 16, dtype=np.int32)
    return pa.StringArray.from_buffers(len(w), pa.py_buffer(offsets.tobytes()), pa.py_buffer(digits.tobytes()))


def _zipf_picks(seed: int, salt: int, n: int, pool: int, s: float = 1.1):
    """n indices into a pool, index r drawn with frequency proportional to (r + 1)^-s."""
    import numpy as np

    cdf = np.cumsum(np.arange(1, pool + 1, dtype=np.float64) ** -s)
    cdf /= cdf[-1]
    return np.searchsorted(cdf, _np_units(seed, salt, n), side="right").clip(0, pool - 1)


def _np_normal(seed: int, salt: int, n: int):
    import numpy as np

    u1, u2 = _np_units(seed, salt, n), _np_units(seed, salt + 100, n)
    return np.sqrt(-2.0 * np.log1p(-u1)) * np.cos(2 * np.pi * u2)


def sorting_tables(rows: int = 2_000_000, pool: int = 200_000, names: int = 50_000, seed: int = 0):
    """The sparse contraction's tables with non-positional keys: a(i, j, v)
    and b(j, k, v), `rows` rows each; i and k 16-hex-digit strings drawn
    uniformly from `names` distinct, j a 63-bit hash from a pool of `pool`
    drawn with Zipf(1.1) frequencies (the same pool and law for a and b),
    v normal(0, 1). SplitMix64 (seed, salts 11-19). Returns the two record
    batches."""
    import numpy as np
    import pyarrow as pa

    hashes = (u64(seed, 13, pool, device="cpu").numpy().view(np.uint64) >> np.uint64(1)).astype(np.int64)
    ia = u64(seed, 11, names, device="cpu").numpy().view(np.uint64)
    kb = u64(seed, 12, names, device="cpu").numpy().view(np.uint64)
    pick_a = (_np_units(seed, 14, rows) * names).astype(np.int64).clip(0, names - 1)
    pick_b = (_np_units(seed, 15, rows) * names).astype(np.int64).clip(0, names - 1)
    ja = hashes[_zipf_picks(seed, 16, rows, pool)]
    jb = hashes[_zipf_picks(seed, 17, rows, pool)]
    a = pa.record_batch([hex_strings(ia[pick_a]), pa.array(ja), pa.array(_np_normal(seed, 18, rows))],
                        names=["i", "j", "v"])
    b = pa.record_batch([pa.array(jb), hex_strings(kb[pick_b]), pa.array(_np_normal(seed, 19, rows))],
                        names=["j", "k", "v"])
    return a, b


def regrid_table(rows: int = 4_000_000, pool: int = 200_000, targets: int = 50_000, seed: int = 0):
    """The regridding variant's weight table w(src, dst, wt): `rows` rows,
    src from the sorting tables' hash pool with Zipf(1.1) frequencies, dst
    an int64 cell id from `targets` distinct, wt uniform[0, 1). SplitMix64
    (seed, salts 13 for the pool, 21-24)."""
    import numpy as np
    import pyarrow as pa

    hashes = (u64(seed, 13, pool, device="cpu").numpy().view(np.uint64) >> np.uint64(1)).astype(np.int64)
    cells = (u64(seed, 21, targets, device="cpu").numpy().view(np.uint64) >> np.uint64(20)).astype(np.int64)
    src = hashes[_zipf_picks(seed, 22, rows, pool)]
    dst = cells[(_np_units(seed, 23, rows) * targets).astype(np.int64).clip(0, targets - 1)]
    return pa.record_batch([pa.array(src), pa.array(dst), pa.array(_np_units(seed, 24, rows))],
                           names=["src", "dst", "wt"])


def joined_pairs(left_keys, right_keys) -> int:
    """The number of (left row, right row) pairs with equal keys."""
    import numpy as np

    ua, ca = np.unique(np.asarray(left_keys), return_counts=True)
    ub, cb = np.unique(np.asarray(right_keys), return_counts=True)
    _, xa, xb = np.intersect1d(ua, ub, return_indices=True)
    return int((ca[xa].astype(np.int64) * cb[xb].astype(np.int64)).sum())

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

"""Philox4x32-10 uniform stream on the host (numpy, vectorised).

Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy as 1, 2, 3",
SC'11.  Draw ``i`` of stream ``stream`` under key ``seed`` uses counter
(lo32(i//2), hi32(i//2), stream, 0); even draws take output words (0,1),
odd draws words (2,3); the 64-bit word hi<<32|lo keeps its top 53 bits as
u = (w >> 11) * 2^-53.  The CUDA library (rq_uniform, the sampling kernel)
computes exactly the same stream, so host-generated workloads, device
measurement draws and the tests all share one documented generator.
"""
from __future__ import annotations

import numpy as np

_M0 = np.uint64(0xD2511F53)
_M1 = np.uint64(0xCD9E8D57)
_W0 = 0x9E3779B9
_W1 = 0xBB67AE85
_MASK32 = np.uint64(0xFFFFFFFF)


def philox4x32_10(c0, c1, c2, c3, k0: int, k1: int):
    """Vectorised Philox4x32-10 over uint32 counter arrays; returns 4 uint32 arrays."""
    c0 = np.asarray(c0, dtype=np.uint64)
    c1 = np.asarray(c1, dtype=np.uint64)
    c2 = np.asarray(c2, dtype=np.uint64)
    c3 = np.asarray(c3, dtype=np.uint64)
    for r in range(10):
        if r > 0:
            k0 = (k0 + _W0) & 0xFFFFFFFF
            k1 = (k1 + _W1) & 0xFFFFFFFF
        p0 = _M0 * c0
        p1 = _M1 * c2
        n0 = (p1 >> np.uint64(32)) ^ c1 ^ np.uint64(k0)
        n1 = p1 & _MASK32
        n2 = (p0 >> np.uint64(32)) ^ c3 ^ np.uint64(k1)
        n3 = p0 & _MASK32
        c0, c1, c2, c3 = n0, n1, n2, n3
    return (c0.astype(np.uint32), c1.astype(np.uint32), c2.astype(np.uint32), c3.astype(np.uint32))


def uniforms(seed: int, stream: int, start: int, count: int) -> np.ndarray:
    """Draws start .. start+count-1 of (seed, stream) as float64 in [0, 1)."""
    idx = np.arange(start, start + count, dtype=np.uint64)
    blk = idx >> np.uint64(1)
    seed &= (1 << 64) - 1
    x0, x1, x2, x3 = philox4x32_10(blk & _MASK32, blk >> np.uint64(32), np.full_like(blk, stream),
                                   np.zeros_like(blk), seed & 0xFFFFFFFF, seed >> 32)
    odd = (idx & np.uint64(1)).astype(bool)
    hi = np.where(odd, x2, x0).astype(np.uint64)
    lo = np.where(odd, x3, x1).astype(np.uint64)
    w = (hi << np.uint64(32)) | lo
    return (w >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def uniforms_keys(seeds, stream: int, index: int) -> np.ndarray:
    """Draw ``index`` of (seed, stream) for every seed of an array (one shot per key, the
    way shot s of a run draws from key base_seed + s)."""
    seeds = np.asarray(seeds, dtype=np.uint64)
    blk = int(index) >> 1
    x0, x1, x2, x3 = philox4x32_10(np.full(seeds.shape, blk & 0xFFFFFFFF, dtype=np.uint64),
                                   np.full(seeds.shape, blk >> 32, dtype=np.uint64),
                                   np.full(seeds.shape, stream, dtype=np.uint64), np.zeros(seeds.shape, dtype=np.uint64),
                                   seeds & _MASK32, seeds >> np.uint64(32))
    if int(index) & 1:
        hi, lo = x2.astype(np.uint64), x3.astype(np.uint64)
    else:
        hi, lo = x0.astype(np.uint64), x1.astype(np.uint64)
    w = (hi << np.uint64(32)) | lo
    return (w >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


class Stream:
    """Sequential reader of one (seed, stream) pair."""

    def __init__(self, seed: int, stream: int):
        self.seed = seed
        self.stream = stream
        self.pos = 0

    def take(self, count: int) -> np.ndarray:
        u = uniforms(self.seed, self.stream, self.pos, count)
        self.pos += count
        return u

    def one(self) -> float:
        return float(self.take(1)[0])

    def normal(self, count: int) -> np.ndarray:
        """Standard normals by Box-Muller over pairs of draws (u1 mapped to (0,1])."""
        m = (count + 1) // 2
        u = self.take(2 * m)
        u1 = 1.0 - u[0::2]
        u2 = u[1::2]
        r = np.sqrt(-2.0 * np.log(u1))
        z = np.concatenate([r * np.cos(2 * np.pi * u2), r * np.sin(2 * np.pi * u2)])
        out = np.empty(2 * m)
        out[0::2] = z[:m]
        out[1::2] = z[m:]
        return out[:count]

    def randint(self, high: int) -> int:
        """Uniform integer in [0, high) (floor of u*high)."""
        return min(int(self.one() * high), high - 1)

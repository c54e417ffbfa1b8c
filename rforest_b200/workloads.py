"""Seeded synthetic workloads for the exact matrix product.

Every input comes from splitmix64 (Steele, Lea and Flood, "Fast splittable
pseudorandom number generators", OOPSLA 2014), used as a counter-based stream:
output ``i`` of the stream with seed ``s`` is ``mix64(s + (i + 1) * GAMMA)``,
which is what the sequential generator returns on its ``i``-th call.  That
makes every draw addressable, so whole matrices are generated with vectorised
numpy and the same entry is reproducible in isolation.

Streams used (``sub(seed, tag) = mix64(seed + tag * 0xD1B54A32D192ED03)``):

* dims of product t:        stream ``sub(seed, 1)``, draws 3t, 3t+1, 3t+2
* bit length of product t:  stream ``sub(seed, 2)``, draws 2t, 2t+1
* entry e of side s (0 = A, 1 = B) of product t: its own stream with seed
  ``mix64(sub(seed, 3) + ((2t + s) * 2^20 + e + 1) * GAMMA)``; draws
  0 .. nl-1 are the limbs (top limb masked to L bits), draw nl is the sign bit
  (a zero magnitude stays zero).
* Poisson arrival gaps: stream ``sub(seed, 4)``, draw t.

A uniform integer in [lo, hi] is ``lo + (((x >> 32) * (hi - lo + 1)) >> 32)``.
A log-uniform bit length in [2^a, 2^b] takes e uniform in [a, b) and then L
uniform in [2^e, 2^(e+1)), all in integers.  The bit length is drawn once per
product: every entry of that product has magnitude uniform in [0, 2^L).
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import List, Optional

import numpy as np

from .packed import Packed, concat

GAMMA = 0x9E3779B97F4A7C15
SUBC = 0xD1B54A32D192ED03
M1 = 0xBF58476D1CE4E5B9
M2 = 0x94D049BB133111EB
MASK = (1 << 64) - 1


def mix64(z: int) -> int:
    z &= MASK
    z = ((z ^ (z >> 30)) * M1) & MASK
    z = ((z ^ (z >> 27)) * M2) & MASK
    return z ^ (z >> 31)


def sub(seed: int, tag: int) -> int:
    return mix64(seed + tag * SUBC)


def draw(seed: int, i: int) -> int:
    return mix64(seed + (i + 1) * GAMMA)


def _mix_vec(z: np.ndarray) -> np.ndarray:
    with np.errstate(over="ignore"):
        z = (z ^ (z >> np.uint64(30))) * np.uint64(M1)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(M2)
        return z ^ (z >> np.uint64(31))


def draws_vec(seeds: np.ndarray, count: int) -> np.ndarray:
    """[len(seeds), count] matrix of draws 0..count-1 of each seed's stream."""
    idx = (np.arange(1, count + 1, dtype=np.uint64) * np.uint64(GAMMA))
    with np.errstate(over="ignore"):
        z = seeds.astype(np.uint64)[:, None] + idx[None, :]
    return _mix_vec(z)


def uniform_int(x: int, lo: int, hi: int) -> int:
    return lo + (((x >> 32) * (hi - lo + 1)) >> 32)


def log_uniform_bits(x: int, y: int, a: int, b: int) -> int:
    e = a + (((x >> 32) * (b - a)) >> 32)
    return (1 << e) + (((y >> 32) << e) >> 32)


def entry_seeds(seed: int, t: int, side: int, count: int) -> np.ndarray:
    base = sub(seed, 3)
    out = np.empty(count, dtype=np.uint64)
    for e in range(count):
        out[e] = mix64(base + (((2 * t + side) << 20) + e + 1) * GAMMA)
    return out


def random_matrix(seed: int, t: int, side: int, rows: int, cols: int, bits: int,
                  signed: bool) -> Packed:
    """rows x cols entries, magnitudes uniform in [0, 2^bits), row-major."""
    cnt = rows * cols
    nl = (bits + 63) // 64
    seeds = entry_seeds(seed, t, side, cnt)
    d = draws_vec(seeds, nl + 1)
    limbs = d[:, :nl].copy()
    if bits % 64:
        limbs[:, nl - 1] &= np.uint64((1 << (bits % 64)) - 1)
    # effective sizes (strip high zero limbs)
    nz = limbs != 0
    any_nz = nz.any(axis=1)
    top = np.where(any_nz, nl - np.argmax(nz[:, ::-1], axis=1), 0).astype(np.int32)
    sign = (d[:, nl] & np.uint64(1)).astype(bool) if signed else np.zeros(cnt, bool)
    sizes = np.where(sign, -top, top).astype(np.int32)
    offs = (np.arange(cnt, dtype=np.int64) * nl)
    return Packed(limbs.reshape(-1), offs, sizes)


@dataclass
class Product:
    m: int
    k: int
    n: int
    A: Packed
    B: Packed
    bits: int

    @property
    def shape(self):
        return (self.m, self.k, self.n)


def fixed_product(seed: int, t: int, m: int, k: int, n: int, bits: int,
                  signed: bool) -> Product:
    A = random_matrix(seed, t, 0, m, k, bits, signed)
    B = random_matrix(seed, t, 1, k, n, bits, signed)
    return Product(m, k, n, A, B, bits)


def product_params(seed: int, t: int, dim_lo: int, dim_hi: int, lg_lo: int,
                   lg_hi: int):
    ds = sub(seed, 1)
    m = uniform_int(draw(ds, 3 * t), dim_lo, dim_hi)
    k = uniform_int(draw(ds, 3 * t + 1), dim_lo, dim_hi)
    n = uniform_int(draw(ds, 3 * t + 2), dim_lo, dim_hi)
    bs = sub(seed, 2)
    bits = log_uniform_bits(draw(bs, 2 * t), draw(bs, 2 * t + 1), lg_lo, lg_hi)
    return m, k, n, bits


def random_product(seed: int, t: int, dim_lo: int, dim_hi: int, lg_lo: int,
                   lg_hi: int, signed: bool = True) -> Product:
    m, k, n, bits = product_params(seed, t, dim_lo, dim_hi, lg_lo, lg_hi)
    return fixed_product(seed, t, m, k, n, bits, signed)


# ---------------------------------------------------------------------------
# The five workloads (seed = workload id * 1000 + replicate)
# ---------------------------------------------------------------------------

def config1(replicate: int = 1) -> Product:
    """4x4 by 4x4, signed entries with magnitudes in [0, 2^4096)."""
    return fixed_product(1000 + replicate, 0, 4, 4, 4, 4096, True)


def config2(replicate: int = 1) -> Product:
    """8x8 by 8x8, signed 65536-bit entries."""
    return fixed_product(2000 + replicate, 0, 8, 8, 8, 65536, True)


def config2_chain(replicate: int = 1, length: int = 16) -> List[Packed]:
    """16 signed 8x8 matrices of 65536-bit entries, multiplied left to right."""
    seed = 2000 + replicate
    return [random_matrix(seed, 1 + i, 0, 8, 8, 65536, True) for i in range(length)]


def config3(replicate: int = 1, count: int = 4096, bits_hi_lg: int = 18) -> List[Product]:
    """``count`` products, m,k,n uniform in {2..16}, bit lengths log-uniform in
    [2^10, 2^18], signed."""
    seed = 3000 + replicate
    return [random_product(seed, t, 2, 16, 10, bits_hi_lg) for t in range(count)]


def config3_shapes(replicate: int = 1, count: int = 4096):
    seed = 3000 + replicate
    return [product_params(seed, t, 2, 16, 10, 18) for t in range(count)]


def config4(replicate: int = 1, dim: int = 64, bits: int = 1 << 20) -> Product:
    """64x64 by 64x64, unsigned entries with magnitudes in [0, 2^(2^20))."""
    return fixed_product(4000 + replicate, 0, dim, dim, dim, bits, False)


def config5_shapes(replicate: int = 1, count: int = 100000):
    seed = 5000 + replicate
    return [product_params(seed, t, 2, 32, 8, 20) for t in range(count)]


def config5_request(replicate: int, t: int) -> Product:
    seed = 5000 + replicate
    return random_product(seed, t, 2, 32, 8, 20)


def poisson_arrivals(replicate: int, count: int, rate: float) -> np.ndarray:
    """Arrival times (seconds) of ``count`` requests at ``rate`` per second."""
    seeds = np.array([sub(5000 + replicate, 4)], dtype=np.uint64)
    u = draws_vec(seeds, count)[0]
    # uniform in (0, 1]: top 53 bits, offset by one ulp so log() is finite
    f = ((u >> np.uint64(11)).astype(np.float64) + 1.0) / float(1 << 53)
    gaps = -np.log(f) / rate
    return np.cumsum(gaps)

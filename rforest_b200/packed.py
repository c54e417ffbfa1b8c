"""Packed big-integer vectors: the plain-array form every entry point takes.

A packed vector holds E signed integers.  Entry ``e`` has ``abs(sizes[e])``
64-bit limbs (least significant first) starting at ``limbs[offs[e]]`` and the
sign of ``sizes[e]`` -- exactly GMP's ``(_mp_size, _mp_d)`` convention for an
``mpz_t`` (GMP manual, "Integer Internals"), so an ``mpz_t`` matrix maps onto
it without any re-encoding of limbs.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Iterable, List, Sequence

import numpy as np


def bit_length_u64(x: np.ndarray) -> np.ndarray:
    """Exact bit length of each uint64 (0 for 0)."""
    x = np.array(x, dtype=np.uint64, copy=True)
    b = np.zeros(x.shape, dtype=np.int64)
    for s in (32, 16, 8, 4, 2, 1):
        m = x >= np.uint64(1 << s)
        b[m] += s
        x[m] >>= np.uint64(s)
    return b + (x > 0)


@dataclass
class Packed:
    limbs: np.ndarray  # uint64
    offs: np.ndarray  # int64
    sizes: np.ndarray  # int32 (signed limb count)

    def __len__(self) -> int:
        return int(self.sizes.shape[0])

    @property
    def nlimbs(self) -> np.ndarray:
        return np.abs(self.sizes.astype(np.int64))

    def max_limbs(self) -> int:
        return int(self.nlimbs.max()) if len(self) else 0

    def max_bits(self) -> int:
        """Largest bit length of an entry's magnitude (0 if all are zero)."""
        n = self.nlimbs
        nz = n > 0
        if not nz.any():
            return 0
        top = self.limbs[self.offs[nz] + n[nz] - 1]
        return int((64 * (n[nz] - 1) + bit_length_u64(top)).max())

    def entry(self, e: int) -> int:
        """Entry ``e`` as a Python int."""
        s = int(self.sizes[e])
        n = abs(s)
        if n == 0:
            return 0
        o = int(self.offs[e])
        v = int.from_bytes(self.limbs[o:o + n].astype("<u8").tobytes(), "little")
        return -v if s < 0 else v

    def to_ints(self) -> List[int]:
        return [self.entry(e) for e in range(len(self))]

    def slice(self, start: int, stop: int) -> "Packed":
        return Packed(self.limbs, self.offs[start:stop].copy(), self.sizes[start:stop].copy())

    def compact(self) -> "Packed":
        """Copy with entries stored back to back in entry order."""
        n = self.nlimbs
        offs = np.zeros(len(self), dtype=np.int64)
        if len(self):
            offs[1:] = np.cumsum(n)[:-1]
        out = np.zeros(int(n.sum()), dtype=np.uint64)
        for e in range(len(self)):
            k = int(n[e])
            if k:
                o = int(self.offs[e])
                out[offs[e]:offs[e] + k] = self.limbs[o:o + k]
        return Packed(out, offs, self.sizes.copy())


def from_ints(values: Iterable[int]) -> Packed:
    vals = list(values)
    chunks: List[bytes] = []
    sizes = np.zeros(len(vals), dtype=np.int32)
    offs = np.zeros(len(vals), dtype=np.int64)
    pos = 0
    for e, v in enumerate(vals):
        mag = -v if v < 0 else v
        n = (mag.bit_length() + 63) // 64
        offs[e] = pos
        sizes[e] = -n if v < 0 else n
        if n:
            chunks.append(mag.to_bytes(8 * n, "little"))
        pos += n
    limbs = np.frombuffer(b"".join(chunks), dtype="<u8").astype(np.uint64) if pos else np.zeros(0, np.uint64)
    return Packed(limbs, offs, sizes)


def concat(parts: Sequence[Packed]) -> Packed:
    """One packed vector holding the entries of ``parts`` in order."""
    limbs, offs, sizes = [], [], []
    base = 0
    for p in parts:
        limbs.append(p.limbs)
        offs.append(p.offs + base)
        sizes.append(p.sizes)
        base += int(p.limbs.shape[0])
    return Packed(
        np.concatenate(limbs) if limbs else np.zeros(0, np.uint64),
        np.concatenate(offs) if offs else np.zeros(0, np.int64),
        np.concatenate(sizes) if sizes else np.zeros(0, np.int32),
    )


def output_layout(caps: np.ndarray):
    """Offsets for an output packed vector with per-entry capacities ``caps``."""
    caps = np.asarray(caps, dtype=np.int64)
    offs = np.zeros(caps.shape[0], dtype=np.int64)
    if caps.shape[0]:
        offs[1:] = np.cumsum(caps)[:-1]
    return offs, int(caps.sum())


def product_limb_bound(a: Packed, b: Packed, k: int) -> int:
    """Limbs sufficient for any entry of an m x k by k x n product."""
    la = a.max_limbs()
    lb = b.max_limbs()
    return la + lb + 1 + (max(k, 1).bit_length() + 63) // 64


def digest(p: Packed) -> str:
    """SHA-256 of a canonical serialisation: per entry, its signed size as
    little-endian int32 followed by its normalised limbs."""
    import hashlib
    h = hashlib.sha256()
    n = p.nlimbs
    for e in range(len(p)):
        k = int(n[e])
        o = int(p.offs[e])
        limbs = p.limbs[o:o + k]
        # normalise: drop high zero limbs (size already normalised by producers)
        while k and limbs[k - 1] == 0:
            k -= 1
        s = k if int(p.sizes[e]) >= 0 else -k
        h.update(int(s).to_bytes(4, "little", signed=True))
        h.update(np.ascontiguousarray(limbs[:k], dtype="<u8").tobytes())
    return h.hexdigest()

"""Seeded synthetic traffic for the one-sided path.

One portable RNG for every generator: splitmix64 over a counter,
out_i = splitmix64(seed + i * GOLDEN) with splitmix64 adding GOLDEN first;
normals by Box-Muller.  No public dataset is involved; the shapes follow the
workloads the library is measured on:
  C1  2 PEs, flag ping-pong and a float put sweep 4 B .. 1 MiB (seed 0)
  C2  8 PEs all-to-all, int32/float32/float64 payloads, 8 B .. 256 MiB (seed 1)
  C3  8 PEs on a periodic 2x2x2 grid, 256^3 float64 blocks, N(0,1) (seed 3)
  C4  64 PEs, 100,000 requests per batch, log-normal sizes (median 2 KiB,
      sigma 1.5, clipped to 4 B .. 4 MiB), put 45% / get 45% / signal 10%,
      uniform PE pairs, 16-byte aligned offsets, disjoint destinations (seed 4)
"""
from __future__ import annotations

import numpy as np

from ._abi import (DT_DOUBLE, DT_FLOAT, DT_INT, REQ_GET, REQ_PUT, REQ_SIGNAL,
                   REQUEST_DTYPE)

GOLDEN = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)


def splitmix64(x: np.ndarray) -> np.ndarray:
    x = np.asarray(x, dtype=np.uint64)
    with np.errstate(over="ignore"):
        x = x + GOLDEN
        x = (x ^ (x >> np.uint64(30))) * _M1
        x = (x ^ (x >> np.uint64(27))) * _M2
    return x ^ (x >> np.uint64(31))


class Stream:
    """Counter-based splitmix64 stream; draws are reproducible by (seed, position)."""

    def __init__(self, seed: int):
        self.seed = np.uint64(seed & 0xFFFFFFFFFFFFFFFF)
        self.pos = 0

    def u64(self, n: int) -> np.ndarray:
        i = np.arange(self.pos, self.pos + n, dtype=np.uint64)
        self.pos += n
        with np.errstate(over="ignore"):
            return splitmix64(self.seed + i * GOLDEN)

    def uniform(self, n: int) -> np.ndarray:
        """float64 in [0, 1) from the top 53 bits."""
        return (self.u64(n) >> np.uint64(11)).astype(np.float64) * (1.0 / (1 << 53))

    def uniform_f32_pm1(self, n: int) -> np.ndarray:
        """float32 in [-1, 1): exact multiples of 2^-23."""
        k = (self.u64(n) >> np.uint64(40)).astype(np.int64)  # 24 bits
        return (k.astype(np.float32) * np.float32(2.0 ** -23) - np.float32(1.0)).astype(np.float32)

    def normal(self, n: int) -> np.ndarray:
        """N(0, 1) by Box-Muller on pairs of uniforms (u1 in (0, 1])."""
        m = (n + 1) // 2
        u1 = 1.0 - self.uniform(m)
        u2 = self.uniform(m)
        r = np.sqrt(-2.0 * np.log(u1))
        z = np.concatenate([r * np.cos(2 * np.pi * u2), r * np.sin(2 * np.pi * u2)])
        return z[:n]

    def randint(self, n: int, hi: int) -> np.ndarray:
        """Integers in [0, hi) (multiply-shift on 32 high bits)."""
        u = (self.u64(n) >> np.uint64(32)).astype(np.uint64)
        return ((u * np.uint64(hi)) >> np.uint64(32)).astype(np.int64)

    def bytes(self, n: int) -> np.ndarray:
        return self.u64((n + 7) // 8).view(np.uint8)[:n].copy()


# ------------------------------------------------------------------ C1 / C2
def c1_float_payload(nelems: int, seed: int = 0) -> np.ndarray:
    return Stream(seed).uniform_f32_pm1(nelems)


def c1_sizes() -> list[int]:
    """4 B .. 1 MiB in powers of two (19 sizes)."""
    return [4 << k for k in range(19)]


def c2_sizes(lo: int = 8, hi: int = 256 << 20) -> list[int]:
    out, s = [], lo
    while s <= hi:
        out.append(s)
        s *= 2
    return out


# ---------------------------------------------------------------------- C3
def c3_block(n: int, pe: int, seed: int = 3) -> np.ndarray:
    """PE pe's n^3 float64 block, N(0,1), stream keyed on (seed, pe)."""
    s = Stream(int(splitmix64(np.uint64(seed) ^ np.uint64(pe << 48))))
    return s.normal(n * n * n).astype(np.float64)


# ---------------------------------------------------------------------- C4
def c4_batch(seed: int = 4, n: int = 100_000, npes: int = 64, heap: int = 64 << 20,
             median: float = 2048.0, sigma: float = 1.5, lo: int = 4, hi: int = 4 << 20,
             p_put: float = 0.45, p_get: float = 0.45) -> np.ndarray:
    """Uneven request batch with disjoint destinations.

    Each PE's heap is split in two halves: sources are drawn anywhere in the
    lower half (they may overlap one another -- they are only read),
    destinations are placed without overlap in the upper half, each rounded
    up to 16 bytes, in generation order with random 16-byte-aligned gaps.
    """
    st = Stream(seed)
    half = heap // 2
    u_op = st.uniform(n)
    op = np.where(u_op < p_put, REQ_PUT, np.where(u_op < p_put + p_get, REQ_GET, REQ_SIGNAL)).astype(np.uint8)
    z = st.normal(n)
    size = np.exp(np.log(median) + sigma * z)
    size = np.clip(size, lo, hi)
    dtype = st.randint(n, 3).astype(np.uint8)
    width = np.where(dtype == DT_DOUBLE, 8, 4)
    nbytes = (np.maximum(size // width, 1) * width).astype(np.int64)
    nbytes = np.minimum(nbytes, (hi // 8) * 8)
    nbytes[op == REQ_SIGNAL] = 0
    src_pe = st.randint(n, npes)
    dst_pe = st.randint(n, npes)
    # source offsets: 16-byte aligned, anywhere the whole range fits
    span = np.maximum((half - nbytes) // 16, 1)
    src_off = (st.randint(n, 1 << 30) % span) * 16
    # destination placement per PE
    occ = np.where(op == REQ_SIGNAL, 16, (nbytes + 15) // 16 * 16)
    gap_u = st.uniform(n)
    dst_off = np.zeros(n, dtype=np.int64)
    for pe in range(npes):
        idx = np.nonzero(dst_pe == pe)[0]
        if len(idx) == 0:
            continue
        tot = int(occ[idx].sum())
        free = half - tot
        if free < 0:
            raise ValueError(f"PE {pe}: destinations need {tot} bytes, more than half the heap")
        gaps = np.floor(gap_u[idx] * (free // 16) / len(idx)).astype(np.int64) * 16
        starts = np.cumsum(np.concatenate([[0], (occ[idx] + gaps)[:-1]])) + gaps[0]
        dst_off[idx] = half + starts
    r = np.zeros(n, dtype=REQUEST_DTYPE)
    r["src_off"] = src_off
    r["dst_off"] = dst_off
    r["bytes"] = nbytes
    r["src_pe"] = src_pe
    r["dst_pe"] = dst_pe
    r["op"] = op
    r["dtype"] = dtype
    r["value"] = (st.u64(n) >> np.uint64(33)).astype(np.int64)
    return r


def check_disjoint(reqs: np.ndarray) -> bool:
    """True when no request writes bytes another request reads or writes."""
    is_sig = reqs["op"] == REQ_SIGNAL
    w_pe = reqs["dst_pe"].astype(np.int64)
    w0 = reqs["dst_off"].astype(np.int64)
    w1 = w0 + np.where(is_sig, 4, reqs["bytes"].astype(np.int64))
    copy = (reqs["op"] == REQ_PUT) | (reqs["op"] == REQ_GET)
    r_pe = reqs["src_pe"][copy].astype(np.int64)
    r0 = reqs["src_off"][copy].astype(np.int64)
    r1 = r0 + reqs["bytes"][copy].astype(np.int64)
    for pe in np.unique(w_pe):
        m = w_pe == pe
        order = np.argsort(w0[m], kind="stable")
        a0, a1 = w0[m][order], w1[m][order]
        if np.any(a0[1:] < a1[:-1]):
            return False
        rm = r_pe == pe
        if not rm.any():
            continue
        # a read [s, e) meets a write iff some write starts before e and ends after s
        k = np.searchsorted(a0, r1[rm], side="left")  # writes starting before e: indices < k
        cummax_end = np.maximum.accumulate(a1)
        hit = (k > 0) & (cummax_end[np.maximum(k - 1, 0)] > r0[rm])
        if hit.any():
            return False
    return True

"""The crate's test-matrix generators (src/lib.rs:22-60, 111-154), restated for
the tests: rand 0.9's StdRng (ChaCha12, rand_chacha 0.9) seeded with
SeedableRng::seed_from_u64 (rand_core 0.9: the u64 expanded to the 32-byte key
by PCG32 steps), and the samplers the generators call -- random_range on
usize (rand 0.9 samples it as u32 when the range fits in u32, with Canon's
method: one widening multiply, plus a second one when the low half of the
product falls in the biased zone) and on f64 (UniformFloat::sample_single:
52 random bits as a value in [1, 2), minus 1, times the scale, plus low).

TEST INFRASTRUCTURE ONLY, and parity unpinned: the crate ships no sample of
these streams, and the rand crates are not in this image, so bit identity
with the crate's matrices is unverified.  The ChaCha block function and the
f64 sampler are the ones the checker's start vector uses, which the crate's
own LAS2 example pins (src/legacy.rs:237-283).  The tests that use these
matrices assert the crate's behaviour on them (a solve that succeeds, two
operators that agree), which holds for any matrix of their kind.
"""
from __future__ import annotations

import struct

import numpy as np

import oracle as O

_M64 = (1 << 64) - 1
_M32 = (1 << 32) - 1


def seed_from_u64(state: int) -> bytes:
    """rand_core's SeedableRng::seed_from_u64: 8 PCG32 outputs, little-endian."""
    mul, inc = 6364136223846793005, 11634580027462260723
    out = b""
    for _ in range(8):
        state = (state * mul + inc) & _M64
        xorshifted = (((state >> 18) ^ state) >> 27) & _M32
        rot = state >> 59
        x = ((xorshifted >> rot) | (xorshifted << ((32 - rot) & 31))) & _M32
        out += struct.pack("<I", x)
    return out


class StdRng:
    """ChaCha12 with a 4-block result buffer (rand_core's BlockRng)."""

    def __init__(self, seed: bytes):
        self.key = bytes(seed)
        self.counter = 0
        self.buf = []
        self.index = 64

    @classmethod
    def from_u64(cls, state: int) -> "StdRng":
        return cls(seed_from_u64(state))

    def _refill(self):
        self.buf = []
        for b in range(4):
            self.buf.extend(int(w) for w in O.chacha_block(self.key, self.counter + b, 0, 12))
        self.counter += 4

    def next_u32(self) -> int:
        if self.index >= 64:
            self._refill()
            self.index = 0
        v = self.buf[self.index]
        self.index += 1
        return v

    def next_u64(self) -> int:
        if self.index < 63:
            lo, hi = self.buf[self.index], self.buf[self.index + 1]
            self.index += 2
        elif self.index >= 64:
            self._refill()
            lo, hi = self.buf[0], self.buf[1]
            self.index = 2
        else:
            lo = self.buf[63]
            self._refill()
            hi = self.buf[0]
            self.index = 1
        return lo | (hi << 32)

    def range_usize(self, low: int, high: int) -> int:
        """random_range(low..high) on usize, a range that fits in u32 (Canon's method)."""
        rng = (high - 1 - low + 1) & _M32
        p = self.next_u32() * rng
        result, lo_order = p >> 32, p & _M32
        if lo_order > ((-rng) & _M32):
            new_hi = (self.next_u32() * rng) >> 32
            if lo_order + new_hi > _M32:
                result += 1
        return low + result

    def range_f64(self, low: float, high: float) -> float:
        """random_range(low..high) on f64 (UniformFloat::sample_single)."""
        scale = high - low
        while True:
            bits = (self.next_u64() >> 12) | 0x3FF0000000000000
            v12 = struct.unpack("<d", struct.pack("<Q", bits))[0]
            res = (v12 - 1.0) * scale + low
            if res < high:
                return res
            scale = np.nextafter(scale, -np.inf)


def create_sparse_matrix(rows: int, cols: int, density: float) -> dict:
    """src/lib.rs:22-60: StdRng::seed_from_u64(42), distinct positions drawn
    with random_range (a HashSet drops repeats), values in (-10, 10) away
    from 0; a COO in push order."""
    rng = StdRng.from_u64(42)
    nnz = max(1, int(round(rows * cols * density)))
    seen, r, c, v = set(), [], [], []
    while len(seen) < nnz:
        i = rng.range_usize(0, rows)
        j = rng.range_usize(0, cols)
        if (i, j) not in seen:
            seen.add((i, j))
            while True:
                x = rng.range_f64(-10.0, 10.0)
                if abs(x) > 1e-10:
                    break
            r.append(i)
            c.append(j)
            v.append(x)
    return {"nrows": rows, "ncols": cols, "row": np.array(r, np.int64), "col": np.array(c, np.int64),
            "data": np.array(v)}


def random_coo(nrows: int, ncols: int, seed: int) -> dict:
    """src/lib.rs:113-125: nrows * ncols / 5 pushes of (random_range(0..nrows),
    random_range(0..ncols), random_range(-10.0..10.0)), repeats kept."""
    rng = StdRng.from_u64(seed)
    r, c, v = [], [], []
    for _ in range(nrows * ncols // 5):
        r.append(rng.range_usize(0, nrows))
        c.append(rng.range_usize(0, ncols))
        v.append(rng.range_f64(-10.0, 10.0))
    return {"nrows": nrows, "ncols": ncols, "row": np.array(r, np.int64), "col": np.array(c, np.int64),
            "data": np.array(v)}


def coo_to_csr(A: dict) -> dict:
    """CsrMatrix::from(&coo) (nalgebra-sparse): repeats summed, columns ascending."""
    import scipy.sparse as sp
    S = sp.coo_matrix((A["data"], (A["row"], A["col"])), shape=(A["nrows"], A["ncols"])).tocsr()
    S.sum_duplicates()
    S.sort_indices()
    return {"nrows": A["nrows"], "ncols": A["ncols"], "indptr": S.indptr.astype(np.int64),
            "indices": S.indices.astype(np.int64), "data": S.data.astype(np.float64)}

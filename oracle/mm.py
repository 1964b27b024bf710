"""TEST INFRASTRUCTURE -- a pure-Python restatement of the reference's Matrix
Market input path, the checker for the library's reader (f3r_b200/csrc/io.cpp).

Restates, for small files:
  * io::mm::_read_matrix_market (umineko-sparse/matrix/io.hpp:129-192):
    banner tokens 4 and 5 give the field and the symmetry; lines starting
    with '%' are skipped; the size line is "nrow ncol nlines"; each data line
    "row col value" (1-based); an off-diagonal entry whose value is exactly 0
    is dropped; in a symmetric file an off-diagonal entry is followed by its
    mirror;
  * io::CSR(COO) (io.hpp:44-60): a stable counting sort by row, then each row
    sorted by column (entries with distinct columns: any sort gives the same
    order);
  * io::mm::read_system (io.hpp:104-126) with the drivers' init
    (work/src/f3r-gpu.cpp:60): b from "<stem>_b.mtx" (io.hpp:196-216) when
    that file exists, else v.random<0, 1>(std::mt19937_64(0))
    (core/tensor.hpp:253-265): std::uniform_real_distribution<double>(0, 1)
    over the 64-bit Mersenne Twister.

The generator is MT19937-64 (Matsumoto and Nishimura, "Mersenne Twister: a
623-dimensionally equidistributed uniform pseudorandom number generator",
1998; 64-bit parameters as standardised for std::mt19937_64 in C++11
[rand.predef]) and the libstdc++ generate_canonical<double, 53> for a 64-bit
engine, which is one draw u scaled to u / 2^64 (rounded to double), with 1.0
replaced by the largest double below 1.
"""
from __future__ import annotations

import math
import os

import numpy as np

# ---- MT19937-64 -----------------------------------------------------------
_W, _N, _M, _R = 64, 312, 156, 31
_A = 0xB5026F5AA96619E9
_U, _D = 29, 0x5555555555555555
_S, _B = 17, 0x71D67FFFEDA60000
_T, _C = 37, 0xFFF7EEE000000000
_L = 43
_F = 6364136223846793005
_MASK = (1 << 64) - 1
_LOWER = (1 << _R) - 1
_UPPER = _MASK ^ _LOWER


class MT19937_64:
    def __init__(self, seed: int = 5489):
        self.mt = [0] * _N
        self.mt[0] = seed & _MASK
        for i in range(1, _N):
            prev = self.mt[i - 1]
            self.mt[i] = (_F * (prev ^ (prev >> (_W - 2))) + i) & _MASK
        self.index = _N

    def _twist(self):
        mt = self.mt
        for i in range(_N):
            x = (mt[i] & _UPPER) | (mt[(i + 1) % _N] & _LOWER)
            xa = x >> 1
            if x & 1:
                xa ^= _A
            mt[i] = mt[(i + _M) % _N] ^ xa
        self.index = 0

    def __call__(self) -> int:
        if self.index >= _N:
            self._twist()
        y = self.mt[self.index]
        self.index += 1
        y ^= (y >> _U) & _D
        y ^= (y << _S) & _B
        y ^= (y << _T) & _C
        y ^= y >> _L
        return y & _MASK


def uniform01(seed: int, n: int) -> np.ndarray:
    """n draws of uniform_real_distribution<double>(0, 1) over mt19937_64(seed)."""
    g = MT19937_64(seed)
    out = np.empty(n)
    below_one = math.nextafter(1.0, 0.0)
    for i in range(n):
        r = float(g()) / 18446744073709551616.0
        out[i] = below_one if r >= 1.0 else r
    return out


# ---- Matrix Market -------------------------------------------------------

def _tokens_after_comments(text: str):
    lines = text.split("\n")
    banner = lines[0].split()
    body = []
    for ln in lines[1:]:
        if ln.startswith("%"):
            continue
        body.extend(ln.split())
    return banner, body


def read_matrix(path: str):
    """(nrow, ncol, rptr, idx, val) as io::CSR(io::mm::read_matrix(path))."""
    with open(path) as f:
        banner, tok = _tokens_after_comments(f.read())
    if len(banner) != 5:
        raise ValueError("bad banner")
    symmetric = banner[4] == "symmetric"
    nrow, ncol, nlines = int(float(tok[0])), int(float(tok[1])), int(float(tok[2]))
    rows, cols, vals = [], [], []
    for k in range(nlines):
        i = int(float(tok[3 + 3 * k])) - 1
        j = int(float(tok[4 + 3 * k])) - 1
        v = float(tok[5 + 3 * k])
        if v == 0.0 and i != j:
            continue
        rows.append(i), cols.append(j), vals.append(v)
        if symmetric and i != j:
            rows.append(j), cols.append(i), vals.append(v)
    rows = np.asarray(rows, np.int64)
    order = np.argsort(rows, kind="stable")
    cols_o = np.asarray(cols, np.int32)[order]
    vals_o = np.asarray(vals, np.float64)[order]
    rptr = np.zeros(nrow + 1, np.int32)
    np.add.at(rptr, rows + 1, 1)
    rptr = np.cumsum(rptr).astype(np.int32)
    for r in range(nrow):
        b, e = rptr[r], rptr[r + 1]
        o = np.argsort(cols_o[b:e], kind="stable")
        cols_o[b:e] = cols_o[b:e][o]
        vals_o[b:e] = vals_o[b:e][o]
    return nrow, ncol, rptr, cols_o, vals_o


def read_rhs(matrix_path: str, n: int) -> np.ndarray:
    """b of io::mm::read_system with the drivers' init."""
    pb = matrix_path[:-4] + "_b" + matrix_path[-4:]
    if not os.path.exists(pb):
        return uniform01(0, n)
    with open(pb) as f:
        banner, tok = _tokens_after_comments(f.read())
    nrow, ncol = int(float(tok[0])), int(float(tok[1]))
    if banner[2] != "array" or banner[4] != "general" or ncol != 1 or nrow != n:
        raise ValueError("bad right-hand side file")
    return np.asarray([float(t) for t in tok[2:2 + n]], np.float64)

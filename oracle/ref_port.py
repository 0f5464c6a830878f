"""numba restatement of the reference CPU state-vector kernels -- the timed CPU
baseline ("port") for bench.py (test infrastructure; see oracle/__init__.py).

The reference CPU path (statevector_simulator.py:168-193) dispatches each gate
to one of four numba kernels in QuICT/ops/linalg/cpu_calculator.py:
  matrix_dot_vector (:139-186)  gather the 2^k amplitudes of each group, dense matvec
  diagonal_matrix   (:189-235)  multiply the touched amplitudes by the diagonal
  swap_matrix       (:238-280)  exchange two amplitudes per group
  reverse_matrix    (:283-326)  anti-diagonal exchange with scaling
Each walks groups i in [0, 2^(n-k)) and rebuilds the group's base index by
inserting a zero at every sorted gate-bit position.  The reference jits them
with @njit() (single-threaded: its prange degrades to range); this port runs
the same per-group algorithm with numba's parallel=True so the baseline uses
every host core it is given.
"""
from __future__ import annotations

import numpy as np
from numba import njit, prange


@njit(cache=True, inline="always")
def _base(i, sorted_bits):
    for b in sorted_bits:
        i = ((i >> b) << (b + 1)) | (i & ((1 << b) - 1))
    return i


@njit(parallel=True, cache=True)
def dense(vec, mat, offs, sorted_bits, cmask):
    """matrix_dot_vector: vec[group] <- mat @ vec[group]."""
    d = offs.size
    groups = vec.size >> sorted_bits.size
    for g in prange(groups):
        base = _base(np.int64(g), sorted_bits) | cmask
        x = np.empty(d, dtype=vec.dtype)
        for r in range(d):
            x[r] = vec[base + offs[r]]
        for r in range(d):
            acc = vec.dtype.type(0)
            for c in range(d):
                acc += mat[r, c] * x[c]
            vec[base + offs[r]] = acc


@njit(parallel=True, cache=True)
def diagonal(vec, diag, offs, sorted_bits, cmask):
    """diagonal_matrix: vec[base + offs[r]] *= diag[r]."""
    d = offs.size
    groups = vec.size >> sorted_bits.size
    for g in prange(groups):
        base = _base(np.int64(g), sorted_bits) | cmask
        for r in range(d):
            vec[base + offs[r]] *= diag[r]


@njit(parallel=True, cache=True)
def swap(vec, a_off, b_off, sa, sb, sorted_bits, cmask):
    """swap_matrix / reverse_matrix: (v_a, v_b) <- (sa * v_b, sb * v_a)."""
    groups = vec.size >> sorted_bits.size
    for g in prange(groups):
        base = _base(np.int64(g), sorted_bits) | cmask
        t = vec[base + a_off]
        vec[base + a_off] = sa * vec[base + b_off]
        vec[base + b_off] = sb * t


def prepare(ops, dtype):
    """Lowered ops -> list of (kernel, args) with per-gate index tables built once."""
    out = []
    for op in ops:
        tb = list(op.tbits)
        cm = 0
        for b in op.cbits:
            cm |= 1 << b
        sorted_bits = np.array(sorted(tb + list(op.cbits)), dtype=np.int64)
        m = len(tb)
        offs = np.zeros(1 << m, dtype=np.int64)
        for r in range(1 << m):
            for j in range(m):
                if (r >> (m - 1 - j)) & 1:
                    offs[r] |= 1 << tb[j]
        if op.kind == "diag":
            out.append((diagonal, (np.asarray(op.mat, dtype=dtype), offs, sorted_bits, np.int64(cm))))
        elif op.kind == "antidiag":
            out.append((swap, (np.int64(0), np.int64(1 << tb[0]), dtype(op.mat[0, 1]), dtype(op.mat[1, 0]),
                               sorted_bits, np.int64(cm))))
        elif op.kind == "swap" and op.mat[0, 0] == 1 and op.mat[3, 3] == 1:
            out.append((swap, (np.int64(1 << tb[1]), np.int64(1 << tb[0]), dtype(op.mat[1, 2]),
                               dtype(op.mat[2, 1]), sorted_bits, np.int64(cm))))
        else:
            out.append((dense, (np.ascontiguousarray(op.dense(), dtype=dtype), offs, sorted_bits, np.int64(cm))))
    return out


def run(vec, prepared):
    for fn, args in prepared:
        fn(vec, *args)
    return vec

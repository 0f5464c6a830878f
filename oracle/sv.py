"""FP64 state-vector oracle (test infrastructure; see oracle/__init__.py).

Restates, in numpy, what QuICT's simulators compute:
  * gate application in QuICT's big-endian convention -- qubit 0 is the most
    significant bit of the amplitude index (QuICT/core/qubit/qubit.py:192-213)
    and a k-qubit matrix acts big-endian on cargs + targs, as
    matrix_product_to_circuit embeds it (QuICT/core/utils/utils.py:8-56) and
    UnitarySimulator applies it (QuICT/simulation/unitary/unitary_simulator.py);
  * the reference SV path's reversed argument order for uncontrolled
    multi-target dense matrices (cpu_calculator.py:139-186), on request;
  * measurement / reset (cpu_calculator.py:329-384);
  * the sampling loop of StateVectorSimulator.sample
    (statevector_simulator.py:595-626), and its one-uniform inverse-CDF form.
"""
from __future__ import annotations

from typing import Iterable, List, Sequence, Tuple

import numpy as np


def zero_state(n: int) -> np.ndarray:
    v = np.zeros(1 << n, dtype=np.complex128)
    v[0] = 1.0
    return v


def apply_matrix(vec: np.ndarray, n: int, mat: np.ndarray, args: Sequence[int]) -> np.ndarray:
    """vec <- (mat on circuit qubits `args`, big-endian) vec.  Returns a new array."""
    k = len(args)
    if k == 1:  # the common case, as two strided row updates (qubit q = axis q)
        q = args[0]
        m = np.asarray(mat, dtype=np.complex128)
        v3 = np.asarray(vec, dtype=np.complex128).reshape(1 << q, 2, -1)
        out = np.empty_like(v3)
        out[:, 0, :] = m[0, 0] * v3[:, 0, :] + m[0, 1] * v3[:, 1, :]
        out[:, 1, :] = m[1, 0] * v3[:, 0, :] + m[1, 1] * v3[:, 1, :]
        return out.reshape(-1)
    t = np.asarray(mat, dtype=np.complex128).reshape([2] * (2 * k))
    psi = vec.reshape([2] * n)
    out = np.tensordot(t, psi, axes=(list(range(k, 2 * k)), list(args)))
    out = np.moveaxis(out, list(range(k)), list(args))
    return np.ascontiguousarray(out).reshape(-1)


def run(gates: Iterable[Tuple[np.ndarray, Sequence[int]]], n: int, vec: np.ndarray = None,
        legacy_2q_order: bool = False, n_controls: Sequence[int] = None) -> np.ndarray:
    """Apply [(matrix, args)] in order.  With legacy_2q_order, gates listed with
    0 controls and >= 2 args are applied with their args reversed, as the
    reference SV kernels do for dense uncontrolled matrices."""
    v = zero_state(n) if vec is None else np.asarray(vec, dtype=np.complex128).copy()
    for i, (m, args) in enumerate(gates):
        args = list(args)
        if legacy_2q_order and len(args) >= 2 and (n_controls is None or n_controls[i] == 0):
            args = args[::-1]
        v = apply_matrix(v, n, m, args)
    return v


def prob0(vec: np.ndarray, n: int, qubit: int) -> float:
    """P(qubit = 0); qubit 0 is the MSB."""
    p = np.abs(vec.reshape([2] * n)) ** 2
    return float(np.take(p, 0, axis=qubit).sum())


def measure(vec: np.ndarray, n: int, qubit: int, u: float) -> Tuple[np.ndarray, int]:
    """Reference rule (cpu_calculator.py:329-363): outcome 1 iff u > P(0); the
    kept half is scaled by 1/sqrt(p) and the other half zeroed."""
    p0 = prob0(vec, n, qubit)
    one = u > p0
    t = vec.reshape([2] * n).copy()
    keep = 1 if one else 0
    alpha = 1.0 / np.sqrt((1.0 - p0) if one else p0)
    idx = [slice(None)] * n
    idx[qubit] = 1 - keep
    t[tuple(idx)] = 0
    idx[qubit] = keep
    t[tuple(idx)] *= alpha
    return t.reshape(-1), int(one)


def reset(vec: np.ndarray, n: int, qubit: int) -> np.ndarray:
    """Reference reset (cpu_calculator.py:366-384): alpha = sqrt(P(0));
    alpha < 1e-6 moves the |1> half into |0>, else |0> half /= alpha; |1> <- 0."""
    p0 = prob0(vec, n, qubit)
    alpha = np.sqrt(p0)
    t = vec.reshape([2] * n).copy()
    i0 = [slice(None)] * n
    i1 = [slice(None)] * n
    i0[qubit], i1[qubit] = 0, 1
    if alpha < 1e-6:
        t[tuple(i0)] = t[tuple(i1)]
    else:
        t[tuple(i0)] = t[tuple(i0)] / alpha
    t[tuple(i1)] = 0
    return t.reshape(-1)


def sample_sequential(vec: np.ndarray, n: int, uniforms: np.ndarray) -> np.ndarray:
    """Reference sampling loop: per shot, measure qubits 0..n-1 in order with
    one uniform each, then restore the state (statevector_simulator.py:595-626).
    Returns the basis index (big-endian outcome integer) of every shot.
    O(shots * n * 2^n): small cases only."""
    u = np.asarray(uniforms, dtype=np.float64).reshape(-1, n)
    out = np.empty(u.shape[0], dtype=np.int64)
    for s in range(u.shape[0]):
        v = vec.copy()
        idx = 0
        for q in range(n):
            v, b = measure(v, n, q, u[s, q])
            idx = (idx << 1) | b
        out[s] = idx
    return out


def sample_sequential_fast(vec: np.ndarray, n: int, uniforms: np.ndarray) -> np.ndarray:
    """Same rule as sample_sequential via conditional probabilities
    P(prefix0) / P(prefix) from prefix sums (equal up to rounding)."""
    p = np.abs(np.asarray(vec)) ** 2
    u = np.asarray(uniforms, dtype=np.float64).reshape(-1, n)
    out = np.empty(u.shape[0], dtype=np.int64)
    cs = np.concatenate([[0.0], np.cumsum(p)])
    N = p.size
    for s in range(u.shape[0]):
        lo, size = 0, N
        for q in range(n):
            half = size // 2
            sl = cs[lo + half] - cs[lo]
            sn = cs[lo + size] - cs[lo]
            if u[s, q] > sl / sn:
                lo += half
            size = half
        out[s] = lo
    return out


def sample_cdf(vec: np.ndarray, uniforms: np.ndarray) -> np.ndarray:
    """One uniform per shot: smallest i with u * total <= CDF[i] (FP64
    cumulative sum, total = CDF[-1]), never an index of probability 0.
    By the chain rule this is the reference's sequential rule fed the derived
    uniform stream u_{k+1} = u_k / p0 or (u_k - p0) / (1 - p0); scaling u by
    the total makes it a distribution over the state's own mass when its norm
    has drifted from 1 (complex64 rounding, a density matrix's trace)."""
    p = np.abs(np.asarray(vec)) ** 2
    return _cdf_pick(p, uniforms)


def _cdf_pick(p: np.ndarray, uniforms: np.ndarray) -> np.ndarray:
    cdf = np.cumsum(p)
    nz = np.flatnonzero(p > 0)
    if nz.size == 0:
        return np.zeros(np.asarray(uniforms).shape, dtype=np.int64)
    t = np.asarray(uniforms, dtype=np.float64) * cdf[-1]
    idx = np.searchsorted(cdf, t, side="left")
    # a flat CDF run (p = 0) is never the first index reaching t, except
    # before the first nonzero probability (t = 0) and past the end (rounding)
    return np.clip(idx, nz[0], nz[-1]).astype(np.int64)


def near_ties(vec: np.ndarray, uniforms: np.ndarray, tol: float = 1e-12) -> np.ndarray:
    """Mask of uniforms within `tol` of a CDF boundary (where FP64 summation
    order may legitimately change the sampled index)."""
    cdf = np.cumsum(np.abs(np.asarray(vec)) ** 2)
    u = np.asarray(uniforms, dtype=np.float64) * cdf[-1]
    j = np.searchsorted(cdf, u)
    d = np.full(u.shape, np.inf)
    for off in (-1, 0):
        jj = np.clip(j + off, 0, cdf.size - 1)
        d = np.minimum(d, np.abs(cdf[jj] - u))
    return d < tol


def permute_qubits(vec: np.ndarray, n: int, dest_from_src: Sequence[int]) -> np.ndarray:
    """Qubit permutation: new qubit i holds old qubit mapping[i]."""
    t = vec.reshape([2] * n)
    return np.ascontiguousarray(np.transpose(t, list(dest_from_src))).reshape(-1)


def vector_permutation(vec: np.ndarray, n: int, mapping) -> np.ndarray:
    """Index-level restatement of the reference's vector_*_permutation kernel
    (QuICT/ops/linalg/gpu_calculator.py:170-207): y[t] = x[xid] with bit
    (n-1-i) of xid taken from bit (n-1-mapping[i]) of t."""
    x = np.asarray(vec)
    y = np.empty_like(x)
    for t in range(1 << n):
        xid = 0
        for i in range(n):
            xid |= ((t >> (n - 1 - mapping[i])) & 1) << (n - 1 - i)
        y[t] = x[xid]
    return y

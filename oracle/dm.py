"""FP64 density-matrix oracle and QuICT noise channels (test infrastructure;
see oracle/__init__.py).

  * rho <- U rho U^dagger and rho <- sum_i K_i rho K_i^dagger in QuICT's
    big-endian convention, the result DensityMatrixSimulator computes with
    dense embeddings (QuICT/simulation/density_matrix/density_matrix_simulator.py:147-180).
  * A noisy gate contributes Kraus operators K_i . U
    (QuantumNoiseError.apply_to_gate, QuICT/core/noise/noise_error.py:132-138),
    replacing U (NoiseModel.transpile, QuICT/core/noise/noise_model.py:152-185).
  * Kraus sets: DepolarizingError (noise_error.py:239-263) as Pauli strings
    over 'ixyz' with probabilities [1 - p (4^k-1)/4^k, p/4^k, ...];
    DampingError (noise_error.py:266-338) with phase = 0, dissipation = 0:
    K0 = [[1, 0], [0, sqrt(1-g)]], K1 = [[0, sqrt g], [0, 0]];
    compose (noise_error.py:100-117): ops A_j . P_i with probability product,
    outer loop over the left error; tensor (noise_error.py:119-130): kron.
"""
from __future__ import annotations

from itertools import product
from typing import Callable, List, Optional, Sequence, Tuple

import numpy as np

PAULI = {
    "i": np.eye(2, dtype=np.complex128),
    "x": np.array([[0, 1], [1, 0]], dtype=np.complex128),
    "y": np.array([[0, -1j], [1j, 0]], dtype=np.complex128),
    "z": np.array([[1, 0], [0, -1]], dtype=np.complex128),
}


def depolarizing_ops(p: float, k: int) -> List[Tuple[np.ndarray, float]]:
    num = 4 ** k
    maxp = num / (num - 1)
    probs = [1 - p / maxp] + [p / num] * (num - 1)
    ops = []
    for s, pr in zip(product("ixyz", repeat=k), probs):
        m = PAULI[s[0]]
        for c in s[1:]:
            m = np.kron(m, PAULI[c])
        ops.append((m, pr))
    return ops


def damping_ops(gamma: float) -> List[Tuple[np.ndarray, float]]:
    k0 = np.array([[1, 0], [0, np.sqrt(1 - gamma)]], dtype=np.complex128)
    k1 = np.array([[0, np.sqrt(gamma)], [0, 0]], dtype=np.complex128)
    return [(k0, 1.0), (k1, 1.0)] if gamma != 0 else [(k0, 1.0)]


def compose(left, right):
    return [(a @ b, pa * pb) for a, pa in left for b, pb in right]


def tensor(left, right):
    return [(np.kron(a, b), pa * pb) for a, pa in left for b, pb in right]


def kraus(ops) -> List[np.ndarray]:
    return [np.sqrt(p) * m for m, p in ops]


def composed_noise_1q(gamma: float, p: float) -> List[np.ndarray]:
    """DampingError(gamma).compose(DepolarizingError(p, 1)) Kraus operators."""
    return kraus(compose(damping_ops(gamma), depolarizing_ops(p, 1)))


def composed_noise_2q(gamma: float, p: float) -> List[np.ndarray]:
    """DampingError(gamma).tensor(same).compose(DepolarizingError(p, 2))."""
    d = damping_ops(gamma)
    return kraus(compose(tensor(d, d), depolarizing_ops(p, 2)))


def zero_dm(n: int) -> np.ndarray:
    r = np.zeros((1 << n, 1 << n), dtype=np.complex128)
    r[0, 0] = 1
    return r


def apply_channel(rho: np.ndarray, n: int, ks: Sequence[np.ndarray], args: Sequence[int]) -> np.ndarray:
    """rho <- sum_i K_i rho K_i^dagger with K_i on qubits `args` (big-endian)."""
    k = len(args)
    t = rho.reshape([2] * (2 * n))
    out = np.zeros_like(t)
    rows = list(args)
    cols = [n + a for a in args]
    for K in ks:
        kt = np.asarray(K, dtype=np.complex128).reshape([2] * (2 * k))
        x = np.tensordot(kt, t, axes=(list(range(k, 2 * k)), rows))
        x = np.moveaxis(x, list(range(k)), rows)
        kc = np.conj(kt)
        x = np.tensordot(kc, x, axes=(list(range(k, 2 * k)), cols))
        x = np.moveaxis(x, list(range(k)), cols)
        out += x
    return out.reshape(1 << n, 1 << n)


def apply_superop(rho: np.ndarray, n: int, ks: Sequence[np.ndarray], args: Sequence[int]) -> np.ndarray:
    """The same map as ``apply_channel`` in one contraction: the channel's
    superoperator S = sum_i K_i (x) conj(K_i) (rows (r_out, c_out), columns
    (r_in, c_in), each big-endian over `args`) times rho's (row bits of args,
    column bits of args) axes, as one matrix product.  Equal to the Kraus sum
    up to FP64 rounding; fast enough for 12-qubit, 150-gate runs."""
    k = len(args)
    S = sum(np.kron(np.asarray(K, dtype=np.complex128), np.conj(np.asarray(K, dtype=np.complex128))) for K in ks)
    axes = list(args) + [n + a for a in args]
    t = np.moveaxis(rho.reshape([2] * (2 * n)), axes, list(range(2 * k)))
    front = t.shape
    y = (S @ t.reshape(1 << (2 * k), -1)).reshape(front)
    return np.ascontiguousarray(np.moveaxis(y, list(range(2 * k)), axes)).reshape(1 << n, 1 << n)


def run(gates, n: int, rho: Optional[np.ndarray] = None,
        noise: Optional[Callable[[Sequence[int]], Optional[List[np.ndarray]]]] = None,
        superop: bool = False) -> np.ndarray:
    """Apply [(U, args)]; when noise(args) returns Kraus ops K_i, the gate is
    replaced by the channel {K_i U} (accumulated mode).  `superop` applies each
    channel as one superoperator product (``apply_superop``) instead of a
    Kraus sum."""
    apply = apply_superop if superop else apply_channel
    r = zero_dm(n) if rho is None else np.asarray(rho, dtype=np.complex128).copy()
    for U, args in gates:
        ks = noise(args) if noise is not None else None
        if ks:
            r = apply(r, n, [K @ U for K in ks], args)
        else:
            r = apply(r, n, [U], args)
    return r


def prob0(rho: np.ndarray, n: int, qubit: int) -> float:
    d = np.real(np.diag(rho)).reshape([2] * n)
    return float(np.take(d, 0, axis=qubit).sum())


def measure(rho: np.ndarray, n: int, qubit: int, u: float):
    """Reference DM measurement (density_matrix_simulator.py:182-208): outcome 1
    iff u > P(0); rho <- P rho P / p."""
    p0 = prob0(rho, n, qubit)
    one = u > p0
    P = np.diag([0.0, 1.0] if one else [1.0, 0.0]).astype(np.complex128) / np.sqrt((1 - p0) if one else p0)
    return apply_channel(rho, n, [P], [qubit]), int(one)

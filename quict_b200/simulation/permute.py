"""Perm gate: a qubit permutation applied as a network of Swap ops.

Semantics follow the reference's VectorPermutation
(QuICT/ops/linalg/gpu_calculator.py:170-250) driven by
StateVectorSimulator.apply_gate (statevector_simulator.py:297-312):
mapping = identity; mapping[args[i]] = args[pargs[i]]; the amplitude of a
destination index takes, for every qubit i, the value of destination qubit
mapping[i] as source qubit i -- i.e. source qubit i moves to qubit mapping[i].
The reference gathers into a fresh vector; here the permutation is decomposed
into at most n-1 transpositions that run in place through the fused passes.
"""
from __future__ import annotations

from typing import List, Sequence, Tuple

import numpy as np

from .lowering import Op

_SWAP = np.array([[1, 0, 0, 0], [0, 0, 1, 0], [0, 1, 0, 0], [0, 0, 0, 1]], dtype=np.complex128)


def perm_mapping(n: int, args: Sequence[int], pargs: Sequence[int]) -> List[int]:
    """Destination qubit of every source qubit (reference semantics)."""
    if len(args) == n:
        return [int(p) for p in pargs]
    mapping = list(range(n))
    for idx, parg in enumerate(pargs):
        mapping[args[idx]] = args[parg]
    return mapping


def swap_network(mapping: Sequence[int]) -> List[Tuple[int, int]]:
    """Qubit swaps (a, b) that move source qubit i to qubit mapping[i]."""
    n = len(mapping)
    if sorted(mapping) != list(range(n)):
        raise ValueError("Perm parameters do not form a permutation")
    where = list(range(n))          # where[s] = current position of source qubit s
    at = list(range(n))             # at[p] = source qubit currently at position p
    swaps = []
    for s in range(n):
        t = mapping[s]
        p = where[s]
        if p == t:
            continue
        other = at[t]
        swaps.append((p, t))
        at[p], at[t] = other, s
        where[other], where[s] = p, t
    return swaps


def perm_ops(n: int, op: Op) -> List[Op]:
    args = [n - 1 - b for b in op.tbits]
    mapping = perm_mapping(n, args, op.perm)
    return [Op("swap", (n - 1 - a, n - 1 - b), (), _SWAP.copy()) for a, b in swap_network(mapping)]


def apply_perm(engine, vec, n: int, op: Op):
    engine.apply_ops(vec, n, perm_ops(n, op))
    return vec

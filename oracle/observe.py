"""FP64 expectation values and parameter-shift gradients (test infrastructure;
see oracle/__init__.py).

Energies are <psi|H|psi> with psi from oracle.sv (big-endian QuICT
convention) and H a dense Pauli sum.  Gradients use the two-term shift rule
g = [E(theta + pi/2) - E(theta - pi/2)] / 2 per occurrence of a parameter in
exp(-i theta G / 2) gates (G^2 = I), times the occurrence's scale.  The
reference has no gradient code (its ML package is not vendored), so these are
restatements of the published rule, cross-checked in tests against central
finite differences of the reference's own state vectors.
"""
from __future__ import annotations

import numpy as np

from . import sv as osv


def energy(gates, n, hmat):
    psi = osv.run(gates, n)
    return float(np.real(np.vdot(psi, hmat @ psi)))


def param_shift(matrices_fn, params, n, hmat, occurrences):
    """occurrences: list of (param index, entry index, scale); matrices_fn(params,
    shifts={entry: delta}) -> [(matrix, qubits)]."""
    g = np.zeros(len(params))
    for k, entry, scale in occurrences:
        ep = energy(matrices_fn(params, {entry: np.pi / 2}), n, hmat)
        em = energy(matrices_fn(params, {entry: -np.pi / 2}), n, hmat)
        g[k] += scale * 0.5 * (ep - em)
    return g


def finite_diff(matrices_fn, params, n, hmat, h=1e-5):
    g = np.zeros(len(params))
    for k in range(len(params)):
        p1, p2 = params.copy(), params.copy()
        p1[k] += h
        p2[k] -= h
        g[k] = (energy(matrices_fn(p1, {}), n, hmat) - energy(matrices_fn(p2, {}), n, hmat)) / (2 * h)
    return g

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
    """<psi|H|psi>; `hmat` a dense matrix, or a Pauli sum as a list of
    (coefficient, {qubit: 'X'|'Y'|'Z'}) terms (see ``pauli_expect``)."""
    psi = osv.run(gates, n)
    if isinstance(hmat, list):
        return pauli_expect(psi, n, hmat)
    return float(np.real(np.vdot(psi, hmat @ psi)))


def pauli_expect(psi, n, terms):
    """sum_t c_t <psi|P_t|psi> without a dense H: a Pauli string with X-part
    mask x and Z-part mask z (vector bits; qubit q is bit n-1-q, Y = i X Z)
    maps amplitude j to (i^|x & z|) (-1)^|z & j| at index j ^ x."""
    idx = np.arange(1 << n, dtype=np.int64)
    total = 0.0
    for c, ps in terms:
        x = z = 0
        for q, p in ps.items():
            b = 1 << (n - 1 - q)
            if p in ("X", "Y"):
                x |= b
            if p in ("Z", "Y"):
                z |= b
        src = idx ^ x
        par = np.bitwise_count(src & z) & 1
        phase = (1j) ** bin(x & z).count("1")
        p_psi = phase * (1.0 - 2.0 * par) * psi[src]
        total += float(np.real(complex(c) * np.vdot(psi, p_psi)))
    return total


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


def shift_energies(base, n, hmat, shifted):
    """Energies of the circuit `base` ([(matrix, qubits)]) with one gate
    replaced at a time: `shifted` = [(entry, m_plus, m_minus)] in ascending
    entry order gives [(E with gate entry = m_plus, E with m_minus)].  The state
    before each entry is carried forward once, so the cost per entry is two
    runs of the gates after it."""
    out = []
    psi = osv.zero_state(n)
    at = 0
    for entry, mp, mm in shifted:
        for m, q in base[at:entry]:
            psi = osv.apply_matrix(psi, n, m, q)
        at = entry
        pair = []
        for m in (mp, mm):
            v = osv.apply_matrix(psi, n, m, base[entry][1])
            for m2, q2 in base[entry + 1:]:
                v = osv.apply_matrix(v, n, m2, q2)
            pair.append(pauli_expect(v, n, hmat) if isinstance(hmat, list)
                        else float(np.real(np.vdot(v, hmat @ v))))
        out.append(tuple(pair))
    return out

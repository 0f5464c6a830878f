"""Parameterised circuits and Pauli-sum observables for batched gradients.

A ``ParamCircuit`` is an ordered list of gate entries on n qubits.  An entry
is either fixed (a matrix, as any QuICT gate) or parameterised:
U(theta) = exp(-i * theta * G / 2) with theta = scale * params[index] and a
generator G from the table below, in QuICT's matrix conventions
(QuICT/core/gate/gate.py: Rx :992-996, Ry :1037-1041, Rz :1083-1087,
Rzz :1805-1814, Rxx :1659-1668, Ryy :1732-1741).  Several entries may share a
parameter (QAOA); the gradient sums their contributions.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

_X = np.array([[0, 1], [1, 0]], dtype=np.complex128)
_Y = np.array([[0, -1j], [1j, 0]], dtype=np.complex128)
_Z = np.array([[1, 0], [0, -1]], dtype=np.complex128)

# generator G (acting on the gate's qubits, big-endian) with U = exp(-i theta G / 2)
GENERATORS: Dict[str, np.ndarray] = {
    "rx": _X,
    "ry": _Y,
    "rz": _Z,
    "rzz": np.kron(_Z, _Z),
    "rxx": np.kron(_X, _X),
    "ryy": np.kron(_Y, _Y),
}


def rotation(kind: str, theta: float) -> np.ndarray:
    """exp(-i theta G / 2) for a Pauli-string generator (G^2 = I)."""
    g = GENERATORS[kind]
    return np.cos(theta / 2) * np.eye(g.shape[0]) - 1j * np.sin(theta / 2) * g


@dataclass
class GateEntry:
    qubits: Tuple[int, ...]
    kind: str                        # "fixed" or a GENERATORS key
    matrix: Optional[np.ndarray] = None  # fixed gates
    index: int = -1                  # parameter index
    scale: float = 1.0               # theta = scale * params[index]


@dataclass
class ParamCircuit:
    n: int
    entries: List[GateEntry] = field(default_factory=list)
    num_params: int = 0

    def fixed(self, matrix, qubits: Sequence[int]):
        self.entries.append(GateEntry(tuple(qubits), "fixed", np.asarray(matrix, dtype=np.complex128)))
        return self

    def rot(self, kind: str, qubits: Sequence[int], index: int, scale: float = 1.0):
        if kind not in GENERATORS:
            raise ValueError(f"unsupported parameterised gate {kind}")
        self.entries.append(GateEntry(tuple(qubits), kind, None, index, scale))
        self.num_params = max(self.num_params, index + 1)
        return self

    def matrices(self, params: np.ndarray) -> List[Tuple[np.ndarray, List[int]]]:
        """[(matrix, qubits)] for one parameter vector (for oracles / export)."""
        out = []
        for e in self.entries:
            m = e.matrix if e.kind == "fixed" else rotation(e.kind, e.scale * float(params[e.index]))
            out.append((m, list(e.qubits)))
        return out


@dataclass
class PauliSum:
    """H = sum_t c_t P_t with P_t a Pauli string given as {qubit: 'X'|'Y'|'Z'}."""
    n: int
    terms: List[Tuple[complex, Dict[int, str]]] = field(default_factory=list)

    def add(self, coeff: complex, paulis: Dict[int, str]):
        self.terms.append((complex(coeff), dict(paulis)))
        return self

    def masks(self) -> Tuple[np.ndarray, np.ndarray, np.ndarray]:
        """(x, z, coeff) over vector bits (qubit q -> bit n-1-q)."""
        xs, zs, cs = [], [], []
        for c, ps in self.terms:
            x = z = 0
            for q, p in ps.items():
                b = 1 << (self.n - 1 - q)
                if p in ("X", "Y"):
                    x |= b
                if p in ("Z", "Y"):
                    z |= b
            xs.append(x)
            zs.append(z)
            cs += [c.real, c.imag]
        return np.array(xs, dtype=np.uint64), np.array(zs, dtype=np.uint64), np.array(cs, dtype=np.float64)

    def matrix(self) -> np.ndarray:
        """Dense 2^n x 2^n matrix (small n; oracle use)."""
        mats = {"X": _X, "Y": _Y, "Z": _Z}
        out = np.zeros((1 << self.n, 1 << self.n), dtype=np.complex128)
        for c, ps in self.terms:
            m = np.eye(1, dtype=np.complex128)
            for q in range(self.n):
                m = np.kron(m, mats[ps[q]] if q in ps else np.eye(2))
            out += c * m
        return out


# ---- the benchmark families -------------------------------------------------------------
def hardware_efficient_ansatz(n: int = 16, layers: int = 8, ring: bool = True) -> ParamCircuit:
    """layers x (Ry, Rz on every qubit, then a CZ ring); 2 * n * layers parameters."""
    cz = np.diag([1, 1, 1, -1]).astype(np.complex128)
    c = ParamCircuit(n)
    p = 0
    for _ in range(layers):
        for q in range(n):
            c.rot("ry", (q,), p)
            p += 1
        for q in range(n):
            c.rot("rz", (q,), p)
            p += 1
        pairs = [(q, q + 1) for q in range(n - 1)] + ([(n - 1, 0)] if ring and n > 2 else [])
        for a, b in pairs:
            c.fixed(cz, (a, b))
    return c


def ising_observable(n: int, j: float = 1.0, h: float = 0.5, periodic: bool = False) -> PauliSum:
    """sum_i j Z_i Z_{i+1} + h sum_i X_i (open chain by default)."""
    hs = PauliSum(n)
    for q in range(n - 1 + (1 if periodic else 0)):
        hs.add(j, {q: "Z", (q + 1) % n: "Z"})
    for q in range(n):
        hs.add(h, {q: "X"})
    return hs


def qaoa_circuit(n: int, edges: Sequence[Tuple[int, int]], p: int) -> ParamCircuit:
    """H on every qubit, then p layers of Rzz(-gamma_l) per edge and Rx(2 beta_l) per
    qubit; parameters [gamma_0..gamma_{p-1}, beta_0..beta_{p-1}]."""
    hmat = np.array([[1, 1], [1, -1]], dtype=np.complex128) / np.sqrt(2)
    c = ParamCircuit(n)
    for q in range(n):
        c.fixed(hmat, (q,))
    for layer in range(p):
        for a, b in edges:
            c.rot("rzz", (a, b), layer, -1.0)
        for q in range(n):
            c.rot("rx", (q,), p + layer, 2.0)
    c.num_params = 2 * p
    return c


def maxcut_observable(n: int, edges: Sequence[Tuple[int, int]]) -> PauliSum:
    """C = sum_edges (1 - Z_a Z_b) / 2."""
    hs = PauliSum(n)
    hs.add(len(edges) / 2.0, {})
    for a, b in edges:
        hs.add(-0.5, {a: "Z", b: "Z"})
    return hs


def random_regular_graph(n: int, d: int, rng: np.random.Generator) -> List[Tuple[int, int]]:
    """Uniform-ish random d-regular simple graph by the pairing model with restarts."""
    for _ in range(1000):
        stubs = np.repeat(np.arange(n), d)
        rng.shuffle(stubs)
        pairs = stubs.reshape(-1, 2)
        ok = all(a != b for a, b in pairs)
        es = {tuple(sorted((int(a), int(b)))) for a, b in pairs}
        if ok and len(es) == len(pairs):
            return sorted(es)
    raise RuntimeError("could not draw a simple regular graph")

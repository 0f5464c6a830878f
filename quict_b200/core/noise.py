"""Noise model compatible with QuICT.core.noise (QuICT/core/noise/).

What the density-matrix simulator consumes:
  * ``NoiseModel.transpile(circuit, accumulated_mode)`` replaces each matched
    gate by a ``NoiseGate`` holding Kraus operators K_i . U
    (noise_model.py:152-185, QuantumNoiseError.apply_to_gate noise_error.py:132-138).
    As in the reference, every matching error absorbs the gate separately, so
    two errors attached to the same gate name apply U twice; attach one
    composed error per gate to model "gate followed by channels".
  * Kraus sets: Pauli / bit-flip / phase-flip errors, DepolarizingError
    (probabilities [1 - p (4^k-1)/4^k, p/4^k, ...] over Pauli strings,
    noise_error.py:239-263) and DampingError (noise_error.py:266-338);
    ``compose`` (operators A . B, outer loop over self) and ``tensor`` (kron).
  * ``ReadoutError`` / ``apply_readout_error`` (readout_error.py,
    noise_model.py:187-215): measured bits are re-drawn from the confusion row.
"""
from __future__ import annotations

from enum import Enum
from itertools import product
from typing import List, Optional, Sequence, Tuple, Union

import numpy as np

_PAULI = {
    "i": np.eye(2, dtype=np.complex128),
    "x": np.array([[0, 1], [1, 0]], dtype=np.complex128),
    "y": np.array([[0, -1j], [1j, 0]], dtype=np.complex128),
    "z": np.array([[1, 0], [0, -1]], dtype=np.complex128),
}


class NoiseChannel(Enum):
    unitary = "Unitary Channel"
    pauil = "Pauli Channel"
    depolarizing = "Depolarizing Channel"
    damping = "Damping Channel"
    readout = "Readout Channel"


def is_kraus_ops(kraus: Sequence[np.ndarray]) -> bool:
    d = kraus[0].shape[0]
    if any(k.shape != (d, d) for k in kraus) or d & (d - 1):
        return False
    s = sum(np.conj(k.T) @ k for k in kraus)
    return bool(np.allclose(s, np.eye(d), rtol=1e-4))


class QuantumNoiseError:
    """Noise error from [(matrix, probability)]; Kraus operators sqrt(p) * M."""

    def __init__(self, ops: List[Tuple[np.ndarray, float]]):
        if not isinstance(ops, list) or not ops:
            raise TypeError("QuantumNoiseError.ops must be a non-empty list of (matrix, prob)")
        self.operators = [(np.asarray(m, dtype=np.complex128), float(p)) for m, p in ops]
        if not is_kraus_ops(self.kraus):
            raise ValueError("the operators do not form a Kraus set")
        self._qubits = int(np.log2(self.operators[0][0].shape[0]))
        self._type = NoiseChannel.unitary

    @property
    def kraus(self) -> List[np.ndarray]:
        return [np.sqrt(p) * m for m, p in self.operators]

    def kraus_array(self) -> np.ndarray:
        """The Kraus operators stacked, shape (count, 2^q, 2^q); built once and
        rebuilt when `operators` is replaced.  Read-only: it is shared."""
        ops = self.operators
        c = self.__dict__.get("_kraus_cache")
        if c is None or c[0] is not ops or c[1] != len(ops):
            arr = np.sqrt(np.array([p for _, p in ops], dtype=np.float64))[:, None, None] * np.array([m for m, _ in ops])
            arr.setflags(write=False)
            c = self._kraus_cache = (ops, len(ops), arr)
        return c[2]

    @property
    def kraus_ct(self) -> List[np.ndarray]:
        return [np.conj(k.T) for k in self.kraus]

    @property
    def qubits(self) -> int:
        return self._qubits

    @property
    def type(self) -> NoiseChannel:
        return self._type

    @type.setter
    def type(self, t: NoiseChannel):
        self._type = t

    def expand(self, extend_qubits: int) -> "QuantumNoiseError":
        eye = np.eye(1 << extend_qubits, dtype=np.complex128)
        return QuantumNoiseError([(np.kron(m, eye), p) for m, p in self.operators])

    def compose(self, other: "QuantumNoiseError") -> "QuantumNoiseError":
        left, right = self.operators, other.operators
        if self.qubits > other.qubits:
            right = other.expand(self.qubits - other.qubits).operators
        elif self.qubits < other.qubits:
            left = self.expand(other.qubits - self.qubits).operators
        return QuantumNoiseError([(a @ b, pa * pb) for a, pa in left for b, pb in right])

    def tensor(self, other: "QuantumNoiseError") -> "QuantumNoiseError":
        return QuantumNoiseError([(np.kron(a, b), pa * pb) for a, pa in self.operators for b, pb in other.operators])

    def apply_to_gate(self, matrix: np.ndarray) -> List[np.ndarray]:
        return list(self.apply_to_gate_array(matrix))

    def apply_to_gate_array(self, matrix: np.ndarray) -> np.ndarray:
        """K_i @ matrix for every Kraus operator, stacked (one batched product)."""
        m = np.asarray(matrix, dtype=np.complex128)
        if m.shape != (1 << self._qubits, 1 << self._qubits):
            raise ValueError("gate matrix size does not match the noise's qubit number")
        return np.matmul(self.kraus_array(), m)

    def prob_mapping_operator(self, prob: float) -> np.ndarray:
        for m, p in self.operators:
            if prob < p:
                return m
            prob -= p
        return self.operators[-1][0]


class PauliError(QuantumNoiseError):
    def __init__(self, ops: List[Tuple[str, float]], num_qubits: int = 1):
        mats = []
        for s, p in ops:
            if len(s) != num_qubits and num_qubits > 1:
                raise ValueError("Pauli string length must equal num_qubits")
            m = _PAULI[s[0]]
            for c in s[1:]:
                m = np.kron(m, _PAULI[c]) if num_qubits > 1 else m @ _PAULI[c]
            mats.append((m, p))
        super().__init__(mats)
        self.type = NoiseChannel.pauil


class BitflipError(PauliError):
    def __init__(self, prob: float):
        super().__init__([("i", 1 - prob), ("x", prob)])


class PhaseflipError(PauliError):
    def __init__(self, prob: float):
        super().__init__([("i", 1 - prob), ("z", prob)])


class PhaseBitflipError(PauliError):
    def __init__(self, prob: float):
        super().__init__([("i", 1 - prob), ("y", prob)])


class DepolarizingError(PauliError):
    def __init__(self, prob: float, num_qubits: int = 1):
        num = 4 ** num_qubits
        maxp = num / (num - 1)
        if prob < 0 or prob > maxp:
            raise ValueError(f"DepolarizingError.prob must lie in [0, {maxp}]")
        probs = [1 - prob / maxp] + [prob / num] * (num - 1)
        strings = ["".join(s) for s in product("ixyz", repeat=num_qubits)]
        super().__init__(list(zip(strings, probs)), num_qubits)
        self.type = NoiseChannel.depolarizing


class DampingError(QuantumNoiseError):
    def __init__(self, amplitude_prob: float, phase_prob: float, dissipation_state: float = 0.0):
        if amplitude_prob + phase_prob > 1:
            raise ValueError("amplitude and phase damping probabilities must sum to <= 1")
        self.amplitude_prob, self.phase_prob, self.dissipation_state = amplitude_prob, phase_prob, dissipation_state
        m0, m1 = np.sqrt(1 - dissipation_state), np.sqrt(dissipation_state)
        sa, sp, sap = np.sqrt(amplitude_prob), np.sqrt(phase_prob), np.sqrt(1 - amplitude_prob - phase_prob)
        ks = [m0 * np.array([[1, 0], [0, sap]]), m0 * np.array([[0, sa], [0, 0]]),
              m0 * np.array([[0, 0], [0, sp]]), m1 * np.array([[sap, 0], [0, 1]]),
              m1 * np.array([[0, 0], [sa, 0]]), m1 * np.array([[sp, 0], [0, 0]])]
        probs = [a * b for a, b in product([1 - dissipation_state, dissipation_state],
                                           [1 - amplitude_prob - phase_prob, amplitude_prob, phase_prob])]
        super().__init__([(k.astype(np.complex128), 1.0) for k, p in zip(ks, probs) if p != 0])
        self.type = NoiseChannel.damping


class ReadoutError:
    """Confusion matrix P[m][n] = p(reading n | true m)."""

    def __init__(self, prob):
        p = np.asarray(prob, dtype=np.float64)
        if p.ndim != 2 or p.shape[0] != p.shape[1] or p.shape[0] & (p.shape[0] - 1):
            raise ValueError("ReadoutError.prob must be 2^n x 2^n")
        if np.any(p < 0) or np.any(p > 1) or not np.allclose(p.sum(axis=1), 1, rtol=1e-6):
            raise ValueError("each row of ReadoutError.prob must be a distribution")
        self._prob = p
        self._qubits = int(np.log2(p.shape[0]))

    prob = property(lambda self: self._prob)
    qubits = property(lambda self: self._qubits)
    type = property(lambda self: NoiseChannel.readout)

    def apply_to_qubits(self, measured_result: int, rng=np.random) -> int:
        u = rng.random()
        for idx, p in enumerate(self._prob[measured_result]):
            if u <= p:
                return idx
            u -= p
        return len(self._prob) - 1


class NoiseGate:
    """Kraus operators standing in for a gate (QuICT/core/operator/noise_gate.py:6-35)."""

    def __init__(self, noise_matrix: List[np.ndarray], args_num: int):
        # a stacked (count, d, d) array is also kept whole for the simulators;
        # noise_matrix then holds read-only views of it
        if isinstance(noise_matrix, np.ndarray) and noise_matrix.ndim == 3:
            stack = np.array(noise_matrix)  # own copy: the caller's array stays writable
            stack.setflags(write=False)
            self._stack = stack
            self.noise_matrix = list(stack)
            self._views = tuple(self.noise_matrix)
        else:
            self._stack = None
            self.noise_matrix = [np.asarray(k) for k in noise_matrix]
        self.targets = args_num
        self.targs: List[int] = []
        self.cargs: List[int] = []
        self.type = "noise"

    def __and__(self, targets):
        self.targs = [targets] if isinstance(targets, int) else list(targets)
        return self

    def kraus_stack(self) -> Optional[np.ndarray]:
        """The stacked Kraus operators, or None when there is no stack or
        `noise_matrix` no longer holds exactly its views."""
        if self._stack is None:
            return None
        nm = self.noise_matrix
        if len(nm) != len(self._views) or any(a is not b for a, b in zip(nm, self._views)):
            return None
        return self._stack

    def __or__(self, circuit):
        circuit.append(self)

    def convert_precision(self):
        pass


class NoiseModel:
    _BASED_GATES = ["h", "s", "sdg", "x", "y", "z", "rx", "ry", "rz", "u1", "t", "tdg", "cx", "cz", "crz", "cu1"]

    def __init__(self, name: str = "Noise Model", basic_gates: Optional[List[str]] = None):
        self._name = name
        self._basic_gates = list(basic_gates) if basic_gates is not None else list(self._BASED_GATES)
        self._error_by_gate = {g: [] for g in self._basic_gates}
        self._readout_errors: List[Tuple[ReadoutError, List[int]]] = []
        self._version = 0  # bumped by every change (simulators key cached lowerings on it)

    def add(self, noise: QuantumNoiseError, gates: Union[str, List[str]], qubits=None):
        gates = [gates] if isinstance(gates, str) else list(gates)
        for g in gates:
            if g not in self._basic_gates:
                raise ValueError(f"gate {g} is not in the noise model's basic gates")
            self._error_by_gate[g].append((noise, -1 if qubits is None else
                                           ([qubits] if isinstance(qubits, int) else list(qubits))))
        self._version += 1

    def add_noise_for_all_qubits(self, noise: QuantumNoiseError, gates: Union[str, List[str]]):
        self.add(noise, gates, None)

    def add_readout_error(self, noise: ReadoutError, qubits: Union[int, List[int]]):
        qubits = [qubits] if isinstance(qubits, int) else list(qubits)
        if noise.qubits > 1 and noise.qubits != len(qubits):
            raise ValueError("multi-qubit readout error needs exactly its qubit count")
        self._readout_errors.append((noise, qubits))
        self._version += 1

    def transpile(self, circuit, accumulated_mode: bool = False, rng=np.random):
        from .circuit import Circuit
        from .gate import UnitaryGate, BasicGate
        out = Circuit(circuit.width())
        for g in circuit.gates:
            if isinstance(getattr(g, "type", None), Enum) and g.type.name in self._basic_gates:
                args = list(g.cargs) + list(g.targs)
                keep = True
                for noise, qubits in self._error_by_gate[g.type.name]:
                    if qubits == -1 or set(args) <= set(qubits):
                        if accumulated_mode or noise.type == NoiseChannel.damping:
                            ng = NoiseGate(noise.apply_to_gate_array(g.matrix), len(args))
                            ng.targs = list(args)
                            out.gates.append(ng)
                            keep = False
                        else:
                            m = noise.prob_mapping_operator(rng.random())
                            u = UnitaryGate.from_matrix(m)
                            u.targs = list(args)
                            out.gates.append(u)
                if keep:
                    out.gates.append(g)
            else:
                out.gates.append(g)
        return out

    def apply_readout_error(self, qureg, rng=np.random):
        for err, qubits in self._readout_errors:
            if err.qubits == 1:
                for q in qubits:
                    if qureg[q].measured is None:
                        continue
                    qureg[q].measured = err.apply_to_qubits(int(qureg[q].measured), rng)
            else:
                if any(qureg[q].measured is None for q in qubits):
                    continue
                v = 0
                for q in qubits:
                    v = (v << 1) | int(qureg[q].measured)
                r = err.apply_to_qubits(v, rng)
                for q in qubits[::-1]:
                    qureg[q].measured = r & 1
                    r >>= 1

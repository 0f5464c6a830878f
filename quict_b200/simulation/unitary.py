"""Drop-in UnitarySimulator (QuICT/simulation/unitary/unitary_simulator.py:12-157).

The reference forms the circuit unitary with dense embeddings
(CircuitMatrix, QuICT/core/utils/circuit_matrix.py) and multiplies it into the
state.  Here the unitary is built by running the circuit on all 2^n basis
columns at once: a 2n-bit vector whose top n bits index the column, set to
the identity, pushed through the same fused passes as a state vector (gates
act on the low n bits only), then read as U[row, col].
"""
from __future__ import annotations

from typing import Optional

import numpy as np
import torch

from .. import _native as N
from .engine import Engine, require_cuda
from .lowering import lower_circuit
from .state_vector import StateArray, StateVectorSimulator


class UnitarySimulator:
    MAX_QUBITS = 15  # 4^15 complex128 = 16 GiB

    def __init__(self, device: str = "GPU", precision: str = "double", *, gpu_device_id: int = 0, seed=None):
        if device != "GPU":
            raise ValueError(f"UnitarySimulator.device must be 'GPU' (quict_b200 has no CPU path), got {device!r}")
        self._precision = np.complex128 if precision == "double" else np.complex64
        self._tdtype = torch.complex128 if precision == "double" else torch.complex64
        self._tdev = require_cuda(gpu_device_id)
        self._engine = Engine(self._tdev)
        self._sv = StateVectorSimulator("GPU", precision, gpu_device_id, seed=seed)
        self._unitary_matrix: Optional[torch.Tensor] = None
        self._vector: Optional[torch.Tensor] = None
        self._qubits_num = 0

    @property
    def vector(self) -> StateArray:
        return StateArray(self._vector)

    @vector.setter
    def vector(self, vec):
        self._vector = torch.as_tensor(np.asarray(vec), dtype=self._tdtype).to(self._tdev)

    def initial_vector_state(self):
        """|0...0> of the current qubit count (unitary_simulator.py:49-57)."""
        self._vector = torch.zeros(1 << self._qubits_num, dtype=self._tdtype, device=self._tdev)
        self._vector[0] = 1

    def get_unitary_matrix(self, circuit) -> StateArray:
        n = int(circuit.width())
        if n > self.MAX_QUBITS:
            raise ValueError(f"a {n}-qubit unitary does not fit (limit {self.MAX_QUBITS} qubits)")
        cols = torch.zeros((1 << n, 1 << n), dtype=self._tdtype, device=self._tdev)
        cols.diagonal().fill_(1)  # row j = basis column j
        ops = lower_circuit(circuit.gates, n)
        self._engine.apply_ops(cols.view(-1), 2 * n, ops)
        self._unitary_matrix = cols.t().contiguous()
        return StateArray(self._unitary_matrix)

    def run(self, circuit, state_vector=None, use_previous: bool = False) -> StateArray:
        """U(circuit) applied to |0...0> (or `state_vector`); `circuit` may also be
        a 2^n x 2^n matrix.  The unitary is kept in ``self._unitary_matrix``."""
        if isinstance(circuit, np.ndarray) or isinstance(circuit, torch.Tensor):
            u = torch.as_tensor(np.asarray(circuit) if isinstance(circuit, np.ndarray) else circuit,
                                dtype=self._tdtype).to(self._tdev)
            if u.dim() != 2 or u.shape[0] != u.shape[1] or u.shape[0] & (u.shape[0] - 1):
                raise ValueError("The unitary matrix should be square with a power-of-two size.")
            self._unitary_matrix = u
            self._qubits_num = int(u.shape[0]).bit_length() - 1
        else:
            self._qubits_num = int(circuit.width())
            self.get_unitary_matrix(circuit)
        n = self._qubits_num
        if state_vector is not None:
            v = torch.as_tensor(np.asarray(state_vector), dtype=self._tdtype).to(self._tdev)
            if v.numel() != (1 << n):
                raise ValueError("The state vector should have the same qubits as the circuit.")
        elif use_previous and self._vector is not None and self._vector.numel() == (1 << n):
            v = self._vector
        else:
            v = torch.zeros(1 << n, dtype=self._tdtype, device=self._tdev)
            v[0] = 1
        self._vector = torch.mv(self._unitary_matrix, v)
        return self.vector

    def sample(self, shots: int, uniforms=None, mode: str = "cdf", seed=None):
        """Counts of `shots` measurements of the last result vector."""
        if self._vector is None:
            raise RuntimeError("UnitarySimulator sample without run any circuit.")
        from ..core import Circuit
        self._sv._circuit = Circuit(self._qubits_num)
        self._sv._qubits = self._qubits_num
        self._sv._vector = self._vector
        return self._sv.sample(shots, uniforms=uniforms, mode=mode, seed=seed)

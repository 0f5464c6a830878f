"""Circuit / Qureg compatible with QuICT.core (the parts the simulators use).

- ``Circuit(wires)``, ``gate | circuit(indexes)``, ``circuit.gates``,
  ``width()``, ``size()``, ``qubits`` (QuICT/core/circuit/circuit.py:105-423).
- ``Qureg`` converts to an int big-endian: qubit 0 is the most significant
  bit (QuICT/core/qubit/qubit.py:192-213).
- ``get_lastcall_for_each_qubits`` (QuICT/core/utils/circuit_info.py:153-167).
- CheckPoints and composite gates: ``cp | circuit`` marks the current end,
  ``cgate | circuit`` inserts at the mark of the composite gate's checkpoint
  child, and ``find_position`` moves the marks (circuit.py:297-360).
"""
from __future__ import annotations

from typing import List, Optional, Sequence, Union

import numpy as np

from .gate import GATE_BY_NAME, BasicGate, GateType


class Qubit:
    def __init__(self):
        self.measured: Optional[int] = None

    def __int__(self) -> int:
        if self.measured is None:
            raise ValueError("qubit has not been measured")
        return int(self.measured)


class Qureg(list):
    """List of Qubit; int(qureg) is the big-endian integer of measured bits."""

    def __int__(self) -> int:
        v = 0
        for q in self:
            v = (v << 1) | int(q)
        return v

    def __call__(self, idx):
        if isinstance(idx, int):
            return Qureg([self[idx]])
        return Qureg([self[i] for i in idx])


class Circuit:
    def __init__(self, wires: int, name: str = "circuit", precision: str = "double"):
        if wires < 1:
            raise ValueError("a circuit needs at least one qubit")
        self.name = name
        self._qubits = Qureg(Qubit() for _ in range(wires))
        self._gates: List = []
        self._checkpoints: List = []
        self._pointer: Optional[List[int]] = None
        self._precision = np.complex128 if precision == "double" else np.complex64

    # ---- QuICT surface --------------------------------------------------------
    @property
    def qubits(self) -> Qureg:
        return self._qubits

    @property
    def gates(self) -> list:
        return self._gates

    @gates.setter
    def gates(self, gates):
        self._gates = list(gates)

    def width(self) -> int:
        return len(self._qubits)

    def size(self) -> int:
        return len(self._gates)

    def __call__(self, indexes: Union[int, Sequence[int]]) -> "Circuit":
        self._pointer = [indexes] if isinstance(indexes, int) else list(indexes)
        return self

    def __getitem__(self, item):
        return self._qubits[item]

    def append(self, op, insert_idx: int = -1):
        from .operator import CheckPoint
        args = self._pointer
        self._pointer = None
        if isinstance(op, BasicGate):
            self._add_gate(op, args, insert_idx)
        elif isinstance(op, CheckPoint):
            # a mark at the current end (check_point.py:44-47); not a gate
            op._pos = self.size()
            self._checkpoints.append(op)
        else:
            # operators (NoiseGate, Trigger-like): keep as given
            if args is not None and hasattr(op, "targs"):
                if len(args) != getattr(op, "targets", len(args)):
                    raise ValueError(f"operator acts on {op.targets} qubits, got {len(args)}")
                op.targs = list(args)
            if insert_idx < 0:
                self._gates.append(op)
            else:
                self._gates.insert(insert_idx, op)

    def extend(self, gates):
        """Append `gates` (a list or a CompositeGate).  A composite gate with
        a checkpoint child goes in at its checkpoint's mark (circuit.py:340-360);
        ``circuit(qubits)`` before it maps the composite gate's qubit i to
        qubits[i]."""
        from .operator import CompositeGate
        mapping = self._pointer
        self._pointer = None
        position = -1
        if isinstance(gates, CompositeGate):
            position = self.find_position(gates.checkpoint)
            gates = gates.gates
        for g in gates:
            if isinstance(g, BasicGate):
                g = g.copy()
                if mapping is not None:
                    g.cargs = [mapping[q] for q in g.cargs]
                    g.targs = [mapping[q] for q in g.targs]
                self._add_gate(g, None, position)
            elif position < 0:
                self._gates.append(g)
            else:
                self._gates.insert(position, g)
            if position >= 0:
                position += 1

    def find_position(self, cp_child) -> int:
        """Mark of the checkpoint `cp_child` belongs to (-1 for None); that
        mark and every later one then move by the child's shift
        (circuit.py:297-310)."""
        position = -1
        if cp_child is None:
            return position
        for cp in self._checkpoints:
            if cp.uid == cp_child.uid:
                position = cp.position
                cp.position = cp_child.shift
            elif position != -1:
                cp.position = cp_child.shift
        return position

    def _add_gate(self, gate: BasicGate, args: Optional[List[int]], insert_idx: int = -1):
        size = gate.controls + gate.targets
        if args is None:
            assigned = gate.cargs + gate.targs
            if assigned:
                args = assigned
            elif size == 1:
                for q in range(self.width()):
                    self._add_gate(gate, [q], insert_idx)
                    if insert_idx >= 0:
                        insert_idx += 1
                return
            elif size == self.width():
                args = list(range(self.width()))
            else:
                raise ValueError(f"{gate.type.name} needs qubits to be assigned")
        if len(args) != size:
            raise ValueError(f"{gate.type.name} acts on {size} qubits, got {len(args)}")
        if any(a < 0 or a >= self.width() for a in args) or len(set(args)) != len(args):
            raise ValueError(f"bad qubit arguments {args} for a {self.width()}-qubit circuit")
        g = gate.copy()
        g.cargs = list(args[:gate.controls])
        g.targs = list(args[gate.controls:])
        if g.precision != self._precision:
            g.convert_precision()
        if insert_idx < 0:
            self._gates.append(g)
        else:
            self._gates.insert(insert_idx, g)

    def get_lastcall_for_each_qubits(self) -> List[Optional[GateType]]:
        last: List[Optional[GateType]] = [None] * self.width()
        for g in self._gates:
            if isinstance(g, BasicGate):
                for q in g.cargs + g.targs:
                    last[q] = g.type
        return last

    def convert_precision(self):
        self._precision = np.complex64 if self._precision == np.complex128 else np.complex128
        for g in self._gates:
            if hasattr(g, "convert_precision"):
                g.convert_precision()

    def reset_qubits(self):
        for q in self._qubits:
            q.measured = None

    def qasm(self) -> str:
        """OpenQASM 2.0 text of the circuit (QuICT's ``Circuit.qasm``)."""
        from .qasm import dumps
        return dumps(self)

    def random_append(self, rand_size: int = 10, typelist: Optional[list] = None, random_params: bool = True,
                      seed: Optional[int] = None):
        """Append `rand_size` gates drawn uniformly from `typelist` on distinct random qubits.

        Uses numpy's default_rng(seed); angles are uniform in [0, 2*pi).
        """
        rng = np.random.default_rng(seed)
        if typelist is None:
            typelist = [GateType.h, GateType.x, GateType.rx, GateType.ry, GateType.rz, GateType.u3,
                        GateType.cx, GateType.cz, GateType.rzz, GateType.swap]
        for _ in range(rand_size):
            t = typelist[rng.integers(len(typelist))]
            tmpl = GATE_BY_NAME[t.name]
            size = tmpl.controls + tmpl.targets
            qs = [int(q) for q in rng.choice(self.width(), size, replace=False)]
            g = tmpl(*[float(rng.uniform(0, 2 * np.pi)) for _ in range(tmpl.params)]) if tmpl.params else tmpl
            g | self(qs)

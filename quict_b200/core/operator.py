"""Dynamic-circuit operators with QuICT's attribute surface: CompositeGate,
Trigger, CheckPoint and CheckPointChild.

* ``CompositeGate`` (QuICT/core/gate/composite_gate.py:19-215): a gate list;
  ``gate | cg(args)`` appends, ``cg | circuit`` extends the circuit, at the
  position of the composite gate's checkpoint when it has one.
* ``Trigger`` (QuICT/core/operator/trigger.py:9-89): measures its target
  qubits during a run and selects a composite gate by the measured value.
* ``CheckPoint`` / ``CheckPointChild`` (QuICT/core/operator/check_point.py):
  a marked index of a circuit; a composite gate holding the child is inserted
  there, and the mark then moves by the child's shift.
"""
from __future__ import annotations

import itertools
from typing import Callable, Dict, List, Optional, Sequence, Union

from .gate import BasicGate

_uid = itertools.count()


class CheckPoint:
    """A mark at the circuit's current end (``cp | circuit``)."""

    def __init__(self):
        self._uid = f"cp{next(_uid)}"
        self._pos = -1

    @property
    def uid(self) -> str:
        return self._uid

    @property
    def position(self) -> int:
        return self._pos

    @position.setter
    def position(self, shift: int):
        # the reference's setter moves the mark by `shift` (check_point.py:27-31)
        if not isinstance(shift, int):
            raise TypeError("CheckPoint.position shift must be an int")
        self._pos += shift

    def get_child(self, shift: int = 0) -> "CheckPointChild":
        if not isinstance(shift, int):
            raise TypeError("CheckPoint.get_child shift must be an int")
        return CheckPointChild(self._uid, shift)

    def match(self, uid: str) -> bool:
        return uid == self._uid

    def __or__(self, circuit):
        circuit.append(self)


class CheckPointChild:
    """Binds a composite gate to its CheckPoint (``child | cgate``)."""

    def __init__(self, uid: str, shift: int = 0):
        self._uid = uid
        self._shift = shift

    @property
    def uid(self) -> str:
        return self._uid

    @property
    def shift(self) -> int:
        return self._shift

    def __or__(self, cgate: "CompositeGate"):
        cgate.append(self)


class CompositeGate:
    """An ordered gate list with an optional checkpoint child."""

    def __init__(self, name: Optional[str] = None, gates: Optional[Sequence[BasicGate]] = None):
        self.name = name or f"composite_gate_{next(_uid)}"
        self._gates: List[BasicGate] = []
        self._pointer: Optional[List[int]] = None
        self._check_point: Optional[CheckPointChild] = None
        if gates is not None:
            for g in gates:
                self.append(g)

    @property
    def gates(self) -> List[BasicGate]:
        return self._gates

    @property
    def checkpoint(self) -> Optional[CheckPointChild]:
        return self._check_point

    def size(self) -> int:
        return len(self._gates)

    def width(self) -> int:
        qs = {q for g in self._gates for q in list(g.cargs) + list(g.targs)}
        return max(qs) + 1 if qs else 0

    def __call__(self, indexes: Union[int, Sequence[int]]) -> "CompositeGate":
        self._pointer = [indexes] if isinstance(indexes, int) else list(indexes)
        return self

    def append(self, op):
        args = self._pointer
        self._pointer = None
        if isinstance(op, CheckPointChild):
            self._check_point = op
            return
        if isinstance(op, BasicGate):
            g = op.copy()
            if args is not None:
                if len(args) != op.controls + op.targets:
                    raise ValueError(f"{op.type.name} acts on {op.controls + op.targets} qubits, got {len(args)}")
                g.cargs = list(args[:op.controls])
                g.targs = list(args[op.controls:])
            self._gates.append(g)
            return
        self._gates.append(op)

    def extend(self, gates):
        for g in (gates.gates if isinstance(gates, CompositeGate) else gates):
            self.append(g)

    def __or__(self, target):
        target.extend(self)

    def __iter__(self):
        return iter(self._gates)

    def __len__(self) -> int:
        return len(self._gates)


class Trigger:
    """Measures `targets` qubits during a run and maps the measured value
    (big-endian over its target qubits) to a CompositeGate, a gate or None."""

    def __init__(self, targets: int,
                 state_gate_mapping: Union[Dict[int, object], Sequence[object], Callable[[int], object]]):
        if not isinstance(targets, int) or targets < 1:
            raise TypeError("Trigger targets must be a positive int")
        self.targets = targets
        self.targs: List[int] = []
        if isinstance(state_gate_mapping, (list, tuple)):
            self._map: Union[dict, Callable] = dict(enumerate(state_gate_mapping))
        elif isinstance(state_gate_mapping, dict):
            self._map = dict(state_gate_mapping)
        elif callable(state_gate_mapping):
            self._map = state_gate_mapping
        else:
            raise TypeError("Trigger mapping must be a list, tuple, dict or function")
        for key in (self._map if isinstance(self._map, dict) else range(1 << targets)):
            v = self._map[key] if isinstance(self._map, dict) else self._map(key)
            if not isinstance(v, (CompositeGate, BasicGate, type(None))):
                raise TypeError(f"Trigger mapping value for {key} is {type(v)}, not a CompositeGate/BasicGate/None")

    def mapping(self, state: int):
        if not 0 <= state < (1 << self.targets):
            raise ValueError(f"Trigger state {state} outside [0, {1 << self.targets})")
        if isinstance(self._map, dict):
            return self._map.get(state)
        return self._map(state)

    def __or__(self, circuit):
        circuit.append(self)

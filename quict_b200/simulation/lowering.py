"""Gate -> kernel-op lowering.

The reference routes each gate by ``(matrix_type, controls, targets)`` to one of
~20 CuPy kernels (statevector_simulator.py:202-496).  Here every gate becomes
one ``Op``: a matrix on target vector bits, an optional set of control bits,
and a structural kind chosen from the matrix itself (diagonal, anti-diagonal,
swap-like, dense), which is what decides how many amplitudes a kernel has to
touch.  Structure is read from the matrix rather than trusted from
``matrix_type`` because some reference types do not describe their matrix
(e.g. sqiSwap is typed ``swap`` but mixes |01> and |10>).

Bit convention: QuICT qubit q of an n-qubit circuit is vector bit n-1-q
(qubit.py:192-213); a k-qubit matrix is big-endian over ``cargs + targs``
(utils.py:8-56).
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import List, Optional, Tuple

import numpy as np

# gate type names handled without a matrix
_SKIP = {"id", "barrier"}
_SPECIAL = {"measure", "reset", "perm"}


@dataclass
class Op:
    kind: str                    # "mat" | "diag" | "antidiag" | "swap" | "measure" | "reset" | "perm"
    tbits: Tuple[int, ...]       # target vector bits; matrix-index bit (m-1-j) <-> tbits[j]
    cbits: Tuple[int, ...] = ()  # control vector bits (all must be 1)
    mat: Optional[np.ndarray] = None  # complex128: mat (2^m,2^m), diag (2^m,), antidiag (2,2), swap (4,4)
    perm: Optional[Tuple[int, ...]] = None  # "perm": source qubit of each destination qubit
    qubit: Optional[int] = None   # measure / reset: circuit qubit index
    tag: object = None            # caller data (e.g. parameter index for gradients); blocks merging
    batch: Optional[np.ndarray] = None  # per-instance tables, shape (instances, entries)
    slot: int = -1                # "expect": output slot
    extra: Tuple[int, ...] = ()   # further bits the op needs in its tile (e.g. the psi/lam pair bit)

    @property
    def m(self) -> int:
        return len(self.tbits)

    @property
    def is_diag_expect(self) -> bool:
        return self.kind == "expect" and classify(self.mat) == "diag"

    @property
    def xbits(self) -> frozenset:
        """Bits on which the op is not diagonal (must be tile-resident when fused)."""
        if self.kind in ("mat", "antidiag", "swap") or (self.kind == "expect" and not self.is_diag_expect):
            return frozenset(self.tbits) | frozenset(self.extra)
        return frozenset(self.extra)

    @property
    def zbits(self) -> frozenset:
        """Bits on which the op is block-diagonal (controls, diagonal targets)."""
        z = set(self.cbits)
        if self.kind == "diag" or self.is_diag_expect:
            z |= set(self.tbits)
        return frozenset(z)

    def dense(self) -> np.ndarray:
        """Full 2^m x 2^m target matrix (controls excluded)."""
        if self.kind == "diag":
            return np.diag(self.mat)
        return self.mat


def _is_controlled(m: np.ndarray, controls: int, targets: int) -> bool:
    """m = diag(I, U) with U on the last 2^targets rows / columns."""
    if controls == 0:
        return False
    d = m.shape[0]
    c = d - (1 << targets)
    top = m[:c]
    # the first c rows hold exactly c nonzeros (NaN counts as one), the c
    # diagonal ones all equal to 1; nothing left of U in the last rows
    return (np.count_nonzero(top) == c and bool(np.all(top.diagonal() == 1))
            and not np.count_nonzero(m[c:, :c]))


_EYES = {}


def _eye(d: int) -> np.ndarray:
    e = _EYES.get(d)
    if e is None:
        e = _EYES[d] = np.eye(d, dtype=np.complex128)
    return e


def classify(u: np.ndarray) -> str:
    """Structural kind of a target matrix (exact zero tests)."""
    d = u.shape[0]
    if d == 2:  # scalar tests: most gates are 1-qubit
        if u[0, 1] == 0 and u[1, 0] == 0:
            return "diag"
        if u[0, 0] == 0 and u[1, 1] == 0:
            return "antidiag"
        return "mat"
    # every nonzero (NaN counts as one) on the diagonal / on the swap pattern
    nz = np.count_nonzero(u)
    if nz == np.count_nonzero(u.diagonal()):
        return "diag"
    if d == 4 and nz == sum(1 for x in (u[0, 0], u[1, 2], u[2, 1], u[3, 3]) if x != 0):
        return "swap"
    return "mat"


def lower_gate(gate, n: int, legacy_2q_order: bool = False) -> List[Op]:
    """Lower one QuICT-style gate to zero or one Op."""
    tname = gate.type.name
    if tname in _SKIP:
        return []
    cargs, targs = list(gate.cargs), list(gate.targs)
    args = cargs + targs
    if args and (min(args) < 0 or max(args) >= n):
        bad = next(a for a in args if not 0 <= a < n)
        raise ValueError(f"gate {tname} argument {bad} outside a {n}-qubit circuit")
    if tname == "measure":
        return [Op("measure", (n - 1 - gate.targ,), qubit=gate.targ)]
    if tname == "reset":
        return [Op("reset", (n - 1 - gate.targ,), qubit=gate.targ)]
    if tname == "perm":
        return [Op("perm", tuple(n - 1 - a for a in args), perm=tuple(int(p) for p in gate.pargs))]
    m = np.array(gate.matrix, dtype=np.complex128)  # always our own copy
    if m.ndim != 2 or m.shape[0] != (1 << len(args)):
        raise ValueError(f"gate {tname}: matrix shape {m.shape} does not match {len(args)} qubits")
    if m[0, 0] == 1 and np.array_equal(m, _eye(m.shape[0])):
        return []
    if _is_controlled(m, gate.controls, gate.targets):
        t = 1 << gate.targets
        u = m[-t:, -t:].copy()
        cq, tq = cargs, targs
    else:
        u = m
        cq, tq = [], args
    kind = classify(u)
    if legacy_2q_order and not cq and len(tq) >= 2 and kind == "mat":
        # The reference SV kernels apply an uncontrolled multi-target dense
        # matrix with its argument order reversed (gate_function.py:153-220,
        # cpu_calculator.py:168-186); reproduce that on request.
        tq = tq[::-1]
    tbits = tuple([n - 1 - q for q in tq])
    cbits = tuple([n - 1 - q for q in cq])
    if kind == "diag":
        return [Op("diag", tbits, cbits, u.diagonal().copy())]
    return [Op(kind, tbits, cbits, u)]


def lower_circuit(gates, n: int, legacy_2q_order: bool = False) -> List[Op]:
    ops: List[Op] = []
    for g in gates:
        ops.extend(lower_gate(g, n, legacy_2q_order))
    return ops

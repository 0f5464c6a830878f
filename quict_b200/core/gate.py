"""Gate IR compatible with QuICT.core.gate (the subset the simulators consume).

The simulators read a gate through the attributes QuICT's BasicGate exposes
(QuICT/core/gate/gate.py:21-558): ``type``, ``matrix_type``, ``controls``,
``targets``, ``cargs``, ``targs``, ``pargs``, ``matrix``, ``precision``.  Gate
objects from the real QuICT package work unchanged; this module exists so that
circuits can be built where QuICT is not installed.

Matrix formulas are the textbook definitions QuICT uses (gate.py:561-2721:
H, Rx = [[c, -is], [-is, c]], U3 per gate.py:944-951, Rzz per gate.py:1804-1814,
...).  Each matrix is formed in complex128 and cast to the gate's precision,
as QuICT does.
"""
from __future__ import annotations

import copy
from enum import Enum
from typing import Callable, Optional

import numpy as np


class GateType(Enum):
    """Same members and values as QuICT/core/utils/gate_type.py:4-60."""
    h = "H gate"
    hy = "Self-inverse gate"
    s = "S gate"
    sdg = "The conjugate transpose of Phase gate"
    x = "Pauli-X gate"
    y = "Pauli-Y gate"
    z = "Pauli-Z gate"
    sx = "sqrt(X) gate"
    sy = "sqrt(Y) gate"
    sw = "sqrt(W) gate"
    id = "Identity gate"
    u1 = "U1 gate"
    u2 = "U2 gate"
    u3 = "U3 gate"
    rx = "Rx gate"
    ry = "Ry gate"
    rz = "Rz gate"
    ri = "Ri gate"
    t = "T gate"
    tdg = "The conjugate transpose of T gate"
    phase = "Phase gate"
    gphase = "Global Phase gate"
    cz = "controlled-Z gate"
    cx = "controlled-X gate"
    cy = "controlled-Y gate"
    ch = "controlled-Hadamard gate"
    crz = "controlled-Rz gate"
    cu1 = "controlled-U1 gate"
    cu3 = "controlled-U3 gate"
    fsim = "fSim gate"
    rxx = "Rxx gate"
    ryy = "Ryy gate"
    rzz = "Rzz gate"
    rzx = "Rzx gate"
    swap = "Swap gate"
    cswap = "cswap gate"
    iswap = "iswap gate"
    iswapdg = "The conjugate transpose of iswap gate"
    sqiswap = "square root of iswap gate"
    ccx = "Toffoli gate"
    ccz = "Multi-Control Z Gate"
    ccrz = "CCRz gate"
    measure = "Measure gate"
    reset = "Reset gate"
    barrier = "Barrier gate"
    unitary = "Unitary gate"
    perm = "Permutation gate"
    perm_fx = "Perm-Fx gate"
    qft = "QFT gate"
    iqft = "IQFT gate"


class MatrixType(Enum):
    """Same members and values as QuICT/core/utils/gate_type.py:63-143."""
    normal = "normal matrix"
    diagonal = "diagonal matrix"
    control = "control matrix"
    swap = "swap matrix"
    reverse = "reverse matrix"
    special = "special matrix"
    diag_diag = "diagonal * diagonal"
    ctrl_normal = "control * matrix"
    normal_normal = "normal * normal"
    diag_normal = "diagonal * normal"


_R2 = 1.0 / np.sqrt(2.0)


def _ctrl(u: np.ndarray, controls: int) -> np.ndarray:
    """Block matrix [[I, 0], [0, u]] with `controls` leading control qubits."""
    d = u.shape[0] << controls
    m = np.eye(d, dtype=np.complex128)
    m[d - u.shape[0]:, d - u.shape[0]:] = u
    return m


def _u3(t, p, l):
    c, s = np.cos(t / 2), np.sin(t / 2)
    return np.array([[c, -np.exp(1j * l) * s], [np.exp(1j * p) * s, np.exp(1j * (p + l)) * c]])


def _rz(t):
    return np.diag([np.exp(-0.5j * t), np.exp(0.5j * t)])


# type -> (controls, targets, params, matrix_type, matrix(pargs) -> complex128 ndarray)
_SPEC: dict = {
    GateType.h: (0, 1, 0, MatrixType.normal, lambda p: _R2 * np.array([[1, 1], [1, -1]])),
    GateType.hy: (0, 1, 0, MatrixType.normal, lambda p: _R2 * np.array([[1, -1j], [1j, -1]])),
    GateType.s: (0, 1, 0, MatrixType.control, lambda p: np.diag([1, 1j])),
    GateType.sdg: (0, 1, 0, MatrixType.control, lambda p: np.diag([1, -1j])),
    GateType.x: (0, 1, 0, MatrixType.swap, lambda p: np.array([[0, 1], [1, 0]])),
    GateType.y: (0, 1, 0, MatrixType.reverse, lambda p: np.array([[0, -1j], [1j, 0]])),
    GateType.z: (0, 1, 0, MatrixType.control, lambda p: np.diag([1, -1])),
    GateType.sx: (0, 1, 0, MatrixType.normal, lambda p: np.array([[0.5 + 0.5j, 0.5 - 0.5j], [0.5 - 0.5j, 0.5 + 0.5j]])),
    GateType.sy: (0, 1, 0, MatrixType.normal, lambda p: _R2 * np.array([[1, -1], [1, 1]])),
    GateType.sw: (0, 1, 0, MatrixType.normal,
                  lambda p: np.array([[_R2, -np.sqrt(1j / 2)], [np.sqrt(-1j / 2), _R2]])),
    GateType.id: (0, 1, 0, MatrixType.diagonal, lambda p: np.eye(2)),
    GateType.u1: (0, 1, 1, MatrixType.control, lambda p: np.diag([1, np.exp(1j * p[0])])),
    GateType.u2: (0, 1, 2, MatrixType.normal,
                  lambda p: _R2 * np.array([[1, -np.exp(1j * p[1])],
                                            [np.exp(1j * p[0]), np.exp(1j * (p[0] + p[1]))]])),
    GateType.u3: (0, 1, 3, MatrixType.normal, lambda p: _u3(*p)),
    GateType.rx: (0, 1, 1, MatrixType.normal,
                  lambda p: np.array([[np.cos(p[0] / 2), -1j * np.sin(p[0] / 2)],
                                      [-1j * np.sin(p[0] / 2), np.cos(p[0] / 2)]])),
    GateType.ry: (0, 1, 1, MatrixType.normal,
                  lambda p: np.array([[np.cos(p[0] / 2), -np.sin(p[0] / 2)],
                                      [np.sin(p[0] / 2), np.cos(p[0] / 2)]])),
    GateType.rz: (0, 1, 1, MatrixType.diagonal, lambda p: _rz(p[0])),
    GateType.t: (0, 1, 0, MatrixType.control, lambda p: np.diag([1, np.exp(0.25j * np.pi)])),
    GateType.tdg: (0, 1, 0, MatrixType.control, lambda p: np.diag([1, np.exp(-0.25j * np.pi)])),
    GateType.phase: (0, 1, 1, MatrixType.control, lambda p: np.diag([1, np.exp(1j * p[0])])),
    GateType.gphase: (0, 1, 1, MatrixType.diagonal, lambda p: np.exp(1j * p[0]) * np.eye(2)),
    GateType.cz: (1, 1, 0, MatrixType.control, lambda p: np.diag([1, 1, 1, -1])),
    GateType.cx: (1, 1, 0, MatrixType.reverse, lambda p: _ctrl(np.array([[0, 1], [1, 0]]), 1)),
    GateType.cy: (1, 1, 0, MatrixType.reverse, lambda p: _ctrl(np.array([[0, -1j], [1j, 0]]), 1)),
    GateType.ch: (1, 1, 0, MatrixType.normal, lambda p: _ctrl(_R2 * np.array([[1, 1], [1, -1]]), 1)),
    GateType.crz: (1, 1, 1, MatrixType.diagonal, lambda p: _ctrl(_rz(p[0]), 1)),
    GateType.cu1: (1, 1, 1, MatrixType.control, lambda p: np.diag([1, 1, 1, np.exp(1j * p[0])])),
    GateType.cu3: (1, 1, 3, MatrixType.normal, lambda p: _ctrl(_u3(*p), 1)),
    GateType.fsim: (0, 2, 2, MatrixType.ctrl_normal,
                    lambda p: np.array([[1, 0, 0, 0],
                                        [0, np.cos(p[0]), -1j * np.sin(p[0]), 0],
                                        [0, -1j * np.sin(p[0]), np.cos(p[0]), 0],
                                        [0, 0, 0, np.exp(-1j * p[1])]])),
    GateType.rxx: (0, 2, 1, MatrixType.normal_normal,
                   lambda p: (lambda c, s: np.array([[c, 0, 0, -1j * s], [0, c, -1j * s, 0],
                                                     [0, -1j * s, c, 0], [-1j * s, 0, 0, c]]))(
                       np.cos(p[0] / 2), np.sin(p[0] / 2))),
    GateType.ryy: (0, 2, 1, MatrixType.normal_normal,
                   lambda p: (lambda c, s: np.array([[c, 0, 0, 1j * s], [0, c, -1j * s, 0],
                                                     [0, -1j * s, c, 0], [1j * s, 0, 0, c]]))(
                       np.cos(p[0] / 2), np.sin(p[0] / 2))),
    GateType.rzz: (0, 2, 1, MatrixType.diag_diag,
                   lambda p: np.diag([np.exp(-0.5j * p[0]), np.exp(0.5j * p[0]),
                                      np.exp(0.5j * p[0]), np.exp(-0.5j * p[0])])),
    GateType.rzx: (0, 2, 1, MatrixType.diag_normal,
                   lambda p: (lambda c, s: np.array([[c, -1j * s, 0, 0], [-1j * s, c, 0, 0],
                                                     [0, 0, c, 1j * s], [0, 0, 1j * s, c]]))(
                       np.cos(p[0] / 2), np.sin(p[0] / 2))),
    GateType.swap: (0, 2, 0, MatrixType.swap,
                    lambda p: np.array([[1, 0, 0, 0], [0, 0, 1, 0], [0, 1, 0, 0], [0, 0, 0, 1]])),
    GateType.iswap: (0, 2, 0, MatrixType.swap,
                     lambda p: np.array([[1, 0, 0, 0], [0, 0, 1j, 0], [0, 1j, 0, 0], [0, 0, 0, 1]])),
    GateType.iswapdg: (0, 2, 0, MatrixType.swap,
                       lambda p: np.array([[1, 0, 0, 0], [0, 0, -1j, 0], [0, -1j, 0, 0], [0, 0, 0, 1]])),
    GateType.sqiswap: (0, 2, 0, MatrixType.swap,
                       lambda p: np.array([[1, 0, 0, 0], [0, _R2, 1j * _R2, 0],
                                           [0, 1j * _R2, _R2, 0], [0, 0, 0, 1]])),
    GateType.cswap: (1, 2, 0, MatrixType.swap,
                     lambda p: _ctrl(np.array([[1, 0, 0, 0], [0, 0, 1, 0], [0, 1, 0, 0], [0, 0, 0, 1]]), 1)),
    GateType.ccx: (2, 1, 0, MatrixType.reverse, lambda p: _ctrl(np.array([[0, 1], [1, 0]]), 2)),
    GateType.ccz: (2, 1, 0, MatrixType.normal, lambda p: _ctrl(np.diag([1, -1]), 2)),
    GateType.ccrz: (2, 1, 1, MatrixType.diagonal, lambda p: _ctrl(_rz(p[0]), 2)),
    GateType.measure: (0, 1, 0, MatrixType.special, None),
    GateType.reset: (0, 1, 0, MatrixType.special, None),
    GateType.barrier: (0, 1, 0, MatrixType.special, None),
}

_QASM_NAME = {GateType.sdg: "sdg", GateType.tdg: "tdg", GateType.id: "id"}


class BasicGate:
    """A quantum gate: QuICT's BasicGate attribute surface without the QCDA parts."""

    def __init__(self, gtype: GateType, controls: int = 0, targets: int = 1, params: int = 0,
                 matrix_type: MatrixType = MatrixType.normal,
                 matrix_fn: Optional[Callable] = None, matrix: Optional[np.ndarray] = None):
        self._type = gtype
        self._controls = controls
        self._targets = targets
        self._params = params
        self._matrix_type = matrix_type
        self._matrix_fn = matrix_fn
        self._static = matrix
        self._precision = np.complex128
        self._cargs: list = []
        self._targs: list = []
        self._pargs: list = []
        self.assigned_qubits: list = []

    # ---- QuICT attribute surface ----------------------------------------------
    type = property(lambda self: self._type)
    matrix_type = property(lambda self: self._matrix_type)
    controls = property(lambda self: self._controls)
    targets = property(lambda self: self._targets)
    params = property(lambda self: self._params)
    precision = property(lambda self: self._precision)
    qasm_name = property(lambda self: _QASM_NAME.get(self._type, self._type.name))

    @property
    def name(self) -> str:
        return self._type.name

    @property
    def cargs(self) -> list:
        return self._cargs

    @cargs.setter
    def cargs(self, v):
        self._cargs = [v] if isinstance(v, int) else list(v)

    @property
    def targs(self) -> list:
        return self._targs

    @targs.setter
    def targs(self, v):
        self._targs = [v] if isinstance(v, int) else list(v)

    @property
    def pargs(self) -> list:
        return self._pargs

    @pargs.setter
    def pargs(self, v):
        self._pargs = list(v) if isinstance(v, (list, tuple)) else [v]

    carg = property(lambda self: self._cargs[0])
    targ = property(lambda self: self._targs[0])
    parg = property(lambda self: self._pargs[0])

    @property
    def matrix(self) -> Optional[np.ndarray]:
        """A fresh copy in the gate's precision.  A parametrised matrix is
        rebuilt only when the parameters change (kept with the gate)."""
        if self._static is not None:
            m = self._static
        elif self._matrix_fn is not None:
            key = tuple(self._pargs)
            cached = self.__dict__.get("_mcache")
            if cached is not None and cached[0] == key:
                m = cached[1]
            else:
                m = np.asarray(self._matrix_fn(self._pargs), dtype=np.complex128)
                self._mcache = (key, m)
        else:
            return None
        return m.astype(self._precision)

    @property
    def target_matrix(self) -> Optional[np.ndarray]:
        m = self.matrix
        if m is None or self._controls == 0:
            return m
        d = 1 << self._targets
        return m[-d:, -d:]

    def is_single(self) -> bool:
        return self._controls + self._targets == 1

    def is_identity(self) -> bool:
        m = self.matrix
        return m is not None and np.allclose(m, np.eye(m.shape[0], dtype=m.dtype))

    def convert_precision(self):
        self._precision = np.complex64 if self._precision == np.complex128 else np.complex128

    # ---- construction -------------------------------------------------------------
    def copy(self) -> "BasicGate":
        g = copy.copy(self)
        g._cargs = list(self._cargs)
        g._targs = list(self._targs)
        g._pargs = list(self._pargs)
        g.assigned_qubits = list(self.assigned_qubits)
        return g

    def __call__(self, *pargs) -> "BasicGate":
        g = self.copy()
        if self._params == 0 and pargs:
            raise ValueError(f"{self._type.name} takes no parameters")
        if pargs:
            if len(pargs) != self._params:
                raise ValueError(f"{self._type.name} takes {self._params} parameters, got {len(pargs)}")
            g._pargs = [float(p) if not isinstance(p, complex) else p for p in pargs]
        return g

    def __and__(self, targets) -> "BasicGate":
        g = self.copy()
        args = [targets] if isinstance(targets, int) else list(targets)
        if len(args) != self._controls + self._targets:
            raise ValueError("the number of qubits must equal the gate's size")
        g._cargs = args[:self._controls]
        g._targs = args[self._controls:]
        return g

    def __or__(self, target):
        target.append(self)

    def inverse(self) -> "BasicGate":
        m = self.matrix
        g = UnitaryGate.from_matrix(np.conj(m.T))
        g._cargs, g._targs = [], list(self._cargs) + list(self._targs)
        return g

    def __repr__(self) -> str:
        return f"{self._type.name}(c={self._cargs}, t={self._targs}, p={self._pargs})"


class UnitaryGate(BasicGate):
    """Custom unitary; ``Unitary(matrix) | circuit([...])`` (gate.py:2235-2328)."""

    def __init__(self):
        super().__init__(GateType.unitary, 0, 0, 0, MatrixType.normal)

    @classmethod
    def from_matrix(cls, m, matrix_type: MatrixType = MatrixType.normal) -> "UnitaryGate":
        m = np.asarray(m, dtype=np.complex128)
        if m.ndim == 1:
            d = int(round(np.sqrt(m.size)))
            m = m.reshape(d, d)
        if m.shape[0] != m.shape[1] or m.shape[0] & (m.shape[0] - 1):
            raise ValueError("unitary matrix must be 2^k x 2^k")
        g = cls()
        g._targets = int(m.shape[0]).bit_length() - 1
        g._static = m
        offdiag = m - np.diag(np.diag(m))
        if g._targets <= 3 and np.allclose(offdiag, 0):
            d = m.shape[0]
            g._matrix_type = (MatrixType.control if np.allclose(m[:d - 1, :d - 1], np.eye(d - 1))
                              else MatrixType.diagonal)
        else:
            g._matrix_type = matrix_type
        return g

    def __call__(self, params, matrix_type: MatrixType = MatrixType.normal) -> "UnitaryGate":
        return UnitaryGate.from_matrix(params, matrix_type)


def _build_matrix(ops, k: int) -> np.ndarray:
    """Dense matrix of a k-qubit gate sequence [(matrix, args)] (big-endian args)."""
    u = np.eye(1 << k, dtype=np.complex128).reshape([2] * k + [1 << k])
    for m, args in ops:
        a = len(args)
        t = np.asarray(m, dtype=np.complex128).reshape([2] * (2 * a))
        u = np.tensordot(t, u, axes=(list(range(a, 2 * a)), list(args)))
        u = np.moveaxis(u, list(range(a)), list(args))
    return u.reshape(1 << k, 1 << k)


class QFTGate(BasicGate):
    """QFT on k qubits: H and CU1(2*pi/2^(j-i+1)) ladder, no final swaps (gate.py:2546-2603)."""

    def __init__(self, targets: int = 3, inverse: bool = False):
        super().__init__(GateType.iqft if inverse else GateType.qft, 0, targets, 0, MatrixType.normal)
        self._inv = inverse

    def __call__(self, targets: int) -> "QFTGate":
        return type(self)(targets, self._inv)

    @property
    def matrix(self) -> np.ndarray:
        k = self._targets
        h = _SPEC[GateType.h][4](None)
        ops = []
        if not self._inv:
            for i in range(k):
                ops.append((h, [i]))
                for j in range(i + 1, k):
                    ops.append((np.diag([1, 1, 1, np.exp(2j * np.pi / (1 << (j - i + 1)))]), [j, i]))
        else:
            for i in range(k - 1, -1, -1):
                for j in range(k - 1, i, -1):
                    ops.append((np.diag([1, 1, 1, np.exp(-2j * np.pi / (1 << (j - i + 1)))]), [j, i]))
                ops.append((h, [i]))
        return _build_matrix(ops, k).astype(self._precision)


class PermGate(BasicGate):
    """Qubit permutation gate (gate.py:2097-2173): pargs[i] is the source index of slot i."""

    def __init__(self, targets: int = 0):
        super().__init__(GateType.perm, 0, targets, targets, MatrixType.special)

    def __call__(self, targets: int, params: list) -> "PermGate":
        g = PermGate(targets)
        if sorted(params) != list(range(targets)):
            raise ValueError("Perm parameters must be a permutation of range(targets)")
        g._pargs = list(params)
        return g


class PermFxGate(BasicGate):
    """Oracle of a boolean function f on n qubits, acting on n + 1:
    |x, y> -> |x, y XOR f(x)>, f(x) = 1 for x in `params`; y is the last
    target (the least significant bit of the big-endian index).  pargs[i]
    is the column of the 1 in row i (gate.py:2176-2229)."""

    def __init__(self, targets: int = 0):
        super().__init__(GateType.perm_fx, 0, targets, 0, MatrixType.normal)

    def __call__(self, n: int, params: list) -> "PermFxGate":
        if not isinstance(params, list) or not isinstance(n, int):
            raise TypeError(f"n must be int ({type(n)}) and params a list ({type(params)})")
        if any(not 0 <= p < (1 << n) for p in params):
            raise ValueError("PermFx params must lie in [0, 2^n)")
        ones = set(int(p) for p in params)
        g = PermFxGate(n + 1)
        g._params = 1 << (n + 1)
        g._pargs = [idx ^ 1 if (idx >> 1) in ones else idx for idx in range(1 << (n + 1))]
        return g

    @property
    def matrix(self) -> np.ndarray:
        d = 1 << self._targets
        m = np.zeros((d, d), dtype=self._precision)
        m[np.arange(d), np.asarray(self._pargs, dtype=np.int64)] = 1
        return m


def _make(t: GateType) -> BasicGate:
    c, tg, p, mt, fn = _SPEC[t]
    if p == 0 and fn is not None:  # a fixed gate: its matrix is built once
        return BasicGate(t, c, tg, p, mt, None, np.asarray(fn([]), dtype=np.complex128))
    return BasicGate(t, c, tg, p, mt, fn)


H = _make(GateType.h)
Hy = _make(GateType.hy)
S = _make(GateType.s)
S_dagger = _make(GateType.sdg)
X = _make(GateType.x)
Y = _make(GateType.y)
Z = _make(GateType.z)
SX = _make(GateType.sx)
SY = _make(GateType.sy)
SW = _make(GateType.sw)
ID = _make(GateType.id)
U1 = _make(GateType.u1)
U2 = _make(GateType.u2)
U3 = _make(GateType.u3)
Rx = _make(GateType.rx)
Ry = _make(GateType.ry)
Rz = _make(GateType.rz)
T = _make(GateType.t)
T_dagger = _make(GateType.tdg)
Phase = _make(GateType.phase)
GPhase = _make(GateType.gphase)
CZ = _make(GateType.cz)
CX = _make(GateType.cx)
CY = _make(GateType.cy)
CH = _make(GateType.ch)
CRz = _make(GateType.crz)
CU1 = _make(GateType.cu1)
CU3 = _make(GateType.cu3)
FSim = _make(GateType.fsim)
Rxx = _make(GateType.rxx)
Ryy = _make(GateType.ryy)
Rzz = _make(GateType.rzz)
Rzx = _make(GateType.rzx)
Swap = _make(GateType.swap)
iSwap = _make(GateType.iswap)
iSwap_dagger = _make(GateType.iswapdg)
sqiSwap = _make(GateType.sqiswap)
CSwap = _make(GateType.cswap)
CCX = _make(GateType.ccx)
CCZ = _make(GateType.ccz)
CCRz = _make(GateType.ccrz)
Measure = _make(GateType.measure)
Reset = _make(GateType.reset)
Barrier = _make(GateType.barrier)
Unitary = UnitaryGate()
QFT = QFTGate()
IQFT = QFTGate(inverse=True)
Perm = PermGate()
PermFx = PermFxGate()

# QASM / generator name -> gate template
GATE_BY_NAME = {
    t.name: _make(t) for t in _SPEC
}
GATE_BY_NAME.update({"unitary": Unitary, "qft": QFT, "iqft": IQFT, "perm": Perm, "perm_fx": PermFx})

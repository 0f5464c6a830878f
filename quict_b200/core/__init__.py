"""QuICT.core-compatible circuit IR (gates, circuits, noise) for the simulators."""
from .gate import *  # noqa: F401,F403
from .gate import BasicGate, GateType, MatrixType, UnitaryGate, QFTGate, PermGate, GATE_BY_NAME  # noqa: F401
from .circuit import Circuit, Qubit, Qureg  # noqa: F401
from .operator import CheckPoint, CheckPointChild, CompositeGate, Trigger  # noqa: F401
from .noise import (NoiseModel, NoiseGate, QuantumNoiseError, PauliError, BitflipError, PhaseflipError,  # noqa: F401
                    PhaseBitflipError, DepolarizingError, DampingError, ReadoutError, NoiseChannel)

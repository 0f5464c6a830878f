"""Simulators: drop-in replacements for QuICT.simulation's GPU backends."""
from .state_vector import StateVectorSimulator, StateArray  # noqa: F401
from .density_matrix import DensityMatrixSimulator  # noqa: F401
from .unitary import UnitarySimulator  # noqa: F401
from .sharded import ShardedStateVector  # noqa: F401
from .simulator import Simulator, Result, SimulatorOptionsUnmatchedError  # noqa: F401

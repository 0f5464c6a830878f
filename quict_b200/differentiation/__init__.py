"""Batched expectation values and adjoint-method gradients (no reference
counterpart: QuICT's ML package is not part of the reference)."""
from .circuit import (GENERATORS, GateEntry, ParamCircuit, PauliSum, hardware_efficient_ansatz,  # noqa: F401
                      ising_observable, maxcut_observable, qaoa_circuit, random_regular_graph, rotation)
from .adjoint import BatchedAdjoint, expectation  # noqa: F401
from .qaoa import UnevenQAOABatch, qaoa_instances  # noqa: F401

"""``Simulator``: QuICT's one-call front end (QuICT/simulation/simulator.py:43-151)
over this package's GPU simulators, with its result record
(QuICT/simulation/utils/result.py:5-110).

Same constructor, option table, argument checks and result dictionary; the
device must be "GPU" (quict_b200 has no CPU path).  ``run`` runs the circuit,
samples ``shots`` times and returns the record: counts keyed by the
zero-padded bit string of every basis index (zeros included, as QuICT does),
and the amplitudes / density matrix as numpy arrays.
"""
from __future__ import annotations

import os
import uuid
from typing import Optional

import numpy as np

from .density_matrix import DensityMatrixSimulator
from .state_vector import StateVectorSimulator
from .unitary import UnitarySimulator


class SimulatorOptionsUnmatchedError(Exception):
    """An option or input that the chosen backend does not take."""


class Result:
    """Record of one ``Simulator.run``: device, backend, options, counts and
    the final amplitudes; optionally dumped under `output_path`."""

    def __init__(self, device: str, backend: str, precision: str, circuit_record: bool, amplitude_record: bool,
                 options: dict, output_path: Optional[str] = None):
        self.device = device
        self.backend = backend
        self.precision = precision
        self._circuit_record = circuit_record
        self._amplitude_record = amplitude_record
        self.options = options
        self.id = uuid.uuid4().hex
        self.shots = 0
        self.counts = {}
        self.state_vector = None
        self.density_matrix = None
        self._dump = circuit_record or amplitude_record
        if self._dump:
            self._output_path = output_path or os.path.join(os.getcwd(), "output")
            os.makedirs(self._output_path, exist_ok=True)

    def __str__(self):
        return f"Device: {self.device}\nBackend: {self.backend}\nOptions: {self.options}\nResults: {self.counts}"

    def __dict__(self):
        return {"id": self.id, "shots": self.shots,
                "backend_info": {"device": self.device, "backend": self.backend, "options": self.options},
                "data": {"counts": self.counts, "state_vector": self.state_vector,
                         "density_matrix": self.density_matrix}}

    def record_circuit(self, circuit):
        self.id = getattr(circuit, "name", None) or self.id
        if self._circuit_record:
            with open(os.path.join(self._output_path, f"circuit_{self.id}.qasm"), "w") as f:
                f.write(circuit.qasm())

    def record_amplitude(self, amplitude):
        a = amplitude.get() if hasattr(amplitude, "get") else np.asarray(amplitude)
        if self._amplitude_record:
            np.savetxt(os.path.join(self._output_path, f"amp_{self.id}.txt"), a)
        if self.backend == "density_matrix":
            self.density_matrix = a.copy()
        else:
            self.state_vector = a.copy()

    def record_sample(self, result: list):
        """Counts keyed by the basis index as a bit string of width log2(len)."""
        self.shots = int(sum(result))
        width = max(len(result) - 1, 0).bit_length()
        self.counts = {format(i, "b").zfill(width): c for i, c in enumerate(result)}
        if self._dump:
            with open(os.path.join(self._output_path, f"result_{self.id}.log"), "w") as f:
                f.write(str(self.__dict__()))


class Simulator:
    """``Simulator(device="GPU", backend="state_vector" | "density_matrix" |
    "unitary", precision="single" | "double", **options)``; options as in
    QuICT: state_vector takes gpu_device_id and matrix_aggregation,
    density_matrix takes accumulated_mode, unitary none."""

    __DEVICE = ["CPU", "GPU"]
    __BACKEND = ["unitary", "state_vector", "density_matrix"]
    __PRECISION = ["single", "double"]
    __OPTIONS_DICT = {"state_vector": ["gpu_device_id", "matrix_aggregation"],
                      "density_matrix": ["accumulated_mode"]}

    def __init__(self, device: str = "GPU", backend: str = "state_vector", precision: str = "double",
                 circuit_record: bool = False, amplitude_record: bool = False, output_path: Optional[str] = None,
                 **options):
        if device not in self.__DEVICE:
            raise ValueError(f"Simulator.device must be one of {self.__DEVICE}, got {device!r}")
        if device != "GPU":
            raise ValueError("Simulator.device must be 'GPU' (quict_b200 has no CPU path)")
        if backend not in self.__BACKEND:
            raise ValueError(f"Simulator.backend must be one of {self.__BACKEND}, got {backend!r}")
        if precision not in self.__PRECISION:
            raise ValueError(f"Simulator.precision must be one of {self.__PRECISION}, got {precision!r}")
        if options and not self._options_valid(backend, options):
            raise SimulatorOptionsUnmatchedError(f"Unmatched options arguments depending on {device} and {backend}.")
        self._device, self._backend, self._precision = device, backend, precision
        self._options = options
        self._simulator = self._load_simulator()
        self._result_recorder = Result(device, backend, precision, circuit_record, amplitude_record, options,
                                       output_path)

    @classmethod
    def _options_valid(cls, backend: str, options: dict) -> bool:
        if backend == "unitary":
            return False
        return all(k in cls.__OPTIONS_DICT[backend] for k in options)

    def _load_simulator(self):
        if self._backend == "state_vector":
            return StateVectorSimulator(self._device, precision=self._precision, **self._options)
        if self._backend == "unitary":
            return UnitarySimulator(device=self._device, precision=self._precision)
        return DensityMatrixSimulator(device=self._device, precision=self._precision, **self._options)

    def run(self, circuit, shots: int = 1, state_vector: np.ndarray = None, density_matrix: np.ndarray = None,
            noise_model=None, use_previous: bool = False) -> dict:
        """Run, sample `shots` times, and return the result record."""
        if isinstance(circuit, np.ndarray) and self._backend != "unitary":
            raise SimulatorOptionsUnmatchedError(
                f"The unitary matrix input only allows in the unitary backend, not {self._backend}.")
        if (density_matrix is not None or noise_model is not None) and self._backend != "density_matrix":
            raise SimulatorOptionsUnmatchedError(
                "The density matrix and noise model input only allows in the density_matrix backend, "
                f"not {self._backend}.")
        if state_vector is not None and self._backend == "density_matrix":
            raise SimulatorOptionsUnmatchedError("The state vector input is not allowed in the density matrix backend.")
        if not isinstance(circuit, np.ndarray):
            self._result_recorder.record_circuit(circuit)
        if self._backend == "density_matrix":
            amplitude = self._simulator.run(circuit, density_matrix, noise_model, use_previous)
        else:
            amplitude = self._simulator.run(circuit, state_vector, use_previous)
        self._result_recorder.record_amplitude(amplitude)
        self._result_recorder.record_sample(self._simulator.sample(shots))
        return self._result_recorder.__dict__()

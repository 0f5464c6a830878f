"""Drop-in StateVectorSimulator (QuICT/simulation/state_vector/statevector_simulator.py:26-626).

Same constructor, ``run`` / ``sample`` / ``vector`` surface and measurement
semantics as the reference GPU simulator; gate application runs on sm_100a
kernels in libqsim instead of per-gate CuPy RawKernels.  Extra keyword
arguments (all optional) select fusion and the tile shape, reproduce the
reference's reversed 2-qubit dense-matrix order (``legacy_2q_order``), and seed
the measurement RNG.
"""
from __future__ import annotations

from typing import List, Optional

import numpy as np
import torch

from .. import _native as N
from .engine import Engine, require_cuda
from .lowering import Op, lower_gate


class StateArray:
    """Device state returned by ``run``; ``.get()`` copies it to a numpy array
    (the CuPy array interface the reference's callers use)."""

    def __init__(self, tensor: torch.Tensor):
        self.tensor = tensor

    def get(self) -> np.ndarray:
        return self.tensor.detach().cpu().numpy()

    @property
    def shape(self):
        return tuple(self.tensor.shape)

    @property
    def dtype(self):
        return np.complex128 if self.tensor.dtype == torch.complex128 else np.complex64

    @property
    def size(self) -> int:
        return self.tensor.numel()

    def __len__(self) -> int:
        return self.tensor.shape[0]

    def __array__(self, dtype=None, copy=None):
        a = self.get()
        return a.astype(dtype) if dtype is not None else a

    @property
    def __cuda_array_interface__(self):
        return self.tensor.__cuda_array_interface__

    def __dlpack__(self, *args, **kwargs):
        return self.tensor.__dlpack__(*args, **kwargs)

    def __dlpack_device__(self):
        return self.tensor.__dlpack_device__()

    def copy(self) -> "StateArray":
        return StateArray(self.tensor.clone())


class StateVectorSimulator:
    __DEVICE = ["GPU"]
    __PRECISION = ["single", "double"]

    def __init__(self, device: str = "GPU", precision: str = "double", gpu_device_id: int = 0,
                 matrix_aggregation: bool = True, sync: bool = True, *, fusion: bool = True,
                 tile_bits: Optional[int] = None, low_bits: Optional[int] = None,
                 max_pass_cost: Optional[float] = None, merge_bits: Optional[int] = None,
                 legacy_2q_order: bool = False, seed: Optional[int] = None, autotune: bool = False):
        if device not in self.__DEVICE:
            raise ValueError(f"StateVectorSimulator.device must be 'GPU' (quict_b200 has no CPU path), got {device!r}")
        if precision not in self.__PRECISION:
            raise ValueError(f"StateVectorSimulator.precision must be one of {self.__PRECISION}, got {precision!r}")
        self._device = device
        self._precision = np.complex128 if precision == "double" else np.complex64
        self._tdtype = torch.complex128 if precision == "double" else torch.complex64
        self._device_id = gpu_device_id
        self._sync = sync
        self._using_matrix_aggregation = matrix_aggregation
        self._legacy = legacy_2q_order
        self._tdev = require_cuda(gpu_device_id)
        # fused-pass knobs left as None come from the tuning cache; with
        # autotune=True a run whose size has no cache entry tunes them first
        self._engine = Engine(self._tdev, fusion=fusion, tile_bits=tile_bits, low_bits=low_bits,
                              max_pass_cost=max_pass_cost, merge_bits=merge_bits)
        self._autotune = autotune
        # measurement uniforms: a seed, or any object with a .random() method
        self._rng = seed if hasattr(seed, "random") else np.random.default_rng(seed)
        self._circuit = None
        self._qubits = 0
        self._vector: Optional[torch.Tensor] = None
        self.last_sample_indices: Optional[torch.Tensor] = None
        self._lowered: dict = {}  # circuit key -> lowered ops (recent circuits)

    # ---- reference properties ---------------------------------------------------------
    @property
    def circuit(self):
        return self._circuit

    @circuit.setter
    def circuit(self, circuit):
        self._circuit = circuit

    @property
    def device(self):
        return self._device_id

    @property
    def engine(self) -> Engine:
        return self._engine

    @property
    def vector(self) -> StateArray:
        return StateArray(self._vector)

    @vector.setter
    def vector(self, vec):
        self._vector = self._to_device(vec)

    def _to_device(self, vec) -> torch.Tensor:
        if isinstance(vec, StateArray):
            vec = vec.tensor
        if isinstance(vec, torch.Tensor):
            return vec.to(device=self._tdev, dtype=self._tdtype).contiguous()
        return torch.from_numpy(np.ascontiguousarray(vec, dtype=self._precision)).to(self._tdev)

    # ---- run ------------------------------------------------------------------------
    def initial_circuit(self, circuit):
        self._circuit = circuit
        self._qubits = int(circuit.width())

    def initial_state_vector(self, all_zeros: bool = False):
        n = self._qubits
        self._vector = torch.empty(1 << n, dtype=self._tdtype, device=self._tdev)
        if all_zeros:
            self._vector.zero_()
        else:
            N.call("qs_init_zero", self._vector.data_ptr(), n, self._qs_dtype, self._engine.stream)

    @property
    def _qs_dtype(self) -> int:
        return N.QS_C128 if self._precision == np.complex128 else N.QS_C64

    def run(self, circuit, state_vector=None, use_previous: bool = False) -> StateArray:
        self.initial_circuit(circuit)
        n = self._qubits
        if state_vector is not None:
            sv = self._to_device(state_vector)
            if sv.numel() != (1 << n):
                raise ValueError("The state vector should have the same qubits as the circuit.")
            self._vector = sv.clone() if isinstance(state_vector, (torch.Tensor, StateArray)) else sv
        elif not use_previous or self._vector is None or self._vector.numel() != (1 << n):
            if self._autotune and self._engine.fusion:
                self._vector = torch.empty(1 << n, dtype=self._tdtype, device=self._tdev)
                ops = [op for g in circuit.gates if not _is_trigger(g)
                       for op in lower_gate(g, n, self._legacy) if op.kind not in ("measure", "reset", "perm")]
                self._engine.autotune(self._vector, n, ops)
            self.initial_state_vector()
        self._run_gates(list(circuit.gates))
        if self._sync:
            torch.cuda.synchronize(self._tdev)
        return self.vector

    def _run_gates(self, gates: List):
        n = self._qubits
        # a circuit of plain gates seen before is not lowered again (the
        # engine then replays its planned program as well)
        key = _circuit_key(gates, n, self._legacy)
        if key is not None:
            ops = self._lowered.get(key)
            if ops is None:
                ops = [op for g in gates for op in lower_gate(g, n, self._legacy)]
                if any(op.kind in ("measure", "reset", "perm") for op in ops):
                    ops = None
                else:
                    self._lowered[key] = ops
                    while len(self._lowered) > 8:
                        self._lowered.pop(next(iter(self._lowered)))
            if ops is not None:
                self._engine.apply_ops(self._vector, n, ops)
                return
        pending: List[Op] = []
        idx = 0
        while idx < len(gates):
            g = gates[idx]
            idx += 1
            if _is_trigger(g):
                self._engine.apply_ops(self._vector, n, pending)
                pending = []
                extra, position = self.apply_trigger(g, idx)
                if extra:
                    gates[position:position] = list(extra)
                continue
            for op in lower_gate(g, n, self._legacy):
                if op.kind in ("measure", "reset", "perm"):
                    self._engine.apply_ops(self._vector, n, pending)
                    pending = []
                    self._apply_special(op)
                else:
                    pending.append(op)
        self._engine.apply_ops(self._vector, n, pending)

    def _apply_special(self, op: Op):
        n = self._qubits
        if op.kind == "measure":
            self._measure_bit(op.tbits[0])
        elif op.kind == "reset":
            p0 = self._engine.prob0(self._vector, n, op.tbits[0])
            self._engine.reset(self._vector, n, op.tbits[0], p0)
        else:
            from .permute import apply_perm
            self._vector = apply_perm(self._engine, self._vector, n, op)

    def _measure_bit(self, bit: int, u: Optional[float] = None) -> int:
        """Measure vector bit `bit` with the reference rule: outcome 1 iff u > P(0)
        (gate_function.py:1779-1815); record it on the circuit's qubit."""
        n = self._qubits
        p0 = self._engine.prob0(self._vector, n, bit)
        if u is None:
            u = float(self._rng.random())
        one = u > p0
        p = (1.0 - p0) if one else p0
        self._engine.collapse(self._vector, n, bit, int(one), 1.0 / np.sqrt(p))
        if self._circuit is not None:
            self._circuit.qubits[n - 1 - bit].measured = int(one)
        return int(one)

    # ---- reference helpers ---------------------------------------------------------------
    def get_measured_prob(self, index: int, all_measured: bool = False) -> "MeasuredProb":
        """P(vector bit `index` = 0) in FP64 (all_measured: total norm).  A
        float that also has QuICT's ``.get()`` (its GPU path returns a device
        scalar that callers read with ``.get()``)."""
        if all_measured:
            return MeasuredProb(self._engine.norm2(self._vector, self._qubits))
        return MeasuredProb(self._engine.prob0(self._vector, self._qubits, index))

    def apply_specialgate(self, index: int, type, prob: float = None):
        name = getattr(type, "name", type)
        if name == "measure":
            return self._measure_bit(index)
        if name == "reset":
            p0 = prob if prob is not None else self._engine.prob0(self._vector, self._qubits, index)
            self._engine.reset(self._vector, self._qubits, index, p0)
            return None
        raise ValueError(f"apply_specialgate: type must be measure or reset, got {name}")

    def apply_gate(self, gate):
        self._engine.apply_ops(self._vector, self._qubits, lower_gate(gate, self._qubits, self._legacy))

    def apply_multiply(self, value):
        c = complex(value)
        N.call("qs_scale", self._vector.data_ptr(), self._qubits, self._qs_dtype, c.real, c.imag,
               self._engine.stream)

    def apply_zeros(self):
        self._vector = torch.zeros_like(self._vector)

    def apply_trigger(self, op, current_idx: int = 0):
        """Measure the trigger's qubits, then return (gates, position): the
        gates its mapping selects for the measured value and the index of
        the run's gate list where they go in (statevector_simulator.py:498-523).
        That is `current_idx` (the index after the trigger), or, when the
        selected composite gate carries a checkpoint child, the mark of its
        CheckPoint in the circuit (``Circuit.find_position``, which also moves
        the marks by the child's shift).  A plain gate or None selects that
        gate alone or nothing."""
        n = self._qubits
        for q in op.targs:
            self._measure_bit(n - 1 - q)
        value = 0
        for q in op.targs:
            value = (value << 1) | int(self._circuit.qubits[q].measured)
        cg = op.mapping(value)
        if cg is None:
            return [], current_idx
        if not hasattr(cg, "gates"):  # a single gate
            return [cg], current_idx
        cp = getattr(cg, "checkpoint", None)
        position = current_idx if cp is None else self._circuit.find_position(cp)
        return list(cg.gates), position

    # ---- sampling ---------------------------------------------------------------------------
    def sample(self, shots: int = 1, uniforms=None, mode: str = "cdf", seed: Optional[int] = None,
               return_counts: bool = True):
        """Sample all qubits `shots` times without changing the state.

        mode="cdf": one uniform per shot; basis index = smallest i with
        u <= CDF[i] (FP64).  mode="sequential": n uniforms per shot, qubit 0
        first, outcome 1 iff u > P(0 | earlier outcomes) -- the reference's
        per-qubit rule (statevector_simulator.py:595-626).  Both rules give the
        same distribution.  Returns counts indexed by the big-endian integer of
        the outcomes (a list of length 2^n, as the reference does).
        """
        if self._circuit is None or self._vector is None:
            raise RuntimeError("StateVectorSimulation sample without run any circuit.")
        n = self._qubits
        m = N.QS_SAMPLE_CDF if mode == "cdf" else N.QS_SAMPLE_SEQ
        per = 1 if m == N.QS_SAMPLE_CDF else n
        if uniforms is None:
            rng = np.random.default_rng(seed) if seed is not None else self._rng
            uniforms = rng.random(shots * per)
        u = torch.as_tensor(np.asarray(uniforms, dtype=np.float64).ravel()[: shots * per])
        idx = self._engine.sample_indices(self._vector, n, u, m)
        self.last_sample_indices = idx
        if not return_counts:
            return idx
        return self._engine.counts_list(idx, 1 << n)


class MeasuredProb(float):
    """A probability read back from the device: a float with ``.get()``."""

    def get(self) -> float:
        return float(self)


# gate types whose matrix follows from the type, the qubit count and pargs
_PARAM_DETERMINED = None


def _circuit_key(gates, n: int, legacy: bool):
    """Exact key of a list of plain gates (None when it holds anything else:
    triggers, measurements, operators): per gate its type, qubits, parameters
    and precision, plus the matrix itself for custom-matrix gates."""
    global _PARAM_DETERMINED
    if _PARAM_DETERMINED is None:
        from ..core.gate import GATE_BY_NAME
        _PARAM_DETERMINED = frozenset(GATE_BY_NAME) - {"unitary", "measure", "reset", "barrier"}
    parts = [n, legacy]
    for g in gates:
        t = getattr(g, "type", None)
        name = getattr(t, "name", None)
        if name is None or name in ("measure", "reset") or _is_trigger(g):
            return None
        k = (name, tuple(g.cargs), tuple(g.targs), tuple(g.pargs), str(getattr(g, "precision", "")))
        if name not in _PARAM_DETERMINED:
            m = g.matrix
            if m is None:
                return None
            k = k + (np.asarray(m).tobytes(),)
        parts.append(k)
    return tuple(parts)


def _is_trigger(g) -> bool:
    return hasattr(g, "mapping") and hasattr(g, "targs") and not hasattr(g, "matrix_type")

"""Density-matrix simulator: CPU checks of the superoperator lowering and the
noise model, GPU parity against the reference fixtures and the FP64 oracle
(complex128 within 1e-12, complex64 within 1e-5)."""
import json

import numpy as np
import pytest

from conftest import build_circuit, golden, oracle_gates
from oracle import dm as odm
from oracle import sv as osv


def _noise_model(gates_1q, gates_2q, gamma=5e-3, p1=1e-3, p2=1e-2):
    from quict_b200.core import NoiseModel, DampingError, DepolarizingError
    amp = DampingError(amplitude_prob=gamma, phase_prob=0)
    nm = NoiseModel(basic_gates=gates_1q + gates_2q)
    nm.add_noise_for_all_qubits(amp.compose(DepolarizingError(p1, 1)), gates_1q)
    nm.add_noise_for_all_qubits(amp.tensor(amp).compose(DepolarizingError(p2, 2)), gates_2q)
    return nm


def _apply_dm_ops(rho, n, ops):
    v = rho.reshape(-1).astype(np.complex128)
    for op in ops:
        bits = list(op.cbits) + list(op.tbits)
        u = op.dense()
        if op.cbits:
            d = u.shape[0] << len(op.cbits)
            f = np.eye(d, dtype=np.complex128)
            f[-u.shape[0]:, -u.shape[0]:] = u
            u = f
        v = osv.apply_matrix(v, 2 * n, u, [2 * n - 1 - b for b in bits])
    return v.reshape(1 << n, 1 << n)


@pytest.mark.parametrize("n", [3, 4])
def test_dm_lowering_matches_reference_fixture(n):
    from quict_b200.simulation.density_matrix import lower_dm
    d = golden("dm.npz")
    gl = json.loads(str(d[f"n{n}_gates"]))
    c = build_circuit(gl, n)
    nm = _noise_model(["h", "u3", "rx"], ["rzz", "swap", "cx", "cz"])
    noisy = nm.transpile(c, accumulated_mode=True)
    ops = [op for g in noisy.gates for op in lower_dm(g, n)]
    rho = _apply_dm_ops(odm.zero_dm(n), n, ops)
    np.testing.assert_allclose(rho, d[f"n{n}_noisy"], rtol=0, atol=1e-12)
    clean = [op for g in c.gates for op in lower_dm(g, n)]
    np.testing.assert_allclose(_apply_dm_ops(odm.zero_dm(n), n, clean), d[f"n{n}_clean"], rtol=0, atol=1e-12)


def test_transpile_attaches_one_noise_gate_per_matched_gate():
    from quict_b200.core import Circuit, H, CX, Rz
    nm = _noise_model(["h"], ["cx"])
    c = Circuit(3)
    H | c(0)
    CX | c([0, 1])
    Rz(0.3) | c(2)
    t = nm.transpile(c, accumulated_mode=True)
    kinds = [getattr(g, "type", None) for g in t.gates]
    assert kinds[0] == "noise" and kinds[1] == "noise" and kinds[2].name == "rz"
    assert len(t.gates[0].noise_matrix) == 8 and len(t.gates[1].noise_matrix) == 64


def test_stacked_kraus_operators_and_superoperator():
    """The batched Kraus path (stacked operators, one product per gate, one
    GEMM per superoperator) equals the per-operator definitions; a noise gate
    whose matrices were replaced falls back to them."""
    from quict_b200.core import DampingError, DepolarizingError, H, CX
    from quict_b200.core.noise import NoiseGate
    from quict_b200.simulation.density_matrix import superop
    amp = DampingError(amplitude_prob=0.05, phase_prob=0.02)
    err = amp.tensor(amp).compose(DepolarizingError(0.03, 2))
    g = CX.matrix
    want = [k @ g for k in err.kraus]
    got = err.apply_to_gate(g)
    assert len(got) == len(want) == 144  # (3 damping operators)^2 x 16 Pauli products
    np.testing.assert_allclose(np.array(got), np.array(want), rtol=0, atol=1e-15)
    ng = NoiseGate(err.apply_to_gate_array(g), 2)
    k = np.array(want)
    ref = np.einsum("kab,kcd->acbd", k, k.conj()).reshape(16, 16)
    np.testing.assert_allclose(superop(ng.kraus_stack()), ref, rtol=0, atol=1e-15)
    np.testing.assert_allclose(superop(ng.noise_matrix), ref, rtol=0, atol=1e-15)
    with pytest.raises(ValueError):
        ng.noise_matrix[0][0, 0] = 1  # views of the shared stack are read-only
    ng.noise_matrix[0] = np.eye(4)
    assert ng.kraus_stack() is None
    # replacing an error's operators rebuilds its stack
    e1 = amp.compose(DepolarizingError(0.01, 1))
    s1 = e1.kraus_array()
    e1.operators = e1.operators[:2]
    assert e1.kraus_array().shape[0] == 2 and s1.shape[0] > 2
    np.testing.assert_allclose(e1.apply_to_gate_array(H.matrix), np.array([k @ H.matrix for k in e1.kraus]),
                               rtol=0, atol=1e-15)


def test_readout_error_is_a_confusion_row_draw():
    from quict_b200.core import ReadoutError, Circuit
    err = ReadoutError([[0.0, 1.0], [1.0, 0.0]])  # always flips
    from quict_b200.core import NoiseModel
    nm = NoiseModel()
    nm.add_readout_error(err, [0, 2])
    c = Circuit(3)
    for q, v in enumerate([0, 1, 1]):
        c.qubits[q].measured = v
    nm.apply_readout_error(c.qubits)
    assert [q.measured for q in c.qubits] == [1, 1, 0]


# ------------------------------------------------------------------ GPU parity
@pytest.mark.gpu
@pytest.mark.parametrize("n", [3, 4])
@pytest.mark.parametrize("fusion", [True, False])
def test_dm_gpu_matches_reference_fixture(cuda_ok, n, fusion):
    from quict_b200.simulation import DensityMatrixSimulator
    d = golden("dm.npz")
    gl = json.loads(str(d[f"n{n}_gates"]))
    nm = _noise_model(["h", "u3", "rx"], ["rzz", "swap", "cx", "cz"])
    sim = DensityMatrixSimulator("GPU", accumulated_mode=True, fusion=fusion)
    rho = sim.run(build_circuit(gl, n), noise_model=nm).get()
    np.testing.assert_allclose(rho, d[f"n{n}_noisy"], rtol=0, atol=1e-12)
    rho = DensityMatrixSimulator("GPU", fusion=fusion).run(build_circuit(gl, n)).get()
    np.testing.assert_allclose(rho, d[f"n{n}_clean"], rtol=0, atol=1e-12)
    sim = DensityMatrixSimulator("GPU", "single", accumulated_mode=True, fusion=fusion)
    rho = sim.run(build_circuit(gl, n), noise_model=nm).get()
    np.testing.assert_allclose(rho, d[f"n{n}_noisy"], rtol=0, atol=1e-5)


@pytest.mark.gpu
@pytest.mark.parametrize("n", [7])
def test_dm_noisy_style_vs_oracle(cuda_ok, n):
    """150-gate uniform-circuit gate set with composed damping+depolarizing per gate,
    against the Kraus-sum oracle (the 12-qubit run is checked in full against
    the superoperator oracle in test_benchmark_sizes.py)."""
    from quict_b200.core import Circuit
    from quict_b200.simulation import DensityMatrixSimulator
    size = 150 if n == 7 else 12
    c = Circuit(n)
    c.random_append(size, seed=n)
    one = ["h", "x", "rx", "ry", "rz", "u3"]
    two = ["cx", "cz", "rzz", "swap"]
    nm = _noise_model(one, two)
    rho = DensityMatrixSimulator("GPU", accumulated_mode=True).run(c, noise_model=nm).get()
    k1, k2 = odm.composed_noise_1q(5e-3, 1e-3), odm.composed_noise_2q(5e-3, 1e-2)
    ref = odm.run(oracle_gates(c), n, noise=lambda a: k1 if len(a) == 1 else k2)
    np.testing.assert_allclose(rho, ref, rtol=0, atol=1e-12)
    assert abs(np.trace(rho) - 1) < 1e-12


@pytest.mark.gpu
def test_dm_measure_and_sample(cuda_ok):
    from quict_b200.core import Circuit, H, CX, Measure
    from quict_b200.simulation import DensityMatrixSimulator
    n = 4
    c = Circuit(n)
    H | c(0)
    for q in range(n - 1):
        CX | c([q, q + 1])
    sim = DensityMatrixSimulator("GPU", seed=11)
    rho = sim.run(c).get()
    counts = sim.sample(2000, seed=5)
    assert counts[0] + counts[-1] == 2000 and counts[0] > 800 and counts[-1] > 800
    # sequential rule with explicit uniforms equals the oracle's per-qubit rule
    u = np.random.default_rng(3).random(64 * n)
    sim.sample(64, uniforms=u, mode="sequential")
    got = sim.last_sample_indices.cpu().numpy()
    probs = np.real(np.diag(rho))
    want = osv.sample_sequential_fast(np.sqrt(probs).astype(np.complex128), n, u)
    np.testing.assert_array_equal(got, want)
    # mid-circuit measurement: collapse matches the oracle projector
    c2 = Circuit(n)
    H | c2(0)
    CX | c2([0, 1])
    Measure | c2(1)
    sim2 = DensityMatrixSimulator("GPU", seed=type("U", (), {"random": staticmethod(lambda: 0.7)})())
    rho2 = sim2.run(c2).get()
    r = odm.run(oracle_gates_unitary(c2), n)
    r, b = odm.measure(r, n, 1, 0.7)
    np.testing.assert_allclose(rho2, r, atol=1e-12)
    assert c2.qubits[1].measured == b


def oracle_gates_unitary(c):
    return [(np.asarray(g.matrix, dtype=np.complex128), list(g.cargs) + list(g.targs))
            for g in c.gates if g.type.name not in ("measure",)]


@pytest.mark.gpu
def test_dm_apply_gates_and_apply_noise(cuda_ok):
    """The reference's public step methods: apply_gates (a composite / gate
    list) and apply_noise (a NoiseGate's Kraus set), against the oracle."""
    from quict_b200.core import CX, H, Rz, Circuit, DampingError, DepolarizingError
    from quict_b200.core.noise import NoiseGate
    from quict_b200.simulation import DensityMatrixSimulator
    n = 3
    c = Circuit(n)
    c.random_append(20, seed=3)
    sim = DensityMatrixSimulator("GPU")
    sim.run(c)
    rho = odm.run(oracle_gates(c), n)
    gates = [H & 0, CX & [0, 2], Rz(0.4) & 1]
    sim.apply_gates(gates)
    rho = odm.run([(np.asarray(g.matrix), list(g.cargs) + list(g.targs)) for g in gates], n, rho=rho)
    err = DampingError(amplitude_prob=0.1, phase_prob=0).compose(DepolarizingError(0.05, 1))
    ng = NoiseGate(err.apply_to_gate_array(np.eye(2)), 1)
    ng.targs = [1]
    sim.apply_noise(ng, n)
    rho = odm.apply_channel(rho, n, [np.asarray(k) for k in ng.noise_matrix], [1])
    np.testing.assert_allclose(sim.density_matrix.get(), rho, rtol=0, atol=1e-12)
    with pytest.raises(ValueError):
        sim.apply_noise(ng, n + 1)


class _NumpyEngine:
    """Applies lowered ops on a CPU tensor with the oracle (host-logic check)."""

    def apply_ops(self, vec, n, ops):
        v = vec.numpy()
        out = _apply_dm_ops(v.reshape(1 << (n // 2), 1 << (n // 2)), n // 2, ops).reshape(-1)
        v[:] = out


def test_dm_step_methods_host_logic():
    """apply_gates / apply_noise lower to the ops the oracle expects (the ops
    are applied by a numpy stand-in here; the GPU test runs the kernels)."""
    import torch
    from quict_b200.core import CX, H, Rz, DampingError, DepolarizingError
    from quict_b200.core.noise import NoiseGate
    from quict_b200.simulation import DensityMatrixSimulator
    n = 3
    sim = DensityMatrixSimulator.__new__(DensityMatrixSimulator)
    sim._qubits = n
    sim._density_matrix = torch.from_numpy(odm.zero_dm(n).copy())
    sim._engine = _NumpyEngine()
    gates = [H & 0, CX & [0, 2], Rz(0.4) & 1]
    sim.apply_gates(gates)
    rho = odm.run([(np.asarray(g.matrix), list(g.cargs) + list(g.targs)) for g in gates], n)
    err = DampingError(amplitude_prob=0.1, phase_prob=0).compose(DepolarizingError(0.05, 1))
    ng = NoiseGate(err.apply_to_gate_array(np.eye(2)), 1)
    ng.targs = [1]
    sim.apply_noise(ng, n)
    rho = odm.apply_channel(rho, n, [np.asarray(k) for k in ng.noise_matrix], [1])
    np.testing.assert_allclose(sim._density_matrix.numpy(), rho, rtol=0, atol=1e-12)
    with pytest.raises(TypeError):
        from quict_b200.core import Measure
        sim.apply_gates([Measure & 0])

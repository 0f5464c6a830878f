"""Perm gates, OpenQASM loading and UnitarySimulator."""
import numpy as np
import pytest

from conftest import build_circuit, golden, oracle_gates
from oracle import sv as osv


def test_qasm_round_trip_reproduces_reference_golden():
    from quict_b200.core.qasm import dumps, loads
    qc = golden("qasm_circuit.json")
    c = build_circuit(qc["gates"], qc["n"])
    c2 = loads(dumps(c))
    assert len(c2.gates) == len(c.gates)
    v = osv.run(oracle_gates(c2), qc["n"])
    np.testing.assert_allclose(v, golden("qasm_state.npy"), rtol=0, atol=1e-12)


def test_qasm_expressions_comments_and_measure():
    from quict_b200.core.qasm import OPENQASMInterface
    text = """OPENQASM 2.0;
    include "qelib1.inc";   // standard header
    qreg q[3]; creg c[3];
    h q[0];
    rz(pi/4) q[1];
    u3(2*pi/3, -pi/2, 0.5) q[2];
    cx q[0], q[1];
    crz(-(pi/8)) q[1], q[2];
    barrier q[0], q[1];
    measure q[2] -> c[2];
    """
    c = OPENQASMInterface.load_string(text).circuit
    names = [g.type.name for g in c.gates]
    assert names == ["h", "rz", "u3", "cx", "crz", "measure"]
    assert abs(c.gates[1].parg - np.pi / 4) < 1e-15 and abs(c.gates[4].parg + np.pi / 8) < 1e-15
    np.testing.assert_allclose(c.gates[2].pargs, [2 * np.pi / 3, -np.pi / 2, 0.5])
    with pytest.raises(ValueError):
        OPENQASMInterface.load_string("qreg q[1]; h q[0]; os.system(1) q[0];")


@pytest.mark.parametrize("seed", range(5))
def test_perm_swap_network_matches_reference_kernel(seed):
    from quict_b200.simulation.permute import perm_mapping, perm_ops
    from quict_b200.simulation.lowering import lower_gate
    from quict_b200.core import Perm
    rng = np.random.default_rng(seed)
    n = 6
    k = int(rng.integers(2, n + 1))
    args = [int(a) for a in rng.choice(n, k, replace=False)]
    pargs = [int(p) for p in rng.permutation(k)]
    g = Perm(k, pargs) & args
    (op,) = lower_gate(g, n)
    v = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
    want = osv.vector_permutation(v, n, perm_mapping(n, args, pargs))
    got = v.copy()
    for sop in perm_ops(n, op):
        got = osv.apply_matrix(got, n, sop.dense(), [n - 1 - b for b in sop.tbits])
    np.testing.assert_allclose(got, want, atol=1e-15)


@pytest.mark.gpu
def test_perm_gate_on_gpu(cuda_ok):
    from quict_b200.core import Circuit, H, Rx, CX, Perm
    from quict_b200.simulation import StateVectorSimulator
    from quict_b200.simulation.permute import perm_mapping
    n = 14
    c = Circuit(n)
    for q in range(n):
        H | c(q)
        Rx(0.1 * q + 0.2) | c(q)
    CX | c([0, 5])
    args, pargs = [1, 4, 7, 9, 13], [3, 0, 4, 1, 2]
    Perm(5, pargs) | c(args)
    v = StateVectorSimulator("GPU").run(c).get()
    pre = osv.run(oracle_gates(Circuit_prefix(c)), n)
    want = osv.vector_permutation(pre, n, perm_mapping(n, args, pargs))
    np.testing.assert_allclose(v, want, atol=1e-12)


def Circuit_prefix(c):
    from quict_b200.core import Circuit
    p = Circuit(c.width())
    p.gates = [g for g in c.gates if g.type.name != "perm"]
    return p


@pytest.mark.gpu
@pytest.mark.parametrize("precision,tol", [("double", 1e-12), ("single", 1e-5)])
def test_unitary_simulator_vs_oracle(cuda_ok, precision, tol):
    from quict_b200.simulation.unitary import UnitarySimulator
    qc = golden("qasm_circuit.json")
    c = build_circuit(qc["gates"], qc["n"])
    sim = UnitarySimulator("GPU", precision)
    v = sim.run(c).get()
    np.testing.assert_allclose(v, golden("qasm_state.npy"), rtol=0, atol=tol * 10)
    n = 7
    from quict_b200.core import Circuit
    c2 = Circuit(n)
    c2.random_append(60, seed=3)
    u = sim.get_unitary_matrix(c2).get()
    eye = np.eye(1 << n, dtype=np.complex128)
    ref = np.stack([osv.run(oracle_gates(c2), n, vec=eye[:, j]) for j in range(1 << n)], axis=1)
    np.testing.assert_allclose(u, ref, atol=tol * 10)
    counts = sim.sample(100, seed=1)
    assert sum(counts) == 100


@pytest.mark.gpu
def test_unitary_initial_vector_state(cuda_ok):
    from quict_b200.core import Circuit
    from quict_b200.simulation.unitary import UnitarySimulator
    c = Circuit(4)
    c.random_append(20, seed=4)
    sim = UnitarySimulator("GPU")
    sim.run(c)
    sim.initial_vector_state()
    v = sim.vector.get()
    assert v.shape == (16,) and v[0] == 1 and np.count_nonzero(v) == 1


def test_circuit_qasm_method_round_trips():
    from quict_b200.core import Circuit
    from quict_b200.core.qasm import loads
    c = Circuit(4)
    c.random_append(30, seed=8)
    c2 = loads(c.qasm())
    assert [g.type.name for g in c2.gates] == [g.type.name for g in c.gates]
    assert [list(g.cargs) + list(g.targs) for g in c2.gates] == [list(g.cargs) + list(g.targs) for g in c.gates]
    np.testing.assert_allclose(osv.run(oracle_gates(c2), 4), osv.run(oracle_gates(c), 4), atol=1e-12)

"""Pin the oracle (and the product's gate matrices) to fixtures produced by the
reference itself (tests/golden/make_golden.py).  CPU only."""
import json

import numpy as np
import pytest

from conftest import build_circuit, golden, oracle_gates
from oracle import dm as odm
from oracle import sv as osv


def test_gate_matrices_match_reference():
    from quict_b200.core import GATE_BY_NAME
    ref = golden("gates.json")
    assert len(ref) >= 40
    for nm, r in ref.items():
        g = GATE_BY_NAME[nm]
        if r["params"]:
            g = g(*r["params"])
        m = np.array(r["re"]) + 1j * np.array(r["im"])
        assert g.controls == r["controls"] and g.targets == r["targets"], nm
        assert g.matrix_type.name == r["matrix_type"], nm
        np.testing.assert_allclose(g.matrix, m, rtol=0, atol=1e-15, err_msg=nm)


def test_oracle_reproduces_reference_golden_vector():
    qc = golden("qasm_circuit.json")
    n = qc["n"]
    c = build_circuit(qc["gates"], n)
    v = osv.run(oracle_gates(c), n)
    np.testing.assert_allclose(v, golden("qasm_state.npy"), rtol=0, atol=1e-12)


@pytest.mark.parametrize("n", [5, 8, 11])
def test_oracle_random_circuits(n):
    d = golden("random_sv.npz")
    gl = json.loads(str(d[f"n{n}_gates"]))
    c = build_circuit(gl, n)
    v = osv.run(oracle_gates(c), n)
    np.testing.assert_allclose(v, d[f"n{n}_double"], rtol=0, atol=1e-12)
    np.testing.assert_allclose(v, d[f"n{n}_single"], rtol=0, atol=1e-5)


def test_oracle_extended_gate_set_matches_reference():
    d = golden("ext_sv.npz")
    # circuit a: reference SV path (reversed uncontrolled 2q dense order)
    ga = json.loads(str(d["a_gates"]))
    c = build_circuit(ga, 6)
    v = osv.run(oracle_gates(c), 6, legacy_2q_order=True, n_controls=[g.controls for g in c.gates])
    np.testing.assert_allclose(v, d["a_sv"], rtol=0, atol=1e-12)
    # circuit b: reference UnitarySimulator (big-endian)
    gb = json.loads(str(d["b_gates"]))
    c = build_circuit(gb, 6)
    np.testing.assert_allclose(osv.run(oracle_gates(c), 6), d["b_unitary"], rtol=0, atol=1e-12)


def test_oracle_haar_both_conventions():
    d = golden("haar_sv.npz")
    gl = json.loads(str(d["gates"]))
    c = build_circuit(gl, 5)
    g = oracle_gates(c)
    nctl = [x.controls for x in c.gates]
    np.testing.assert_allclose(osv.run(g, 5), d["unitary_reference"], rtol=0, atol=1e-12)
    np.testing.assert_allclose(osv.run(g, 5, legacy_2q_order=True, n_controls=nctl), d["sv_reference"],
                               rtol=0, atol=1e-12)


@pytest.mark.parametrize("n", [4, 6])
def test_oracle_sampling_matches_reference_counts(n):
    d = golden("sample.npz")
    sv = d[f"n{n}_state"]
    u = d[f"n{n}_uniforms"]
    idx = osv.sample_sequential(sv, n, u)
    counts = np.bincount(idx, minlength=1 << n)
    np.testing.assert_array_equal(counts, d[f"n{n}_counts"])
    # the prefix-sum form gives the same indices
    np.testing.assert_array_equal(osv.sample_sequential_fast(sv, n, u), idx)


def test_cdf_rule_equals_sequential_rule_on_derived_uniforms():
    rng = np.random.default_rng(5)
    n = 7
    v = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
    v /= np.linalg.norm(v)
    u = rng.random(400)
    # derive the per-qubit uniform stream from one uniform per shot
    p = np.abs(v) ** 2
    cs = np.concatenate([[0.0], np.cumsum(p)])
    seq_u = np.empty((u.size, n))
    for s, x in enumerate(u):
        lo, size = 0, 1 << n
        for q in range(n):
            half = size // 2
            pl = (cs[lo + half] - cs[lo]) / (cs[lo + size] - cs[lo])
            seq_u[s, q] = x
            if x > pl:
                x = (x - pl) / (1 - pl)
                lo += half
            else:
                x = x / pl
            size = half
    a = osv.sample_cdf(v, u)
    b = osv.sample_sequential_fast(v, n, seq_u.ravel())
    ties = osv.near_ties(v, u, 1e-9)
    assert np.all((a == b) | ties)


def test_oracle_midcircuit_measure_reset():
    d = golden("midmeasure.npz")
    gl = json.loads(str(d["gates"]))
    n = 5
    u = list(d["uniforms"])
    v = osv.zero_state(n)
    from quict_b200.core import GATE_BY_NAME
    measured = [-1] * n
    for nm, args, params in gl:
        if nm == "measure":
            v, b = osv.measure(v, n, args[0], u.pop(0))
            measured[args[0]] = b
        elif nm == "reset":
            v = osv.reset(v, n, args[0])
        else:
            g = GATE_BY_NAME[nm](*params) if params else GATE_BY_NAME[nm]
            v = osv.apply_matrix(v, n, g.matrix, args)
    np.testing.assert_allclose(v, d["state"], rtol=0, atol=1e-12)
    assert [m for m in measured if m >= 0] == [int(x) for x in d["measured"] if x >= 0]


@pytest.mark.parametrize("n", [3, 4])
def test_dm_oracle_matches_reference(n):
    d = golden("dm.npz")
    gl = json.loads(str(d[f"n{n}_gates"]))
    c = build_circuit(gl, n)
    rho = odm.run(oracle_gates(c), n)
    np.testing.assert_allclose(rho, d[f"n{n}_clean"], rtol=0, atol=1e-12)
    k1, k2 = odm.composed_noise_1q(5e-3, 1e-3), odm.composed_noise_2q(5e-3, 1e-2)
    np.testing.assert_allclose(np.array(k1), d[f"n{n}_kraus1"], rtol=0, atol=1e-14)
    np.testing.assert_allclose(np.array(k2), d[f"n{n}_kraus2"], rtol=0, atol=1e-14)
    noisy = odm.run(oracle_gates(c), n, noise=lambda args: k1 if len(args) == 1 else k2)
    np.testing.assert_allclose(noisy, d[f"n{n}_noisy"], rtol=0, atol=1e-12)


@pytest.mark.parametrize("n", [5, 8, 11])
def test_cpu_port_reproduces_reference_states(n):
    """oracle/ref_port.py (the timed CPU baseline) against the reference CPU
    simulator's own states."""
    from oracle import ref_port
    from quict_b200.simulation.lowering import lower_circuit
    d = golden("random_sv.npz")
    gl = json.loads(str(d[f"n{n}_gates"]))
    v = osv.zero_state(n)
    ref_port.run(v, ref_port.prepare(lower_circuit(build_circuit(gl, n).gates, n), np.complex128))
    np.testing.assert_allclose(v, d[f"n{n}_double"], rtol=0, atol=1e-12)


def test_cpu_port_on_the_benchmark_circuit_shape():
    """The port on a 12-qubit spread circuit (Haar 2q unitaries, low and high
    qubits) against the FP64 oracle, on all amplitudes."""
    from oracle import ref_port
    from quict_b200.simulation.lowering import lower_circuit
    from quict_b200.workloads import spread_circuit
    n = 12
    c = spread_circuit(n, 300, seed=3)
    v = osv.zero_state(n)
    ref_port.run(v, ref_port.prepare(lower_circuit(c.gates, n), np.complex128))
    np.testing.assert_allclose(v, osv.run(oracle_gates(c), n), rtol=0, atol=1e-12)

"""State-vector parity on the GPU (through libqsim's C-ABI) against the
reference's golden fixtures and the FP64 oracle.

Tolerances (stated by the parity contract): complex128 amplitudes within
1e-12, complex64 within 1e-5; sampled indices bit-exact given the same
uniforms except draws within 1e-12 of a CDF boundary."""
import json

import numpy as np
import pytest

from conftest import build_circuit, golden, oracle_gates
from oracle import sv as osv

pytestmark = pytest.mark.gpu

TOL = {"double": 1e-12, "single": 1e-5}


class ListRNG:
    """Feeds recorded uniforms to the simulator's measurement RNG."""

    def __init__(self, u):
        self.u = list(u)

    def random(self):
        return self.u.pop(0)


def sim(precision="double", **kw):
    from quict_b200.simulation import StateVectorSimulator
    return StateVectorSimulator("GPU", precision, **kw)


@pytest.mark.parametrize("precision", ["double", "single"])
@pytest.mark.parametrize("fusion", [True, False])
def test_reference_golden_vector(cuda_ok, precision, fusion):
    qc = golden("qasm_circuit.json")
    c = build_circuit(qc["gates"], qc["n"])
    sv = sim(precision, fusion=fusion).run(c).get()
    ref = golden("qasm_state.npy")
    np.testing.assert_allclose(sv, ref, rtol=0, atol=TOL[precision])


@pytest.mark.parametrize("n", [5, 8, 11])
@pytest.mark.parametrize("fusion", [True, False])
def test_random_uniform_circuits(cuda_ok, n, fusion):
    d = golden("random_sv.npz")
    gl = json.loads(str(d[f"n{n}_gates"]))
    v = sim("double", fusion=fusion).run(build_circuit(gl, n)).get()
    np.testing.assert_allclose(v, d[f"n{n}_double"], rtol=0, atol=1e-12)
    v = sim("single", fusion=fusion).run(build_circuit(gl, n, "single")).get()
    np.testing.assert_allclose(v, d[f"n{n}_single"], rtol=0, atol=1e-5)


@pytest.mark.parametrize("fusion", [True, False])
def test_extended_gate_set(cuda_ok, fusion):
    d = golden("ext_sv.npz")
    ga = json.loads(str(d["a_gates"]))
    v = sim(fusion=fusion, legacy_2q_order=True).run(build_circuit(ga, 6)).get()
    np.testing.assert_allclose(v, d["a_sv"], rtol=0, atol=1e-12)
    gb = json.loads(str(d["b_gates"]))
    v = sim(fusion=fusion).run(build_circuit(gb, 6)).get()
    np.testing.assert_allclose(v, d["b_unitary"], rtol=0, atol=1e-12)


@pytest.mark.parametrize("fusion", [True, False])
def test_haar_2q_both_orders(cuda_ok, fusion):
    d = golden("haar_sv.npz")
    gl = json.loads(str(d["gates"]))
    v = sim(fusion=fusion).run(build_circuit(gl, 5)).get()
    np.testing.assert_allclose(v, d["unitary_reference"], rtol=0, atol=1e-12)
    v = sim(fusion=fusion, legacy_2q_order=True).run(build_circuit(gl, 5)).get()
    np.testing.assert_allclose(v, d["sv_reference"], rtol=0, atol=1e-12)


def _every_placement_circuit(n, seed):
    """Every gate family on targets/controls spread over low (<5) and high bits."""
    from quict_b200.core import GATE_BY_NAME
    rng = np.random.default_rng(seed)
    names = ["h", "x", "y", "z", "s", "t", "rx", "ry", "rz", "u3", "u1", "sx", "cx", "cy", "cz", "ch", "crz",
             "cu1", "cu3", "rzz", "rxx", "ryy", "rzx", "fsim", "swap", "iswap", "sqiswap", "ccx", "ccz", "ccrz",
             "cswap"]
    gl = [["h", [q], []] for q in range(n)]
    for nm in names:
        g = GATE_BY_NAME[nm]
        k = g.controls + g.targets
        for _ in range(3):
            args = [int(a) for a in rng.choice(n, k, replace=False)]
            gl.append([nm, args, [float(x) for x in rng.uniform(0, 2 * np.pi, g.params)]])
    # 3-, 4- and 5-qubit dense unitaries (fused up to 4, per-gate kernel beyond)
    for k in (3, 4, 5):
        z = rng.normal(size=(1 << k, 1 << k)) + 1j * rng.normal(size=(1 << k, 1 << k))
        q, _ = np.linalg.qr(z)
        args = [int(a) for a in rng.choice(n, k, replace=False)]
        gl.append(["unitary", args, [[x.real, x.imag] for x in q.ravel()]])
    return gl


@pytest.mark.parametrize("n", [6, 9, 14, 17])
@pytest.mark.parametrize("tile", [(None, None), (8, 3), (6, 0), (10, 5), (11, 5)])
def test_every_gate_every_placement_vs_oracle(cuda_ok, n, tile):
    gl = _every_placement_circuit(n, seed=n)
    c = build_circuit(gl, n)
    ref = osv.run(oracle_gates(c), n)
    for fusion in (True, False):
        v = sim(fusion=fusion, tile_bits=tile[0], low_bits=tile[1]).run(build_circuit(gl, n)).get()
        np.testing.assert_allclose(v, ref, rtol=0, atol=1e-12)
        # complex64 single-gate kernels move two adjacent amplitudes per 128-bit access
        v = sim("single", fusion=fusion, tile_bits=tile[0], low_bits=tile[1]).run(build_circuit(gl, n, "single")).get()
        np.testing.assert_allclose(v, ref, rtol=0, atol=1e-5)


def test_uniform_20q_200_gates(cuda_ok):
    from quict_b200.core import Circuit
    c = Circuit(20)
    c.random_append(200, seed=2024)
    ref = osv.run(oracle_gates(c), 20)
    for fusion in (True, False):
        v = sim(fusion=fusion).run(c).get()
        np.testing.assert_allclose(v, ref, rtol=0, atol=1e-12)


@pytest.mark.parametrize("n", [4, 6])
def test_sampling_bit_exact_reference_counts(cuda_ok, n):
    d = golden("sample.npz")
    gl = json.loads(str(d[f"n{n}_gates"]))
    s = sim()
    s.run(build_circuit(gl, n))
    counts = s.sample(len(d[f"n{n}_uniforms"]) // n, uniforms=d[f"n{n}_uniforms"], mode="sequential")
    np.testing.assert_array_equal(np.asarray(counts), d[f"n{n}_counts"])


@pytest.mark.parametrize("n", [3, 12, 20])
@pytest.mark.parametrize("precision", ["double", "single"])
def test_sampling_cdf_and_sequential_vs_oracle(cuda_ok, n, precision):
    from quict_b200.core import Circuit
    c = Circuit(n)
    c.random_append(8 * n, seed=n)
    s = sim(precision)
    v = s.run(build_circuit([[g.type.name, g.cargs + g.targs, g.pargs] for g in c.gates], n, precision)).get()
    rng = np.random.default_rng(99)
    shots = 8192
    u = rng.random(shots)
    s.sample(shots, uniforms=u, mode="cdf")
    got = s.last_sample_indices.cpu().numpy()
    v64 = v.astype(np.complex128)
    want = osv.sample_cdf(v64, u)
    ties = osv.near_ties(v64, u, 1e-12)
    assert np.all((got == want) | ties), np.flatnonzero((got != want) & ~ties)[:10]
    us = rng.random(512 * n)
    s.sample(512, uniforms=us, mode="sequential")
    got = s.last_sample_indices.cpu().numpy()
    want = osv.sample_sequential_fast(v64, n, us)
    assert np.mean(got == want) > 0.999


def test_sample_does_not_change_state_and_counts_sum(cuda_ok):
    from quict_b200.core import Circuit, H, CX
    c = Circuit(4)
    H | c(0)
    for q in range(3):
        CX | c([q, q + 1])
    s = sim(seed=3)
    v0 = s.run(c).get()
    counts = s.sample(1000)
    assert counts[0] + counts[-1] == 1000
    np.testing.assert_array_equal(s.vector.get(), v0)


def test_midcircuit_measure_reset_with_reference_uniforms(cuda_ok):
    d = golden("midmeasure.npz")
    gl = json.loads(str(d["gates"]))
    n = 5
    c = build_circuit(gl, n)
    s = sim(seed=ListRNG(d["uniforms"]))
    v = s.run(c).get()
    np.testing.assert_allclose(v, d["state"], rtol=0, atol=1e-12)
    got = [c.qubits[q].measured if c.qubits[q].measured is not None else -1 for q in range(n)]
    assert got == [int(x) for x in d["measured"]]


def test_norm_conserved_and_fused_equals_unfused_24q(cuda_ok):
    import torch
    from quict_b200.core import Circuit
    c = Circuit(24)
    c.random_append(300, seed=7)
    a = sim(fusion=True)
    b = sim(fusion=False)
    va = a.run(c).tensor
    vb = b.run(c).tensor
    assert torch.max(torch.abs(va - vb)).item() < 1e-12
    assert abs(a.get_measured_prob(0, all_measured=True) - 1.0) < 1e-12


def test_state_vector_argument_and_use_previous(cuda_ok):
    from quict_b200.core import Circuit, H, Rx
    rng = np.random.default_rng(1)
    v0 = rng.normal(size=64) + 1j * rng.normal(size=64)
    v0 /= np.linalg.norm(v0)
    c = Circuit(6)
    H | c(2)
    Rx(0.3) | c(5)
    s = sim()
    v = s.run(c, state_vector=v0).get()
    ref = osv.run(oracle_gates(c), 6, vec=v0)
    np.testing.assert_allclose(v, ref, atol=1e-12)
    v2 = s.run(c, use_previous=True).get()
    np.testing.assert_allclose(v2, osv.run(oracle_gates(c), 6, vec=ref), atol=1e-12)


def test_errors_are_raised_not_silently_ignored(cuda_ok):
    from quict_b200 import _native as N
    from quict_b200.simulation.engine import Engine
    import torch
    v = torch.zeros(8, dtype=torch.complex128, device="cuda")
    with pytest.raises(N.QsimError):
        N.call("qs_apply_1q", v.data_ptr(), 3, N.QS_C128, 5, 0, N.QS_K_DENSE, N.mat_ptr(np.eye(2))[1], None)


@pytest.mark.parametrize("n", [1, 2])
@pytest.mark.parametrize("precision", ["double", "single"])
def test_smallest_and_empty_circuits(cuda_ok, n, precision):
    """1- and 2-qubit circuits from every fixed-size gate type that fits, fused
    and gate by gate, against the oracle; an empty circuit leaves |0...0>;
    sampling and P(0) on the smallest vectors."""
    from quict_b200.core import Circuit, GATE_BY_NAME
    from quict_b200.core.gate import GateType
    types = [GateType[nm] for nm, g in GATE_BY_NAME.items()
             if nm not in ("measure", "reset", "barrier", "id", "unitary", "qft", "iqft", "perm", "perm_fx")
             and g.controls + g.targets <= n]
    c = Circuit(n)
    c.random_append(40, typelist=types, seed=n)
    ref = osv.run(oracle_gates(c), n)
    for fusion in (True, False):
        s = sim(precision, fusion=fusion)
        v = s.run(build_circuit([[g.type.name, g.cargs + g.targs, g.pargs] for g in c.gates], n, precision)).get()
        np.testing.assert_allclose(v, ref, rtol=0, atol=TOL[precision])
        u = np.random.default_rng(5).random(256)
        s.sample(256, uniforms=u, mode="cdf")
        got = s.last_sample_indices.cpu().numpy()
        ties = osv.near_ties(ref, u, 1e-5)
        assert np.all((got == osv.sample_cdf(ref, u)) | ties)
        p0 = s.get_measured_prob(0)
        assert abs(p0 - np.sum(np.abs(ref[0::2]) ** 2)) < 10 * TOL[precision]  # vector bit 0
        e = sim(precision, fusion=fusion).run(Circuit(n)).get()
        want = np.zeros(1 << n)
        want[0] = 1
        np.testing.assert_array_equal(e, want)


def test_sample_counts_list_sparse_and_dense(cuda_ok):
    """Counts come back as a list of length 2^n (as the reference returns), the
    same whether few bins are hit (only nonzero bins are copied back) or many."""
    from quict_b200.core import Circuit
    from quict_b200.simulation import DensityMatrixSimulator
    c = Circuit(12)
    c.random_append(60, seed=12)
    s = sim()
    s.run(c)
    for shots in (300, 20000):  # 4096 bins: fewer and more than 4 shots per bin
        counts = s.sample(shots, seed=shots)
        idx = s.last_sample_indices.cpu().numpy()
        assert isinstance(counts, list) and len(counts) == 4096 and sum(counts) == shots
        assert counts == np.bincount(idx, minlength=4096).tolist()
    c6 = Circuit(6)
    c6.random_append(30, seed=6)
    dm = DensityMatrixSimulator("GPU")
    dm.run(c6)
    counts = dm.sample(10, seed=1)
    idx = dm.last_sample_indices.cpu().numpy()
    assert isinstance(counts, list) and counts == np.bincount(idx, minlength=64).tolist()


@pytest.mark.parametrize("precision", ["double", "single"])
def test_cdf_sampling_of_a_subnormalised_state_never_picks_zero_mass(cuda_ok, precision):
    """A state whose norm has drifted below 1 (here scaled to 1 - 1e-4) and
    whose last amplitudes are 0: uniforms near 1 must land on the last index
    of nonzero probability, never past it (the CDF rule scales u by the total
    mass), through the workspace and the allocation-free entry points."""
    import ctypes as C
    import torch
    from quict_b200 import _native as N
    n = 12
    rng = np.random.default_rng(21)
    v = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
    v[-3:] = 0  # indices 2^n-3 .. 2^n-1 have probability 0
    v /= np.linalg.norm(v)
    v *= np.sqrt(1 - 1e-4)
    npdt = np.complex128 if precision == "double" else np.complex64
    from quict_b200.core import Circuit
    s = sim(precision)
    s.run(Circuit(n))  # sets the width; the vector is replaced next
    s.vector = v.astype(npdt)
    u = np.concatenate([1 - np.logspace(-16, -3, 200), rng.random(800)])
    s.sample(u.size, uniforms=u, mode="cdf")
    got = s.last_sample_indices.cpu().numpy()
    assert got.max() <= (1 << n) - 4
    vd = v.astype(npdt).astype(np.complex128)
    ties = osv.near_ties(vd, u, 1e-12 if precision == "double" else 1e-6)
    assert np.all((got == osv.sample_cdf(vd, u)) | ties)
    out = torch.empty(u.size, dtype=torch.int64, device="cuda")
    ud = torch.from_numpy(u).cuda()
    N.call("qs_sample_noalloc", C.c_void_p(s._vector.data_ptr()), n, s._qs_dtype, N.QS_SRC_SV,
           C.c_void_p(ud.data_ptr()), u.size, N.QS_SAMPLE_CDF, C.c_void_p(out.data_ptr()), None)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(out.cpu().numpy(), got)

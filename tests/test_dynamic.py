"""PermFx, QFT / IQFT, Trigger and CheckPoint against fixtures made by running
the reference (tests/golden/make_golden.py, dynamic.npz).

CPU tests pin the gate definitions, the circuit-building rules of CheckPoint
and the oracle; GPU tests run the simulator through libqsim.  The reference's
CPU state-vector path applies uncontrolled multi-qubit dense matrices with
their arguments reversed (cpu_calculator.py:139-186), PermFx and QFT among
them, so the fixtures are compared with ``legacy_2q_order=True`` and the
big-endian result with the oracle."""
import numpy as np
import pytest

from conftest import golden
from oracle import sv as osv


class ListRNG:
    """Feeds recorded uniforms to the simulator's measurement RNG."""

    def __init__(self, u):
        self.u = list(u)

    def random(self):
        return self.u.pop(0)


def _permfx_circuit(d, n):
    from quict_b200.core import Circuit, H, PermFx, Ry, Rz
    width = int(d[f"permfx{n}_width"])
    pre = d[f"permfx{n}_pre"]
    c = Circuit(width)
    for q in range(width):
        H | c(q)
        Ry(float(pre[q])) | c(q)
    PermFx(n, [int(x) for x in d[f"permfx{n}_ones"]]) | c([int(x) for x in d[f"permfx{n}_args"]])
    Rz(0.4) | c(0)
    return c


def _qft_circuit(d, k):
    from quict_b200.core import CX, Circuit, IQFT, QFT, Ry, Rz
    width = k + 2
    args = [int(x) for x in d[f"qft{k}_args"]]
    c = Circuit(width)
    for q in range(width):
        Ry(float(0.3 + 0.2 * q)) | c(q)
    QFT(k) | c(args)
    Rz(0.7) | c(width - 1)
    CX | c([k - 1, width - 1])
    IQFT(k) | c(args)
    return c


def _trigger_plain():
    from quict_b200.core import CX, Circuit, CompositeGate, H, Rx, Ry, Trigger, X
    c = Circuit(4)
    H | c(0)
    Ry(1.1) | c(1)
    cg0 = CompositeGate()
    X | cg0(2)
    cg1 = CompositeGate()
    CX | cg1([0, 1])
    CX | cg1([1, 2])
    CX | cg1([2, 3])
    Trigger(1, [cg0, cg1]) | c(0)
    Rx(0.3) | c(3)
    CX | c([3, 1])
    return c


def _trigger_checkpoint():
    from quict_b200.core import CX, CheckPoint, Circuit, CompositeGate, H, Rx, Ry, Rz, Swap, Trigger, X, Y
    c = Circuit(5)
    H | c(0)
    H | c(1)
    Ry(0.8) | c(2)
    cp = CheckPoint()
    cgs = []
    for v in range(4):
        cg = CompositeGate()
        if v & 1:
            X | cg(3)
        if v & 2:
            Y | cg(4)
        Ry(0.2 + 0.3 * v) | cg(2)
        Swap | cg([2, 4])
        cp.get_child(len(cg.gates)) | cg
        cgs.append(cg)
    Trigger(2, cgs) | c([0, 1])
    Rx(0.5) | c(3)
    CX | c([2, 3])
    cp | c
    Rz(0.9) | c(4)
    CX | c([3, 4])
    Rx(0.25) | c(2)
    return c


# ------------------------------------------------------------------ CPU
@pytest.mark.parametrize("n", [1, 2, 3, 4])
def test_permfx_gate_matches_reference(n):
    d = golden("dynamic.npz")
    c = _permfx_circuit(d, n)
    g = next(g for g in c.gates if g.type.name == "perm_fx")
    assert g.targets == n + 1 and g.params == 1 << (n + 1)
    np.testing.assert_array_equal(g.pargs, d[f"permfx{n}_pargs"])
    m = g.matrix
    assert np.array_equal(m @ m.conj().T, np.eye(1 << (n + 1)))
    # the oracle with the reference's reversed-argument rule reproduces its SV
    gates = [(np.asarray(x.matrix, dtype=np.complex128), list(x.cargs) + list(x.targs)) for x in c.gates]
    v = osv.run(gates, c.width(), legacy_2q_order=True, n_controls=[x.controls for x in c.gates])
    np.testing.assert_allclose(v, d[f"permfx{n}_state"], rtol=0, atol=1e-12)


@pytest.mark.parametrize("k", [2, 3, 4, 5])
def test_qft_iqft_matrices_and_oracle_match_reference(k):
    from quict_b200.core import IQFT, QFT
    d = golden("dynamic.npz")
    np.testing.assert_allclose(QFT(k).matrix, d[f"qft{k}_matrix"], rtol=0, atol=1e-12)
    np.testing.assert_allclose(IQFT(k).matrix, d[f"iqft{k}_matrix"], rtol=0, atol=1e-12)
    c = _qft_circuit(d, k)
    gates = [(np.asarray(x.matrix, dtype=np.complex128), list(x.cargs) + list(x.targs)) for x in c.gates]
    v = osv.run(gates, c.width(), legacy_2q_order=True, n_controls=[x.controls for x in c.gates])
    np.testing.assert_allclose(v, d[f"qft{k}_state"], rtol=0, atol=1e-12)


def test_checkpoint_marks_and_shifts():
    """The reference's operator_unit_test.test_checkpoint rules with single
    gates: a CheckPoint marks the circuit's end when added; a composite gate
    holding its child goes in at the mark, which then moves by the child's
    shift (circuit.py:297-360)."""
    from quict_b200.core import CheckPoint, Circuit, CompositeGate, H, X, Y, Z
    cir = Circuit(5)
    for q in range(5):
        H | cir(q)
    first = cir.size()
    cp = CheckPoint()
    child = cp.get_child(5)
    cp | cir
    assert cp.position == first
    for q in range(5):
        Z | cir(q)
    cg = CompositeGate()
    X | cg(0)
    X | cg(1)
    cg1 = CompositeGate()
    Y | cg1(0)
    Y | cg1(1)
    child | cg
    child | cg1
    cg | cir
    cg1 | cir
    names = [g.type.name for g in cir.gates]
    assert names[first:first + 2] == ["x", "x"]
    assert names[first + 5:first + 7] == ["y", "y"]
    assert cir.size() == 14 and cp.position == first + 10
    # a composite gate without a checkpoint goes at the end, mapped by circuit(qubits)
    cg2 = CompositeGate()
    X | cg2(0)
    cg2 | cir([3])
    assert cir.gates[-1].type.name == "x" and cir.gates[-1].targs == [3]


def test_trigger_mapping_forms():
    from quict_b200.core import CompositeGate, Trigger, X
    cg = CompositeGate()
    X | cg(0)
    t = Trigger(1, {0: None, 1: cg})
    assert t.mapping(1) is cg and t.mapping(0) is None
    t = Trigger(2, lambda v: cg if v == 3 else None)
    assert t.mapping(3) is cg and t.mapping(1) is None
    with pytest.raises(ValueError):
        t.mapping(4)
    with pytest.raises(TypeError):
        Trigger(1, [1, 2])


# ------------------------------------------------------------------ GPU
@pytest.mark.gpu
@pytest.mark.parametrize("n", [1, 2, 3, 4])
@pytest.mark.parametrize("fusion", [True, False])
def test_permfx_on_the_gpu(cuda_ok, n, fusion):
    from quict_b200.simulation import StateVectorSimulator
    d = golden("dynamic.npz")
    c = _permfx_circuit(d, n)
    v = StateVectorSimulator("GPU", fusion=fusion, legacy_2q_order=True).run(c).get()
    np.testing.assert_allclose(v, d[f"permfx{n}_state"], rtol=0, atol=1e-12)
    c = _permfx_circuit(d, n)
    gates = [(np.asarray(x.matrix, dtype=np.complex128), list(x.cargs) + list(x.targs)) for x in c.gates]
    want = osv.run(gates, c.width())
    v = StateVectorSimulator("GPU", fusion=fusion).run(c).get()
    np.testing.assert_allclose(v, want, rtol=0, atol=1e-12)
    v = StateVectorSimulator("GPU", "single", fusion=fusion).run(_permfx_circuit(d, n)).get()
    np.testing.assert_allclose(v, want, rtol=0, atol=1e-5)


@pytest.mark.gpu
@pytest.mark.parametrize("k", [2, 3, 4, 5])
@pytest.mark.parametrize("fusion", [True, False])
def test_qft_iqft_on_the_gpu(cuda_ok, k, fusion):
    from quict_b200.core import Circuit, IQFT, QFT, Ry
    from quict_b200.simulation import StateVectorSimulator
    d = golden("dynamic.npz")
    v = StateVectorSimulator("GPU", fusion=fusion, legacy_2q_order=True).run(_qft_circuit(d, k)).get()
    np.testing.assert_allclose(v, d[f"qft{k}_state"], rtol=0, atol=1e-12)
    # big-endian QFT on scattered qubits of a larger register, and QFT . IQFT = I
    n = 12
    rng = np.random.default_rng(k)
    args = [int(x) for x in rng.choice(n, k, replace=False)]
    c = Circuit(n)
    for q in range(n):
        Ry(float(rng.uniform(0, 2 * np.pi))) | c(q)
    QFT(k) | c(args)
    gates = [(np.asarray(x.matrix, dtype=np.complex128), list(x.cargs) + list(x.targs)) for x in c.gates]
    want = osv.run(gates, n)
    v = StateVectorSimulator("GPU", fusion=fusion).run(c).get()
    np.testing.assert_allclose(v, want, rtol=0, atol=1e-12)
    IQFT(k) | c(args)
    v = StateVectorSimulator("GPU", fusion=fusion).run(c).get()
    np.testing.assert_allclose(v, osv.run(gates[:n], n), rtol=0, atol=1e-12)


@pytest.mark.gpu
@pytest.mark.parametrize("seed", [701, 702, 703, 704])
def test_trigger_without_checkpoint_matches_reference(cuda_ok, seed):
    from quict_b200.simulation import StateVectorSimulator
    d = golden("dynamic.npz")
    c = _trigger_plain()
    s = StateVectorSimulator("GPU", seed=ListRNG(d[f"trig_plain_{seed}_uniforms"]))
    v = s.run(c).get()
    np.testing.assert_allclose(v, d[f"trig_plain_{seed}_state"], rtol=0, atol=1e-12)
    got = [-1 if q.measured is None else int(q.measured) for q in c.qubits]
    assert got == [int(x) for x in d[f"trig_plain_{seed}_measured"]]


@pytest.mark.gpu
@pytest.mark.parametrize("seed", [711, 712, 713, 714, 715, 716])
@pytest.mark.parametrize("fusion", [True, False])
def test_trigger_with_checkpoint_matches_reference(cuda_ok, seed, fusion):
    from quict_b200.simulation import StateVectorSimulator
    d = golden("dynamic.npz")
    c = _trigger_checkpoint()
    s = StateVectorSimulator("GPU", fusion=fusion, seed=ListRNG(d[f"trig_cp_{seed}_uniforms"]))
    v = s.run(c).get()
    np.testing.assert_allclose(v, d[f"trig_cp_{seed}_state"], rtol=0, atol=1e-12)
    got = [-1 if q.measured is None else int(q.measured) for q in c.qubits]
    assert got == [int(x) for x in d[f"trig_cp_{seed}_measured"]]

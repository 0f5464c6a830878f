"""``Simulator``: QuICT's one-call front end over the GPU simulators
(QuICT/simulation/simulator.py:43-151, utils/result.py:5-110)."""
import numpy as np
import pytest

from conftest import oracle_gates
from oracle import sv as osv


def test_argument_checks_before_any_device():
    from quict_b200.simulation import Simulator, SimulatorOptionsUnmatchedError
    with pytest.raises(ValueError):
        Simulator("TPU")
    with pytest.raises(ValueError):
        Simulator("CPU")  # quict_b200 has no CPU path
    with pytest.raises(ValueError):
        Simulator("GPU", backend="tensor_network")
    with pytest.raises(ValueError):
        Simulator("GPU", precision="half")
    with pytest.raises(SimulatorOptionsUnmatchedError):
        Simulator("GPU", backend="unitary", gpu_device_id=0)
    with pytest.raises(SimulatorOptionsUnmatchedError):
        Simulator("GPU", backend="density_matrix", matrix_aggregation=True)


def test_result_record_keys_every_basis_index():
    from quict_b200.simulation import Result
    r = Result("GPU", "state_vector", "double", False, False, {})
    r.record_sample([3, 0, 5, 2])
    assert r.counts == {"00": 3, "01": 0, "10": 5, "11": 2} and r.shots == 10
    d = r.__dict__()
    assert d["data"]["counts"] is r.counts and d["backend_info"]["backend"] == "state_vector"
    r.record_sample([7, 1])
    assert r.counts == {"0": 7, "1": 1}


def test_result_dumps_files(tmp_path):
    from quict_b200.core import Circuit, H
    from quict_b200.simulation import Result
    c = Circuit(2)
    H | c(0)
    r = Result("GPU", "state_vector", "double", True, True, {}, output_path=str(tmp_path))
    r.record_circuit(c)
    r.record_amplitude(np.array([1, 0, 0, 0], dtype=np.complex128))
    r.record_sample([1, 0, 0, 0])
    names = sorted(p.name for p in tmp_path.iterdir())
    assert any(n.startswith("circuit_") for n in names) and any(n.startswith("amp_") for n in names)
    assert any(n.startswith("result_") for n in names)


@pytest.mark.gpu
def test_simulator_runs_each_backend(cuda_ok):
    from quict_b200.core import Circuit
    from quict_b200.simulation import Simulator
    c = Circuit(5)
    c.random_append(40, seed=5)
    ref = osv.run(oracle_gates(c), 5)
    res = Simulator("GPU", "state_vector", "double").run(c, shots=200)
    np.testing.assert_allclose(res["data"]["state_vector"], ref, rtol=0, atol=1e-12)
    assert res["shots"] == 200 and len(res["data"]["counts"]) == 32
    res = Simulator("GPU", "density_matrix", "double").run(c, shots=100)
    np.testing.assert_allclose(res["data"]["density_matrix"], np.outer(ref, ref.conj()), rtol=0, atol=1e-12)
    assert res["shots"] == 100
    res = Simulator("GPU", "unitary", "double").run(c, shots=50)
    np.testing.assert_allclose(res["data"]["state_vector"], ref, rtol=0, atol=1e-12)
    assert res["shots"] == 50


def test_run_flow_with_a_stand_in_backend():
    """Simulator.run's checks, record and sampling order, with a stand-in
    backend (the GPU test runs the real ones)."""
    from quict_b200.core import Circuit, H
    from quict_b200.simulation import Result, Simulator, SimulatorOptionsUnmatchedError

    class Fake:
        def __init__(self):
            self.calls = []

        def run(self, *args):
            self.calls.append(("run", args[1:]))
            return np.array([0.6, 0.8], dtype=np.complex128)

        def sample(self, shots):
            self.calls.append(("sample", shots))
            return [shots - 1, 1]

    for backend in ("state_vector", "density_matrix", "unitary"):
        s = Simulator.__new__(Simulator)
        s._device, s._backend, s._precision, s._options = "GPU", backend, "double", {}
        s._simulator = Fake()
        s._result_recorder = Result("GPU", backend, "double", False, False, {})
        c = Circuit(1)
        H | c(0)
        res = s.run(c, shots=10)
        assert res["shots"] == 10 and res["data"]["counts"] == {"0": 9, "1": 1}
        key = "density_matrix" if backend == "density_matrix" else "state_vector"
        np.testing.assert_allclose(res["data"][key], [0.6, 0.8])
        assert [k for k, _ in s._simulator.calls] == ["run", "sample"]
        if backend != "density_matrix":
            with pytest.raises(SimulatorOptionsUnmatchedError):
                s.run(c, noise_model=object())
        else:
            with pytest.raises(SimulatorOptionsUnmatchedError):
                s.run(c, state_vector=np.ones(2))
        if backend != "unitary":
            with pytest.raises(SimulatorOptionsUnmatchedError):
                s.run(np.eye(2))

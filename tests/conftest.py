import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libqsim.so")


def golden(name):
    p = os.path.join(GOLDEN, name)
    if name.endswith(".json"):
        return json.load(open(p))
    return np.load(p, allow_pickle=False)


def build_circuit(gate_list, n, precision="double"):
    """Gate list [[name, args, params]] -> quict_b200.core.Circuit."""
    from quict_b200.core import Circuit, GATE_BY_NAME, Unitary
    c = Circuit(n)
    for nm, args, params in gate_list:
        if nm == "unitary":
            m = np.array([complex(a, b) for a, b in params]).reshape(1 << len(args), 1 << len(args))
            g = Unitary(m)
        else:
            g = GATE_BY_NAME[nm]
            if params:
                g = g(*params)
        g | c(list(args))
    if precision == "single":
        c.convert_precision()
    return c


def oracle_gates(circuit):
    """Circuit -> [(matrix, args)] for the oracle (unitary gates only)."""
    out = []
    for g in circuit.gates:
        if g.type.name in ("measure", "reset", "barrier"):
            raise ValueError("oracle_gates: unitary gates only")
        out.append((np.asarray(g.matrix, dtype=np.complex128), list(g.cargs) + list(g.targs)))
    return out


@pytest.fixture(scope="session")
def cuda_ok():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from quict_b200 import _native
    _native.load()
    return True

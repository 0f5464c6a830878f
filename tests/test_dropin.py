"""Drop-in check: real QuICT.core gate objects lower to the same kernel ops as
quict_b200.core's.  The simulators read gates only through QuICT's attribute
surface (type, matrix_type, cargs, targs, pargs, matrix), so a QuICT circuit
runs unchanged when both lowerings agree.

tests/golden/dropin.npz holds the ops that quict_b200's lowering produced from
real QuICT circuits (made by make_golden.py in a checkout of the reference);
the CPU test rebuilds the same circuits with quict_b200.core and compares.
With QUICT_REFERENCE pointing at a QuICT checkout, a second test redoes the
comparison live on freshly built QuICT objects."""
import json
import os
import sys

import numpy as np
import pytest

from conftest import golden


def _ours(name, n, gl):
    from quict_b200.core import Circuit, GATE_BY_NAME, IQFT, PermFx, QFT, Unitary
    c = Circuit(n)
    for nm, args, params in gl:
        if nm == "unitary":
            m = np.array([complex(a, b) for a, b in params]).reshape(1 << len(args), 1 << len(args))
            g = Unitary(m)
        elif nm in ("qft", "iqft"):
            g = (QFT if nm == "qft" else IQFT)(params[0])
        elif nm == "perm_fx":
            g = PermFx(params[0], list(params[1]))
        else:
            g = GATE_BY_NAME[nm]
            if params:
                g = g(*params)
        g | c(list(args))
    return c


def _compare(ops, want_ops, want_mats):
    assert [[op.kind, list(op.tbits), list(op.cbits)] for op in ops] == want_ops
    mats = np.concatenate([np.asarray(op.mat, dtype=np.complex128).ravel() for op in ops])
    np.testing.assert_allclose(mats, want_mats, rtol=0, atol=1e-14)


@pytest.mark.parametrize("case", ["cfg0", "ext", "special"])
def test_quict_circuits_lower_like_ours(case):
    from quict_b200.simulation.lowering import lower_circuit
    d = golden("dropin.npz")
    n = int(d[f"{case}_n"])
    c = _ours(case, n, json.loads(str(d[f"{case}_gates"])))
    _compare(lower_circuit(c.gates, n), json.loads(str(d[f"{case}_ops"])), d[f"{case}_mats"])


@pytest.mark.skipif(not os.environ.get("QUICT_REFERENCE"), reason="QUICT_REFERENCE (a QuICT checkout) not set")
def test_live_quict_objects_lower_like_ours():
    """Builds the fixture circuits with the real QuICT package and lowers them."""
    import importlib.util
    import torch  # noqa: F401  (before the stub modules the reference needs)
    here = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "make_golden.py")
    spec = importlib.util.spec_from_file_location("make_golden", here)
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    mg.shim(os.environ["QUICT_REFERENCE"])
    from QuICT.core import Circuit
    from QuICT.core.gate import GATE_TYPE_TO_CLASS, GateType, IQFT, PermFx, QFT, Unitary
    from quict_b200.simulation.lowering import lower_circuit
    d = golden("dropin.npz")
    for case in ("cfg0", "ext", "special"):
        n = int(d[f"{case}_n"])
        c = Circuit(n)
        for nm, args, params in json.loads(str(d[f"{case}_gates"])):
            if nm == "unitary":
                g = Unitary(np.array([complex(a, b) for a, b in params]).reshape(1 << len(args), 1 << len(args)))
            elif nm in ("qft", "iqft"):
                g = (QFT if nm == "qft" else IQFT)(params[0])
            elif nm == "perm_fx":
                g = PermFx(params[0], list(params[1]))
            else:
                g = GATE_TYPE_TO_CLASS[GateType.__members__[nm]]()
                if params:
                    g = g(*params)
            g | c(list(args))
        _compare(lower_circuit(c.gates, n), json.loads(str(d[f"{case}_ops"])), d[f"{case}_mats"])
    assert "QuICT" in sys.modules

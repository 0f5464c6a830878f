"""Generate the golden fixtures in tests/golden/ by running the REFERENCE
(taofei95/quict) CPU simulators in this container.

    python tests/golden/make_golden.py --ref <QuICT checkout> [--only core,dynamic,dropin]

The reference is imported with stub modules for its plotting / QASM-lexer
dependencies (matplotlib, IPython, ply, pylatexenc, prettytable), which are
off the arithmetic path, and with numpy.complex restored (removed in numpy 2,
used in an annotation at statevector_simulator.py:525).  Only derived data is
written: gate lists, amplitudes, density matrices, counts and the uniforms the
reference consumed.  Nothing of the reference checkout is copied.

Fixtures
  gates.json          matrix / matrix_type / arity of every reference gate type
  qasm_circuit.json   random_circuit_for_correction.qasm as a gate list
  qasm_state.npy      the reference's own golden state_vector.npy (10 qubits)
  random_sv.npz       uniform random circuits (n=5, 8, 11), reference
                      CPU StateVectorSimulator, double and single precision
  ext_sv.npz          every gate family incl. 3-qubit gates (n=6): reference
                      SV and reference UnitarySimulator
  haar_sv.npz         random Haar 2q unitaries: reference SV (reversed order)
                      and reference UnitarySimulator (big-endian)
  sample.npz          reference CPU sample() counts with the numba-RNG uniforms
  midmeasure.npz      Measure / Reset inside a circuit with recorded uniforms
  dm.npz              reference DensityMatrixSimulator with noise (n=3, 4)
  grad.npz            energies and parameter-shift gradients (HEA, QAOA)
  dynamic.npz         PermFx oracles, QFT / IQFT, Triggers with and without
                      CheckPoints with the numba-RNG uniforms they consumed
  dropin.npz          real QuICT.core circuits as lowered by quict_b200 (the
                      ops its simulators run), with gate lists to rebuild them
"""
from __future__ import annotations

import argparse
import json
import os
import re
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

CFG0 = ["h", "x", "rx", "ry", "rz", "u3", "cx", "cz", "rzz", "swap"]
EXT = ["h", "hy", "s", "sdg", "x", "y", "z", "sx", "sy", "sw", "u1", "u2", "u3", "rx", "ry", "rz", "t", "tdg",
       "phase", "gphase", "cz", "cx", "cy", "ch", "crz", "cu1", "cu3", "fsim", "rxx", "ryy", "rzz", "rzx",
       "swap", "iswap", "iswapdg", "ccx", "ccz", "ccrz", "cswap"]


def shim(ref: str):
    np.complex = complex  # type: ignore[attr-defined]
    names = ["matplotlib", "matplotlib.pyplot", "matplotlib.patches", "matplotlib.path", "matplotlib.lines",
             "matplotlib.text", "matplotlib.figure", "matplotlib.collections", "matplotlib.transforms",
             "matplotlib.colors", "IPython", "IPython.display", "ply", "ply.lex", "ply.yacc", "pylatexenc",
             "pylatexenc.latexencode", "prettytable"]
    for name in names:
        m = types.ModuleType(name)
        m.__path__ = []

        def _ga(attr, _n=name):
            if attr[:1].islower():
                return lambda *a, **k: None
            return type(attr, (), {"__init__": lambda self, *a, **k: None})

        m.__getattr__ = _ga
        sys.modules[name] = m
    sys.path.insert(0, ref)


def gate_list_random(rng, n, size, names):
    out = []
    from QuICT.core.gate import GATE_TYPE_TO_CLASS, GateType
    for _ in range(size):
        nm = names[rng.integers(len(names))]
        g = GATE_TYPE_TO_CLASS[GateType.__members__[nm]]()
        k = g.controls + g.targets
        args = [int(a) for a in rng.choice(n, k, replace=False)]
        params = [float(rng.uniform(0, 2 * np.pi)) for _ in range(g.params)]
        out.append([nm, args, params])
    return out


def build(gl, n, precision="double"):
    from QuICT.core import Circuit
    from QuICT.core.gate import GATE_TYPE_TO_CLASS, GateType
    c = Circuit(n)
    for nm, args, params in gl:
        if nm == "unitary":
            from QuICT.core.gate import Unitary
            g = Unitary(np.array(params, dtype=np.complex128))
        else:
            g = GATE_TYPE_TO_CLASS[GateType.__members__[nm]]()
            if params:
                g = g(*params)
        g | c(list(args))
    if precision == "single":
        c.convert_precision()
    return c


def sv_cpu(c, precision="double"):
    from QuICT.simulation.state_vector import StateVectorSimulator
    return np.asarray(StateVectorSimulator(device="CPU", precision=precision).run(c)).copy()


def unitary_cpu(c):
    from QuICT.simulation.unitary import UnitarySimulator
    return np.asarray(UnitarySimulator(device="CPU").run(c)).copy()


def parse_qasm(path):
    gl, n = [], None
    for line in open(path):
        line = line.strip()
        if not line or line.startswith(("OPENQASM", "include", "creg")):
            continue
        m = re.match(r"qreg\s+\w+\[(\d+)\];", line)
        if m:
            n = int(m.group(1))
            continue
        m = re.match(r"(\w+)(?:\(([^)]*)\))?\s+(.*);", line)
        name, ps, qs = m.group(1), m.group(2), m.group(3)
        params = [float(eval(p, {"pi": np.pi})) for p in ps.split(",")] if ps else []
        args = [int(x) for x in re.findall(r"\[(\d+)\]", qs)]
        gl.append([name, args, params])
    return n, gl


def haar(rng, d):
    z = (rng.normal(size=(d, d)) + 1j * rng.normal(size=(d, d))) / np.sqrt(2)
    q, r = np.linalg.qr(z)
    return q * (np.diag(r) / np.abs(np.diag(r)))


def core_fixtures(ref: str):
    """gates.json ... grad.npz (see the module docstring)."""
    from QuICT.core.gate import GATE_TYPE_TO_CLASS, GateType

    # ---- gate matrices ---------------------------------------------------------------
    rng = np.random.default_rng(7)
    gates = {}
    for nm in EXT + ["id"]:
        g = GATE_TYPE_TO_CLASS[GateType.__members__[nm]]()
        params = [float(rng.uniform(0, 2 * np.pi)) for _ in range(g.params)]
        if params:
            g = g(*params)
        m = np.asarray(g.matrix, dtype=np.complex128)
        gates[nm] = {"controls": g.controls, "targets": g.targets, "params": params,
                     "matrix_type": g.matrix_type.name, "re": m.real.tolist(), "im": m.imag.tolist()}
    json.dump(gates, open(os.path.join(HERE, "gates.json"), "w"))

    # ---- the reference's own golden circuit ---------------------------------------------
    qasm = os.path.join(ref, "unit_test/simulation/data/random_circuit_for_correction.qasm")
    n, gl = parse_qasm(qasm)
    golden = np.load(os.path.join(ref, "unit_test/simulation/data/state_vector.npy"))
    ours = sv_cpu(build(gl, n))
    assert np.allclose(ours, golden, atol=1e-12), "reference CPU SV does not reproduce its golden vector"
    json.dump({"n": n, "gates": gl}, open(os.path.join(HERE, "qasm_circuit.json"), "w"))
    np.save(os.path.join(HERE, "qasm_state.npy"), golden)

    # ---- random uniform circuits ---------------------------------------------------------
    out = {}
    for n, size, seed in [(5, 40, 11), (8, 80, 12), (11, 120, 13)]:
        rng = np.random.default_rng(seed)
        gl = gate_list_random(rng, n, size, CFG0)
        out[f"n{n}_gates"] = np.array(json.dumps(gl))
        out[f"n{n}_double"] = sv_cpu(build(gl, n))
        out[f"n{n}_single"] = sv_cpu(build(gl, n, "single"), "single")
    np.savez_compressed(os.path.join(HERE, "random_sv.npz"), **out)

    # ---- every gate family ----------------------------------------------------------------
    # Two circuits, each avoiding one reference inconsistency:
    #  * the CPU SV path applies iSwap-family gates as plain swaps
    #    (swap_matrix ignores the matrix, cpu_calculator.py:238-280), so the
    #    SV circuit "a" has no iswap / iswapdg;
    #  * UnitarySimulator's CircuitMatrix applies Rzx with reversed arguments
    #    in some gate contexts only, so the Unitary circuit "b" has no rzx.
    from QuICT.simulation.unitary import UnitarySimulator
    out = {}
    n = 6
    rng = np.random.default_rng(21)
    ga = [["h", [q], []] for q in range(n)] + gate_list_random(
        rng, n, 160, [x for x in EXT if x not in ("iswap", "iswapdg")])
    out["a_gates"] = np.array(json.dumps(ga))
    out["a_sv"] = sv_cpu(build(ga, n))
    rng = np.random.default_rng(22)
    gb = [["h", [q], []] for q in range(n)] + gate_list_random(rng, n, 160, [x for x in EXT if x != "rzx"])
    out["b_gates"] = np.array(json.dumps(gb))
    out["b_unitary"] = np.asarray(UnitarySimulator(device="CPU").run(build(gb, n))).copy()
    np.savez_compressed(os.path.join(HERE, "ext_sv.npz"), **out)

    # ---- Haar 2q unitaries --------------------------------------------------------------------
    out = {}
    rng = np.random.default_rng(31)
    n = 5
    gl = [["h", [q], []] for q in range(n)]
    for _ in range(12):
        args = [int(x) for x in rng.choice(n, 2, replace=False)]
        m = haar(rng, 4)
        gl.append(["unitary", args, m.tolist()])
        gl.append(["rx", [int(rng.integers(n))], [float(rng.uniform(0, 2 * np.pi))]])
    ser = [[nm, args, ([[complex(x).real, complex(x).imag] for x in np.ravel(p)] if nm == "unitary" else p)]
           for nm, args, p in gl]
    out["gates"] = np.array(json.dumps(ser))
    out["sv_reference"] = sv_cpu(build(gl, n))
    out["unitary_reference"] = np.asarray(UnitarySimulator(device="CPU").run(build(gl, n))).copy()
    np.savez_compressed(os.path.join(HERE, "haar_sv.npz"), **out)

    # ---- sampling with the reference's numba RNG --------------------------------------------------
    import numba
    import random

    @numba.njit
    def nb_seed(s):
        random.seed(s)

    @numba.njit
    def nb_draw(k):
        r = np.empty(k)
        for i in range(k):
            r[i] = random.random()
        return r

    from QuICT.simulation.state_vector import StateVectorSimulator
    out = {}
    for n, shots, seed in [(4, 300, 101), (6, 200, 102)]:
        rng = np.random.default_rng(seed)
        gl = gate_list_random(rng, n, 6 * n, CFG0)
        c = build(gl, n)
        sim = StateVectorSimulator(device="CPU")
        sv = np.asarray(sim.run(c)).copy()
        nb_seed(seed)
        u = nb_draw(shots * n)
        nb_seed(seed)
        counts = np.asarray(sim.sample(shots), dtype=np.int64)
        out[f"n{n}_gates"] = np.array(json.dumps(gl))
        out[f"n{n}_state"] = sv
        out[f"n{n}_uniforms"] = u
        out[f"n{n}_counts"] = counts
    np.savez_compressed(os.path.join(HERE, "sample.npz"), **out)

    # ---- measure / reset inside a circuit --------------------------------------------------------
    out = {}
    n = 5
    rng = np.random.default_rng(202)
    gl = gate_list_random(rng, n, 20, CFG0)
    gl += [["measure", [1], []], ["reset", [3], []]]
    gl += gate_list_random(rng, n, 10, CFG0)
    gl += [["measure", [4], []], ["reset", [0], []], ["measure", [2], []]]
    c = build(gl, n)
    nb_seed(303)
    u = nb_draw(8)
    nb_seed(303)
    sim = StateVectorSimulator(device="CPU")
    sv = np.asarray(sim.run(c)).copy()
    out["gates"] = np.array(json.dumps(gl))
    out["uniforms"] = u
    out["state"] = sv
    out["measured"] = np.array([c.qubits[q].measured if c.qubits[q].measured is not None else -1
                                for q in range(n)])
    np.savez_compressed(os.path.join(HERE, "midmeasure.npz"), **out)

    # ---- noisy density matrix ------------------------------------------------------------------------
    from QuICT.core.noise import NoiseModel, DepolarizingError, DampingError
    from QuICT.simulation.density_matrix import DensityMatrixSimulator
    out = {}
    for n, size, seed in [(3, 10, 401), (4, 14, 402)]:
        rng = np.random.default_rng(seed)
        gl = gate_list_random(rng, n, size, ["h", "u3", "rx", "rzz", "swap", "cx", "cz"])
        amp1 = DampingError(amplitude_prob=5e-3, phase_prob=0)
        e1 = amp1.compose(DepolarizingError(1e-3, 1))
        e2 = amp1.tensor(amp1).compose(DepolarizingError(1e-2, 2))
        nm = NoiseModel(basic_gates=["h", "u3", "rx", "rzz", "swap", "cx", "cz"])
        nm.add_noise_for_all_qubits(e1, ["h", "u3", "rx"])
        nm.add_noise_for_all_qubits(e2, ["rzz", "swap", "cx", "cz"])
        dm = DensityMatrixSimulator(device="CPU", accumulated_mode=True).run(build(gl, n), noise_model=nm)
        clean = DensityMatrixSimulator(device="CPU").run(build(gl, n))
        out[f"n{n}_gates"] = np.array(json.dumps(gl))
        out[f"n{n}_noisy"] = np.asarray(dm).copy()
        out[f"n{n}_clean"] = np.asarray(clean).copy()
        out[f"n{n}_kraus1"] = np.array([np.asarray(k) for k in e1.kraus])
        out[f"n{n}_kraus2"] = np.array([np.asarray(k) for k in e2.kraus])
    np.savez_compressed(os.path.join(HERE, "dm.npz"), **out)

    # ---- energies and parameter-shift gradients from reference amplitudes --------------------
    # hardware-efficient ansatz: layers of Ry, Rz on every qubit + CZ ring;
    # H = sum Z_i Z_{i+1} + 0.5 sum X_i (open chain).  QAOA MaxCut: H on all,
    # p layers of Rzz(-gamma) per edge and Rx(2 beta) per qubit; C = sum (1 - ZZ)/2.
    out = {}
    X = np.array([[0, 1], [1, 0]])
    Z = np.diag([1.0, -1.0])

    def op_on(n, ps):
        m = np.eye(1)
        for q in range(n):
            m = np.kron(m, ps.get(q, np.eye(2)))
        return m

    def hea_gates(n, layers, th):
        gl, p = [], 0
        for _ in range(layers):
            for q in range(n):
                gl.append(["ry", [q], [float(th[p])]]); p += 1
            for q in range(n):
                gl.append(["rz", [q], [float(th[p])]]); p += 1
            for q in range(n - 1):
                gl.append(["cz", [q, q + 1], []])
            gl.append(["cz", [n - 1, 0], []])
        return gl

    def energy(gl, n, h):
        v = sv_cpu(build(gl, n))
        return float(np.real(np.vdot(v, h @ v)))

    n, layers = 4, 2
    h = sum(op_on(n, {q: Z, q + 1: Z}) for q in range(n - 1)) + 0.5 * sum(op_on(n, {q: X}) for q in range(n))
    rng = np.random.default_rng(501)
    th = rng.uniform(0, 2 * np.pi, 2 * n * layers)
    g = np.zeros_like(th)
    for k in range(th.size):
        tp, tm = th.copy(), th.copy()
        tp[k] += np.pi / 2
        tm[k] -= np.pi / 2
        g[k] = 0.5 * (energy(hea_gates(n, layers, tp), n, h) - energy(hea_gates(n, layers, tm), n, h))
    out["hea_params"], out["hea_energy"], out["hea_grad"] = th, energy(hea_gates(n, layers, th), n, h), g

    n, p = 6, 2
    edges = [(0, 1), (1, 2), (2, 3), (3, 4), (4, 5), (5, 0), (0, 3), (1, 4), (2, 5)]
    cost = sum(0.5 * (np.eye(1 << n) - op_on(n, {a: Z, b: Z})) for a, b in edges)

    def qaoa_gates(gb):
        gl = [["h", [q], []] for q in range(n)]
        for layer in range(p):
            for a, b in edges:
                gl.append(["rzz", [a, b], [float(-gb[layer])]])
            for q in range(n):
                gl.append(["rx", [q], [float(2 * gb[p + layer])]])
        return gl

    gb = rng.uniform(0, np.pi, 2 * p)
    # per-occurrence shift rule: gamma_l appears in |E| gates with scale -1, beta_l in n gates with scale 2
    gq = np.zeros(2 * p)
    for layer in range(p):
        for which, scale, count in ((layer, -1.0, len(edges)), (p + layer, 2.0, n)):
            for occ in range(count):
                for sign in (1, -1):
                    gl = qaoa_gates(gb)
                    # locate the occ-th gate of this parameter and shift its angle by +-pi/2
                    pos = [i for i, (nm, _, _) in enumerate(gl) if (nm == "rzz" and which == layer
                           and i >= n + layer * (len(edges) + n) and i < n + layer * (len(edges) + n) + len(edges))
                           or (nm == "rx" and which == p + layer and i >= n + layer * (len(edges) + n) + len(edges)
                               and i < n + (layer + 1) * (len(edges) + n))][occ]
                    gl[pos][2] = [gl[pos][2][0] + sign * np.pi / 2]
                    gq[which] += sign * 0.5 * scale * energy(gl, n, cost)
    out["qaoa_edges"], out["qaoa_params"] = np.array(edges), gb
    out["qaoa_energy"], out["qaoa_grad"] = energy(qaoa_gates(gb), n, cost), gq
    np.savez_compressed(os.path.join(HERE, "grad.npz"), **out)


def dynamic_fixtures(ref: str):
    """dynamic.npz: PermFx oracles, QFT / IQFT and Triggers with and without CheckPoints,
    run by the reference CPU StateVectorSimulator; the measurement uniforms
    come from the reference's numba RNG, seeded before each run, and are
    recorded."""
    import numba
    import random
    from QuICT.core import Circuit
    from QuICT.core.gate import CompositeGate, CX, H, PermFx, Rx, Ry, Rz, X, Y, Swap
    from QuICT.core.operator import CheckPoint, Trigger
    from QuICT.simulation.state_vector import StateVectorSimulator

    @numba.njit
    def nb_seed(s):
        random.seed(s)

    @numba.njit
    def nb_draw(k):
        r = np.empty(k)
        for i in range(k):
            r[i] = random.random()
        return r

    out = {}
    # ---- PermFx: |x, y> -> |x, y ^ f(x)> on n + 1 qubits, behind H layers
    rng = np.random.default_rng(601)
    for n in (1, 2, 3, 4):
        width = n + 2
        ones = sorted(int(x) for x in rng.choice(1 << n, max(1, (1 << n) // 2), replace=False))
        args = [int(x) for x in rng.permutation(width)[: n + 1]]
        c = Circuit(width)
        for q in range(width):
            H | c(q)
            Ry(float(rng.uniform(0, 2 * np.pi))) | c(q)
        PermFx(n, ones) | c(args)
        Rz(0.4) | c(0)
        out[f"permfx{n}_ones"] = np.array(ones)
        out[f"permfx{n}_args"] = np.array(args)
        out[f"permfx{n}_width"] = np.array(width)
        out[f"permfx{n}_pre"] = np.array([float(g.pargs[0]) for g in c.gates if g.type.name == "ry"])
        out[f"permfx{n}_pargs"] = np.array(c.gates[2 * width].pargs)
        out[f"permfx{n}_state"] = np.asarray(StateVectorSimulator(device="CPU").run(c)).copy()

    # ---- QFT / IQFT: the reference's matrices (its gate-sequence build) and
    # SV runs with the gates on scattered qubits
    from QuICT.core.gate import IQFT, QFT
    for k in (2, 3, 4, 5):
        out[f"qft{k}_matrix"] = np.asarray(QFT(k).matrix, dtype=np.complex128)
        out[f"iqft{k}_matrix"] = np.asarray(IQFT(k).matrix, dtype=np.complex128)
        width = k + 2
        # qubits 0..k-1 in order: the reference's QFTGate.matrix fails for a
        # gate placed on other qubits (circuit_matrix.py:175 looks the gate's
        # qubits up among 0..k-1), and for a permutation of them it expresses
        # the matrix in sorted-qubit order while the gate keeps its own order
        args = list(range(k))
        c = Circuit(width)
        for q in range(width):
            Ry(float(0.3 + 0.2 * q)) | c(q)
        QFT(k) | c(args)
        Rz(0.7) | c(width - 1)
        CX | c([k - 1, width - 1])
        IQFT(k) | c(args)
        out[f"qft{k}_args"] = np.array(args)
        out[f"qft{k}_state"] = np.asarray(StateVectorSimulator(device="CPU").run(c)).copy()

    def run_traced(c, seed):
        nb_seed(seed)
        u = nb_draw(8)
        nb_seed(seed)
        sv = np.asarray(StateVectorSimulator(device="CPU").run(c)).copy()
        meas = np.array([-1 if q.measured is None else int(q.measured) for q in c.qubits])
        return u, sv, meas

    # ---- Trigger without a checkpoint: the selected gates run right after it
    # (the reference's operator_unit_test.test_trigger, plus gates after it)
    for seed in (701, 702, 703, 704):
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
        u, sv, meas = run_traced(c, seed)
        out[f"trig_plain_{seed}_uniforms"], out[f"trig_plain_{seed}_state"] = u, sv
        out[f"trig_plain_{seed}_measured"] = meas

    # ---- Trigger on two qubits whose composite gates carry CheckPoint
    # children: they go in at the checkpoint's mark, after the gates between
    # the trigger and the mark; the mark then moves by the child's shift
    for seed in (711, 712, 713, 714, 715, 716):
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
        u, sv, meas = run_traced(c, seed)
        out[f"trig_cp_{seed}_uniforms"], out[f"trig_cp_{seed}_state"] = u, sv
        out[f"trig_cp_{seed}_measured"] = meas
    np.savez_compressed(os.path.join(HERE, "dynamic.npz"), **out)


def dropin_fixtures(ref: str):
    """dropin.npz: real QuICT.core circuits lowered by quict_b200's lowering
    (the ops the simulator would run), beside the gate lists that rebuild the
    same circuits with quict_b200.core.  The test compares the two lowerings."""
    from QuICT.core import Circuit
    from QuICT.core.gate import GATE_TYPE_TO_CLASS, GateType, IQFT, PermFx, QFT, Unitary
    sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
    from quict_b200.simulation.lowering import lower_circuit

    out = {}
    rng = np.random.default_rng(801)
    cases = {
        "cfg0": (8, gate_list_random(rng, 8, 120, CFG0)),
        "ext": (6, [["h", [q], []] for q in range(6)] + gate_list_random(rng, 6, 120, EXT)),
    }
    special = [["unitary", [int(x) for x in rng.choice(7, 3, replace=False)], haar(rng, 8).tolist()],
               ["qft", [0, 1, 2], [3]], ["iqft", [0, 1, 2, 3], [4]],
               ["perm_fx", [4, 1, 6], [2, [1, 2]]], ["unitary", [5, 2], haar(rng, 4).tolist()]]
    cases["special"] = (7, [["h", [q], []] for q in range(7)] + special)
    for name, (n, gl) in cases.items():
        c = Circuit(n)
        ser = []
        for nm, args, params in gl:
            if nm == "unitary":
                g = Unitary(np.array(params, dtype=np.complex128))
                ps = [[complex(x).real, complex(x).imag] for x in np.ravel(params)]
            elif nm in ("qft", "iqft"):
                g = (QFT if nm == "qft" else IQFT)(params[0])
                ps = params
            elif nm == "perm_fx":
                g = PermFx(params[0], list(params[1]))
                ps = params
            else:
                g = GATE_TYPE_TO_CLASS[GateType.__members__[nm]]()
                if params:
                    g = g(*params)
                ps = params
            g | c(list(args))
            ser.append([nm, list(args), ps])
        ops = lower_circuit(c.gates, n)
        out[f"{name}_n"] = np.array(n)
        out[f"{name}_gates"] = np.array(json.dumps(ser))
        out[f"{name}_ops"] = np.array(json.dumps([[op.kind, list(op.tbits), list(op.cbits)] for op in ops]))
        out[f"{name}_mats"] = np.concatenate([np.asarray(op.mat, dtype=np.complex128).ravel() for op in ops])
    np.savez_compressed(os.path.join(HERE, "dropin.npz"), **out)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", required=True, help="path of the QuICT reference checkout to run")
    ap.add_argument("--only", default="core,dynamic,dropin",
                    help="comma list of fixture groups to write: core (gates.json .. grad.npz), dynamic, dropin")
    a = ap.parse_args()
    parts = set(a.only.split(","))
    if "dropin" in parts:
        import torch  # noqa: F401  (before the stub modules, which torch's import would trip over)
    shim(a.ref)
    if "core" in parts:
        core_fixtures(a.ref)
    if "dynamic" in parts:
        dynamic_fixtures(a.ref)
    if "dropin" in parts:
        dropin_fixtures(a.ref)
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()

"""OpenQASM 2.0 loader and writer for the gate set of quict_b200.core.

Reads the subset QuICT writes and its unit tests use (qelib1 gate names,
parameter expressions with pi, one qreg, creg declarations, measure, reset,
barrier): the role of QuICT's ply-based parser
(QuICT/tools/interface/qasm_interface.py, QuICT/lib/qasm/) for simulation
inputs.  ``OPENQASMInterface.load_file(path).circuit`` mirrors the
reference's entry point.
"""
from __future__ import annotations

import ast
import math
import operator
import re
from typing import List, Optional

from .circuit import Circuit
from .gate import GATE_BY_NAME, BasicGate

_ALIASES = {"cnot": "cx", "toffoli": "ccx", "u": "u3", "p": "phase", "sxdg": None}

_OPS = {ast.Add: operator.add, ast.Sub: operator.sub, ast.Mult: operator.mul, ast.Div: operator.truediv,
        ast.Pow: operator.pow, ast.USub: operator.neg, ast.UAdd: operator.pos}
_FUNCS = {"sin": math.sin, "cos": math.cos, "tan": math.tan, "exp": math.exp, "ln": math.log, "sqrt": math.sqrt}


def _eval(expr: str) -> float:
    """Safe evaluation of a QASM parameter expression (numbers, pi, + - * / ^, functions)."""
    tree = ast.parse(expr.strip().replace("^", "**"), mode="eval")

    def ev(node):
        if isinstance(node, ast.Expression):
            return ev(node.body)
        if isinstance(node, ast.Constant) and isinstance(node.value, (int, float)):
            return float(node.value)
        if isinstance(node, ast.Name) and node.id == "pi":
            return math.pi
        if isinstance(node, ast.BinOp) and type(node.op) in _OPS:
            return _OPS[type(node.op)](ev(node.left), ev(node.right))
        if isinstance(node, ast.UnaryOp) and type(node.op) in _OPS:
            return _OPS[type(node.op)](ev(node.operand))
        if isinstance(node, ast.Call) and isinstance(node.func, ast.Name) and node.func.id in _FUNCS:
            return _FUNCS[node.func.id](*[ev(a) for a in node.args])
        raise ValueError(f"unsupported QASM expression: {expr!r}")

    return ev(tree)


def _split_params(s: str) -> List[str]:
    out, depth, cur = [], 0, ""
    for ch in s:
        if ch == "," and depth == 0:
            out.append(cur)
            cur = ""
            continue
        depth += ch == "("
        depth -= ch == ")"
        cur += ch
    if cur.strip():
        out.append(cur)
    return out


def loads(text: str) -> Circuit:
    text = re.sub(r"//[^\n]*", "", text)
    stmts = [s.strip() for s in text.split(";") if s.strip()]
    circuit: Optional[Circuit] = None
    reg = None
    for st in stmts:
        if st.startswith("OPENQASM") or st.startswith("include") or st.startswith("creg"):
            continue
        m = re.fullmatch(r"qreg\s+(\w+)\s*\[\s*(\d+)\s*\]", st)
        if m:
            if circuit is not None:
                raise ValueError("only one qreg is supported")
            reg, circuit = m.group(1), Circuit(int(m.group(2)))
            continue
        if circuit is None:
            raise ValueError("gate before qreg declaration")
        m = re.fullmatch(r"(\w+)\s*(?:\((.*)\))?\s+(.+)", st, flags=re.S)
        if not m:
            raise ValueError(f"cannot parse QASM statement {st!r}")
        name, params, operands = m.group(1).lower(), m.group(2), m.group(3)
        if name == "measure":
            operands = operands.split("->")[0]
        qubits = [int(q) for r, q in re.findall(r"(\w+)\s*\[\s*(\d+)\s*\]", operands) if r == reg]
        if name == "barrier":
            continue
        name = _ALIASES.get(name, name) or name
        if name not in GATE_BY_NAME:
            raise ValueError(f"unsupported gate {name!r}")
        g: BasicGate = GATE_BY_NAME[name]
        if params:
            g = g(*[_eval(p) for p in _split_params(params)])
        g | circuit(qubits)
    if circuit is None:
        raise ValueError("no qreg in the QASM text")
    return circuit


def dumps(circuit: Circuit) -> str:
    lines = ["OPENQASM 2.0;", 'include "qelib1.inc";', f"qreg q[{circuit.width()}];",
             f"creg c[{circuit.width()}];"]
    for g in circuit.gates:
        args = ", ".join(f"q[{a}]" for a in list(g.cargs) + list(g.targs))
        if g.type.name == "measure":
            lines.append(f"measure q[{g.targ}] -> c[{g.targ}];")
            continue
        p = f"({', '.join(repr(float(x)) for x in g.pargs)})" if g.pargs else ""
        lines.append(f"{g.qasm_name}{p} {args};")
    return "\n".join(lines) + "\n"


class OPENQASMInterface:
    """``OPENQASMInterface.load_file(path).circuit`` as in QuICT."""

    def __init__(self, circuit: Circuit):
        self.circuit = circuit

    @classmethod
    def load_file(cls, path: str) -> "OPENQASMInterface":
        with open(path) as f:
            return cls(loads(f.read()))

    @classmethod
    def load_string(cls, text: str) -> "OPENQASMInterface":
        return cls(loads(text))

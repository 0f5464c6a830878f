"""Host-side logic on CPU: lowering, fusion planning, C-ABI exports and
argument validation (no kernel runs)."""
import ctypes as C
import json
import os
import re

import numpy as np
import pytest

from conftest import ROOT, build_circuit, golden, oracle_gates
from oracle import sv as osv


def _apply_ops_oracle(vec, n, ops):
    """Apply lowered Ops with the oracle (vector bits -> circuit qubits)."""
    for op in ops:
        args = [n - 1 - b for b in op.cbits] + [n - 1 - b for b in op.tbits]
        u = op.dense()
        d = 1 << len(op.cbits)
        if d > 1:
            full = np.eye(u.shape[0] * d, dtype=np.complex128)
            full[-u.shape[0]:, -u.shape[0]:] = u
            u = full
        vec = osv.apply_matrix(vec, n, u, args)
    return vec


def _all_ops(n, seed, size=120):
    from quict_b200.simulation.lowering import lower_circuit
    d = golden("ext_sv.npz")
    gl = json.loads(str(d["b_gates"]))
    rng = np.random.default_rng(seed)
    perm = rng.permutation(6)
    gl = [[nm, [int(perm[a]) for a in args], p] for nm, args, p in gl][:size]
    c = build_circuit(gl, 6)
    return c, lower_circuit(c.gates, 6)


def test_lowering_reproduces_circuit():
    c, ops = _all_ops(6, 0)
    ref = osv.run(oracle_gates(c), 6)
    got = _apply_ops_oracle(osv.zero_state(6), 6, ops)
    np.testing.assert_allclose(got, ref, atol=1e-12)
    kinds = {o.kind for o in ops}
    assert kinds >= {"mat", "diag", "antidiag", "swap"}


def test_gate_matrix_follows_parameters_and_is_a_copy():
    """Fixed matrices are built once and parametrised ones are kept per gate,
    yet every access returns a fresh array that tracks the current pargs."""
    from quict_b200.core import H, Rx
    r = Rx(0.3)
    a = r.matrix
    a[...] = 0
    np.testing.assert_allclose(r.matrix, [[np.cos(0.15), -1j * np.sin(0.15)], [-1j * np.sin(0.15), np.cos(0.15)]])
    r.pargs = [1.1]
    np.testing.assert_allclose(r.matrix[0, 0], np.cos(0.55))
    r.pargs[0] = 2.0  # in-place change of the parameter list
    np.testing.assert_allclose(r.matrix[0, 0], np.cos(1.0))
    h = H.copy()
    h.matrix[0, 0] = 5
    np.testing.assert_allclose(H.matrix, np.array([[1, 1], [1, -1]]) / np.sqrt(2))
    h.convert_precision()
    assert h.matrix.dtype == np.complex64 and H.matrix.dtype == np.complex128


def test_lowering_kinds_and_controls():
    from quict_b200.core import CX, CZ, Rz, Rzz, Swap, H, CCX, sqiSwap
    from quict_b200.simulation.lowering import lower_gate
    n = 5
    (op,) = lower_gate(CX & [0, 3], n)
    assert op.kind == "antidiag" and op.cbits == (4,) and op.tbits == (1,)
    (op,) = lower_gate(CZ & [2, 1], n)
    assert op.kind == "diag" and op.cbits == (2,) and op.tbits == (3,)
    (op,) = lower_gate(Rzz(0.3) & [0, 4], n)
    assert op.kind == "diag" and op.tbits == (4, 0) and op.cbits == ()
    (op,) = lower_gate(Swap & [1, 2], n)
    assert op.kind == "swap"
    (op,) = lower_gate(CCX & [0, 1, 2], n)
    assert op.kind == "antidiag" and set(op.cbits) == {4, 3}
    (op,) = lower_gate(sqiSwap & [0, 1], n)  # typed "swap" by QuICT, but not a pure swap
    assert op.kind == "mat"
    assert lower_gate(Rz(0.0) & 1, n) == []   # identity is skipped


def test_legacy_order_reverses_only_uncontrolled_dense():
    from quict_b200.core import Unitary, CH, Rzz
    from quict_b200.simulation.lowering import lower_gate
    m = np.arange(16).reshape(4, 4) + 1j
    (a,) = lower_gate(Unitary(m) & [0, 2], 4, legacy_2q_order=True)
    (b,) = lower_gate(Unitary(m) & [0, 2], 4)
    assert a.tbits == b.tbits[::-1]
    (c,) = lower_gate(CH & [0, 2], 4, legacy_2q_order=True)
    assert c.cbits == (3,) and c.tbits == (1,)
    (d,) = lower_gate(Rzz(0.4) & [0, 2], 4, legacy_2q_order=True)
    assert d.tbits == (3, 1)


@pytest.mark.parametrize("seed", range(6))
@pytest.mark.parametrize("k,nlow", [(3, 1), (4, 2), (5, 5), (4, 0)])
@pytest.mark.parametrize("merge", [0, 2, 3])
def test_fusion_plan_preserves_semantics(seed, k, nlow, merge):
    """Executing the planner's passes in order equals the original order."""
    from quict_b200.simulation.fusion import Pass, Single, plan
    c, ops = _all_ops(6, seed)
    steps = plan(ops, 6, k, nlow, max_ops=7, merge_bits=merge)
    flat = []
    for s in steps:
        if isinstance(s, Pass):
            tile = set(range(min(nlow, k))) | set(s.hi)
            assert len(tile) == min(k, 6)
            for op in s.ops:
                assert op.xbits <= tile
            flat.extend(s.ops)
        else:
            flat.append(s.op)
    if not merge:
        assert sorted(map(id, flat)) == sorted(map(id, ops))
    ref = _apply_ops_oracle(osv.zero_state(6), 6, ops)
    got = _apply_ops_oracle(osv.zero_state(6), 6, flat)
    np.testing.assert_allclose(got, ref, atol=1e-12)


def _tiny_circuit(n, seed, size=30):
    """Random circuit on n <= 3 qubits from every fixed-size gate type that fits."""
    from quict_b200.core import Circuit, GATE_BY_NAME
    from quict_b200.core.gate import GateType
    types = [GateType[nm] for nm, g in GATE_BY_NAME.items()
             if nm not in ("measure", "reset", "barrier", "id", "unitary", "qft", "iqft", "perm", "perm_fx")
             and g.controls + g.targets <= n]
    c = Circuit(n)
    c.random_append(size, typelist=types, seed=seed)
    return c


@pytest.mark.parametrize("n", [1, 2, 3])
@pytest.mark.parametrize("merge", [0, 2])
def test_fusion_plan_on_the_smallest_circuits(n, merge):
    """1-3 qubit circuits: the planner clips the tile to the vector (k <= n,
    nlow <= k), every op lands in a pass, and the passes act like the circuit."""
    from quict_b200.simulation.fusion import Pass, iter_plan, relabel_swaps
    from quict_b200.simulation.lowering import lower_circuit
    for seed in range(4):
        c = _tiny_circuit(n, seed)
        ops = lower_circuit(c.gates, n)
        steps = list(iter_plan(relabel_swaps(ops, n), n, 11, 5, merge_bits=merge))
        flat = []
        for s in steps:
            assert isinstance(s, Pass)
            assert len(set(range(min(5, n))) | set(s.hi)) == n and all(b < n for b in s.hi)
            flat.extend(s.ops)
        ref = osv.run(oracle_gates(c), n)
        np.testing.assert_allclose(_apply_ops_oracle(osv.zero_state(n), n, flat), ref, atol=1e-12)


def test_fusion_hoists_diagonal_and_controls():
    from quict_b200.core import Circuit, H, Rz, CZ, CX, Rzz
    from quict_b200.simulation.fusion import plan
    from quict_b200.simulation.lowering import lower_circuit
    n = 20
    c = Circuit(n)
    for q in range(n):
        Rz(0.1 * q) | c(q)
    for q in range(n - 1):
        CZ | c([q, q + 1])
        Rzz(0.2) | c([q, q + 1])
    for q in range(10, 20):
        H | c(q)          # vector bits 9..0
    CX | c([0, 19])        # control bit 19 (outside any tile), target bit 0
    steps = plan(lower_circuit(c.gates, n), n, 12, 5)
    assert len(steps) == 1 and len(steps[0].ops) == len(lower_circuit(c.gates, n))


def test_matrix_table_dedups():
    from quict_b200.simulation.fusion import MatrixTable
    t = MatrixTable()
    a = t.add(np.eye(2))
    b = t.add(np.diag([1, 1j]))
    c = t.add(np.eye(2))
    assert a == c and b == 4 and t.size == 8


# ---- C-ABI ----------------------------------------------------------------------------
def _declared_symbols():
    txt = open(os.path.join(ROOT, "include", "qsim.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(qs_[a-z0-9_]+)\s*\(", txt)))


def _lib():
    from quict_b200 import build
    from quict_b200 import _native as N
    if not os.path.exists(N.LIB_PATH):
        build.build(quiet=True)
    return N.load()


def test_library_exports_every_declared_symbol():
    lib = _lib()
    syms = _declared_symbols()
    assert len(syms) >= 18
    for s in syms:
        assert hasattr(lib, s), s
    from quict_b200 import _native as N
    assert set(syms) <= set(N.SIGNATURES), set(syms) - set(N.SIGNATURES)


def test_abi_validation_without_gpu():
    """Bad arguments are rejected on the host before any CUDA call."""
    lib = _lib()
    from quict_b200 import _native as N
    assert lib.qs_version() >= 1
    m = np.eye(2, dtype=np.complex128)
    mp = m.ctypes.data_as(C.POINTER(C.c_double))
    fake = C.c_void_p(0x1000)  # never dereferenced: validation fails first
    assert lib.qs_apply_1q(None, 4, N.QS_C128, 0, 0, N.QS_K_DENSE, mp, None) == N.QS_EINVAL
    assert lib.qs_apply_1q(fake, 4, N.QS_C128, 4, 0, N.QS_K_DENSE, mp, None) == N.QS_EINVAL
    assert b"target bit" in lib.qs_last_error()
    assert lib.qs_apply_1q(fake, 4, 7, 0, 0, N.QS_K_DENSE, mp, None) == N.QS_EINVAL
    assert lib.qs_apply_1q(fake, 4, N.QS_C64, 1, 0b10, N.QS_K_DENSE, mp, None) == N.QS_EINVAL
    assert lib.qs_apply_2q(fake, 4, N.QS_C64, 1, 1, 0, N.QS_K_DENSE, mp, None) == N.QS_EINVAL
    bits = (C.c_int32 * 3)(0, 1, 1)
    assert lib.qs_apply_kq(fake, 4, N.QS_C64, 3, bits, 0, fake, None) == N.QS_EINVAL
    assert lib.qs_prob0(fake, 4, N.QS_C64, N.QS_SRC_SV, 0, None, 0, fake, None) == N.QS_EWORKSPACE
    assert lib.qs_sample_ws_bytes(20) == 8 * 2 * (1 << 10)
    # fused: a dense target outside the tile is rejected
    ps = (N.qs_pass * 1)()
    ps[0].k, ps[0].nlow, ps[0].op_begin, ps[0].op_count = 3, 2, 0, 1
    ps[0].hi[0] = 5
    ops = (N.qs_op * 1)()
    ops[0].kind, ops[0].m, ops[0].mat = N.QS_OP_MAT, 1, 0
    ops[0].gbit[0], ops[0].tgt[0] = 4, -1
    rc = lib.qs_apply_fused(fake, 8, N.QS_C128, ps, 1, ops, 1, fake, 4, None)
    assert rc == N.QS_EINVAL and b"outside the tile" in lib.qs_last_error()
    ops[0].gbit[0], ops[0].tgt[0] = 5, 2
    ops[0].mat = 1  # 4 entries needed from offset 1 in a 4-entry table
    assert lib.qs_apply_fused(fake, 8, N.QS_C128, ps, 1, ops, 1, fake, 4, None) == N.QS_EINVAL
    # adjoint pair passes: every case below fails validation before any device access
    assert lib.qs_adjoint_pair(None, 10, N.QS_C64, ps, 1, ops, 1, fake, 4, fake, 2, None) == N.QS_EINVAL
    assert lib.qs_adjoint_pair(fake, 1, N.QS_C64, ps, 1, ops, 1, fake, 4, fake, 2, None) == N.QS_EINVAL
    assert b"bit count" in lib.qs_last_error()
    assert lib.qs_adjoint_pair(fake, 10, 7, ps, 1, ops, 1, fake, 4, fake, 2, None) == N.QS_EINVAL
    assert lib.qs_adjoint_pair(fake, 10, N.QS_C64, None, 1, ops, 1, fake, 4, fake, 2, None) == N.QS_EINVAL
    # a register tile needs nlow >= 5 and k - R in [5, 8]: a 2^3 tile is refused
    ops[0].mat = 0
    ps[0].pair = 8
    assert lib.qs_adjoint_pair(fake, 8, N.QS_C64, ps, 1, ops, 1, fake, 4, fake, 2, None) == N.QS_EINVAL
    assert b"register tile" in lib.qs_last_error() or b"pair" in lib.qs_last_error()


def test_merge_ops_reduces_op_count_and_keeps_kinds():
    from quict_b200.core import Circuit, H, Rz, CX, X
    from quict_b200.simulation.fusion import merge_ops
    from quict_b200.simulation.lowering import lower_circuit
    n = 6
    c = Circuit(n)
    H | c(0); Rz(0.3) | c(0); H | c(0); CX | c([0, 1]); Rz(0.2) | c(1)
    X | c(4)                     # alone: keeps its anti-diagonal kind
    ops = lower_circuit(c.gates, n)
    merged = merge_ops(ops, frozenset(range(n)), 2)
    assert len(merged) == 2
    assert any(o.kind == "antidiag" and o.tbits == (1,) for o in merged)
    ref = _apply_ops_oracle(osv.zero_state(n), n, ops)
    got = _apply_ops_oracle(osv.zero_state(n), n, merged)
    np.testing.assert_allclose(got, ref, atol=1e-13)


@pytest.mark.parametrize("seed", range(6))
def test_swap_relabelling_acts_like_the_swaps(seed):
    """Plain SWAP gates become relabellings plus a closing swap network; the
    rewritten op list gives the same state (FP64 oracle)."""
    from quict_b200.core import Circuit, Swap
    from quict_b200.simulation.fusion import relabel_swaps
    from quict_b200.simulation.lowering import lower_circuit
    n = 7
    rng = np.random.default_rng(seed)
    c = Circuit(n)
    c.random_append(40, seed=seed)
    for _ in range(6):
        a, b = rng.choice(n, 2, replace=False)
        Swap | c([int(a), int(b)])
    c.random_append(20, seed=seed + 50)
    ops = lower_circuit(c.gates, n)
    new = relabel_swaps(ops, n)
    assert sum(o.kind == "swap" for o in new) <= sum(o.kind == "swap" for o in ops)

    def run(lst):
        v = np.zeros(1 << n, dtype=np.complex128)
        v[0] = 1
        for op in lst:
            u = op.dense()
            bits = tuple(op.cbits) + tuple(op.tbits)
            if op.cbits:
                d = u.shape[0] << len(op.cbits)
                f = np.eye(d, dtype=np.complex128)
                f[d - u.shape[0]:, d - u.shape[0]:] = u
                u = f
            v = osv.apply_matrix(v, n, u, [n - 1 - b for b in bits])
        return v

    np.testing.assert_allclose(run(new), run(ops), atol=1e-12)


@pytest.mark.parametrize("seed", range(6))
def test_merged_blocks_act_like_the_ops(seed):
    """Gate merging (dense blocks on at most 2 tile bits, diagonal blocks on at
    most 4 bits anywhere, also outside the tile) keeps the circuit's action."""
    from quict_b200.core import Circuit
    from quict_b200.simulation.fusion import _full_matrix, merge_ops
    from quict_b200.simulation.lowering import lower_circuit
    n = 7
    c = Circuit(n)
    c.random_append(90, seed=seed)
    ops = lower_circuit(c.gates, n)
    merged = merge_ops(ops, frozenset(range(4)), 2)   # bits 4..6 lie outside the tile
    assert len(merged) < len(ops)
    assert all(o.m <= 4 and (o.kind == "diag" or o.m <= 2 or o in ops) for o in merged)

    def run(lst):
        v = np.full(1 << n, 1 / np.sqrt(1 << n), dtype=np.complex128)
        for op in lst:
            bits, u = _full_matrix(op)
            v = osv.apply_matrix(v, n, u, [n - 1 - b for b in bits])
        return v

    np.testing.assert_allclose(run(merged), run(ops), atol=1e-12)


def test_planner_property_random_circuits_and_knobs():
    """Property check over random circuits and planner knobs: the passes keep
    every op's non-diagonal bits inside their tile, never exceed the op or
    matrix-table limits, and act like the circuit (FP64 oracle)."""
    from hypothesis import given, settings, strategies as st, HealthCheck
    from quict_b200 import _native as N
    from quict_b200.core import Circuit
    from quict_b200.simulation.fusion import Pass, iter_plan, op_entries, relabel_swaps
    from quict_b200.simulation.lowering import lower_circuit

    @settings(max_examples=40, deadline=None, suppress_health_check=[HealthCheck.too_slow])
    @given(n=st.integers(2, 7), seed=st.integers(0, 10 ** 6), size=st.integers(0, 60),
           k=st.integers(1, 12), nlow=st.integers(0, 6), merge=st.sampled_from([0, 2, 3]),
           max_ops=st.integers(1, 40))
    def check(n, seed, size, k, nlow, merge, max_ops):
        c = Circuit(n)
        if size:
            c.random_append(size, seed=seed)
        ops = lower_circuit(c.gates, n)
        flat = []
        for s in iter_plan(relabel_swaps(ops, n), n, k, nlow, max_ops=max_ops, merge_bits=merge):
            if isinstance(s, Pass):
                tile = set(range(min(nlow, k, n))) | set(s.hi)
                assert len(tile) == min(k, n)
                assert len(s.ops) <= max(max_ops, 1)
                assert sum(op_entries(o) for o in s.ops) <= N.QS_MAX_PASS_MATS
                for o in s.ops:
                    assert o.xbits <= tile
                flat.extend(s.ops)
            else:
                flat.append(s.op)
        ref = osv.run(oracle_gates(c), n) if size else osv.zero_state(n)
        np.testing.assert_allclose(_apply_ops_oracle(osv.zero_state(n), n, flat), ref, atol=1e-12)

    check()


def test_measured_prob_is_a_float_with_get():
    """get_measured_prob returns a float that also answers QuICT's ``.get()``."""
    from quict_b200.simulation.state_vector import MeasuredProb
    p = MeasuredProb(0.375)
    assert isinstance(p, float) and p.get() == 0.375 and p * 2 == 0.75 and type(p.get()) is float


def test_counts_list_sparse_and_dense_conversion():
    """Engine.counts_list: the nonzero-bin path and the full-list path give the
    same list (histogram replaced by a CPU bincount here)."""
    import torch
    from quict_b200.simulation.engine import Engine
    eng = Engine.__new__(Engine)
    eng.histogram = lambda idx, n: torch.bincount(idx, minlength=n)
    rng = np.random.default_rng(2)
    for ncounts, shots in ((4096, 100), (16, 1000), (1 << 12, 0), (8, 2)):
        idx = torch.as_tensor(rng.integers(0, ncounts, shots), dtype=torch.int64)
        got = eng.counts_list(idx, ncounts)
        assert isinstance(got, list) and len(got) == ncounts and sum(got) == shots
        assert got == np.bincount(idx.numpy(), minlength=ncounts).tolist()
        assert all(type(c) is int for c in got[:4])

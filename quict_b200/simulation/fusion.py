"""Fusion planner: groups a gate sequence into shared-memory tile passes.

A pass keeps a tile of 2^k amplitudes on chip: vector bits 0..nlow-1 (so each
warp streams contiguous 2^nlow-amplitude runs) plus k - nlow chosen higher
bits.  An op joins the current pass when

  * its non-diagonal targets (``Op.xbits``) fit into the tile, and
  * it commutes with every op deferred so far.

Two ops commute whenever every bit they share is a control or a diagonal
target of both (each is then block-diagonal over those bits, acting on
disjoint remaining bits), so diagonal gates (Rz, Rzz, CZ, phases) and controls
never occupy tile bits and can be hoisted past unrelated work.  Ops that
cannot be fused (dense on more than 4 bits, measurement, permutation) are
returned as ``single`` steps that run with the per-gate kernels.

The reference has no counterpart: it launches one kernel per gate
(statevector_simulator.py:155-164).
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Dict, Iterator, List, Optional, Sequence, Tuple, Union

import numpy as np

from .. import _native as N
from .lowering import Op

MAX_FUSED_M = 4


@dataclass
class Pass:
    k: int
    nlow: int
    hi: Tuple[int, ...]
    ops: List[Op] = field(default_factory=list)


@dataclass
class Single:
    op: Op


Step = Union[Pass, Single]


def fusable(op: Op) -> bool:
    if op.kind == "expect":
        return op.m <= 2 or op.is_diag_expect
    return op.kind in ("mat", "diag", "antidiag", "swap") and op.m <= MAX_FUSED_M


def default_tile(dtype_bytes: int) -> Tuple[int, int]:
    """(k, nlow) giving a 64 KiB tile with 512-byte contiguous warp runs."""
    k = 12 if dtype_bytes == 16 else 13
    nlow = 5
    return k, nlow


def _unit_swap(op: Op) -> bool:
    m = op.mat
    return (op.kind == "swap" and not op.cbits and m[0, 0] == 1 and m[1, 2] == 1 and m[2, 1] == 1
            and m[3, 3] == 1)


def relabel_swaps(ops: Sequence[Op], n: int) -> List[Op]:
    """Turn plain SWAP gates into relabellings: after swap(a, b) every later op
    addresses the other bit, so the swap moves no data.  At the end a short
    swap network (at most n - 1 swaps, usually far fewer than were removed)
    puts every bit back in place.  The result acts exactly like `ops`."""
    if not any(_unit_swap(op) for op in ops):
        return list(ops)
    where = list(range(n))  # logical bit -> physical bit
    out: List[Op] = []
    for op in ops:
        if _unit_swap(op):
            a, b = op.tbits
            where[a], where[b] = where[b], where[a]
            continue
        out.append(Op(op.kind, tuple(where[b] for b in op.tbits), tuple(where[b] for b in op.cbits), op.mat,
                      op.perm, op.qubit, op.tag, op.batch, op.slot, op.extra))
    swap = np.eye(4, dtype=np.complex128)[[0, 2, 1, 3]]
    holder = {p: q for q, p in enumerate(where)}  # physical bit -> logical bit held
    for lb in range(n):
        p = where[lb]
        if p != lb:
            other = holder[lb]  # the logical bit sitting where lb belongs
            out.append(Op("swap", (p, lb), (), swap))
            where[lb], where[other] = lb, p
            holder[lb], holder[p] = lb, other
    return out


def plan(ops: Sequence[Op], n: int, k: int, nlow: int, max_ops: int = N.QS_MAX_PASS_OPS,
         max_cost: float = float("inf"), merge_bits: int = 0) -> List[Step]:
    """All steps of ``iter_plan`` as a list."""
    return list(iter_plan(ops, n, k, nlow, max_ops, max_cost, merge_bits))


def iter_plan(ops: Sequence[Op], n: int, k: int, nlow: int, max_ops: int = N.QS_MAX_PASS_OPS,
              max_cost: float = float("inf"), merge_bits: int = 0) -> Iterator[Step]:
    """Greedy in-order planner with commutation-aware hoisting; yields each step
    as soon as it is final, so a caller can launch it while planning the rest.

    ``max_cost`` bounds the per-pass arithmetic, measured in dense-1q-gate
    equivalents (see ``op_cost``), so that a pass stays bandwidth-bound.
    ``merge_bits`` > 0 multiplies runs of ops on at most that many tile bits
    into single ops (``merge_ops``).
    """
    k = min(k, n)
    nlow = min(nlow, k)
    H = k - nlow
    low = frozenset(range(nlow))

    # per-op facts the scan reads on every pass, computed once:
    # (op, fits a tile, bits outside `low` it needs, conflict bits as a
    #  writer, block-diagonal bits, all conflict bits, cost, table entries)
    def facts(op: Op):
        xb, zb = op.xbits, op.zbits
        xc = xb - frozenset(op.extra)  # extra bits are tile requirements, not conflicts
        xh = xb - low
        return (op, fusable(op) and len(xh) <= H, xh, xc, zb, xc | zb, op_cost(op), op_entries(op))

    pending = [facts(op) for op in ops]
    while pending:
        # leading ops that can never be tile-resident run on their own
        if not pending[0][1]:
            yield Single(pending.pop(0)[0])
            continue
        hi: set = set()
        chosen: List[Op] = []
        deferred: list = []
        xblk: set = set()
        zblk: set = set()
        cost = 0.0
        entries = 0
        for idx, f in enumerate(pending):
            op, fits, xh, xc, zb, allb, c, ent = f
            if not fits:
                # a barrier: nothing after it may be hoisted above it
                deferred.extend(pending[idx:])
                break
            hoistable = not (allb & xblk) and not (xc & zblk)
            if (hoistable and len(hi | xh) <= H and len(chosen) < max_ops
                    and entries + ent <= N.QS_MAX_PASS_MATS and (cost + c <= max_cost or not chosen)):
                hi |= xh
                chosen.append(op)
                cost += c
                entries += ent
            else:
                deferred.append(f)
                xblk |= xc
                zblk |= zb
        # fill unused tile bits with the lowest free bits (longer contiguous runs)
        b = nlow
        while len(hi) < H:
            if b not in hi:
                hi.add(b)
            b += 1
        if merge_bits > 0:
            chosen = merge_ops(chosen, frozenset(range(nlow)) | frozenset(hi), merge_bits)
        yield Pass(k, nlow, tuple(sorted(hi)), chosen)
        pending = deferred


def _embed(u: np.ndarray, bits: Tuple[int, ...], into: Tuple[int, ...]) -> np.ndarray:
    """Matrix `u` acting big-endian on `bits`, expressed on `into` (a superset)."""
    k, m = len(into), len(bits)
    if tuple(bits) == tuple(into):
        return u
    if k == 2 and m == 1:  # the common merge step, written out (np.kron dominates planning time)
        t = np.zeros((2, 2, 2, 2), dtype=np.complex128)
        if bits[0] == into[0]:
            t[:, 0, :, 0] = u
            t[:, 1, :, 1] = u
        else:
            t[0, :, 0, :] = u
            t[1, :, 1, :] = u
        return t.reshape(4, 4)
    if m == 0:
        return np.eye(1 << k, dtype=np.complex128) * u.reshape(())
    full = np.kron(u, np.eye(1 << (k - m), dtype=np.complex128))  # order: bits, then the rest
    order = list(bits) + [b for b in into if b not in bits]
    # permute tensor axes from `order` to `into`
    perm = [order.index(b) for b in into]
    t = full.reshape([2] * (2 * k))
    t = np.transpose(t, perm + [k + p for p in perm])
    return t.reshape(1 << k, 1 << k)


def _full_matrix(op: Op) -> Tuple[Tuple[int, ...], np.ndarray]:
    """(bits, matrix) of an op with its controls folded in (controls first)."""
    u = op.dense()
    bits = tuple(op.cbits) + tuple(op.tbits)
    if op.cbits:
        d = u.shape[0] << len(op.cbits)
        full = np.eye(d, dtype=np.complex128)
        full[d - u.shape[0]:, d - u.shape[0]:] = u
        u = full
    return bits, u


def _to_op(bits: Tuple[int, ...], u: np.ndarray) -> Op:
    from .lowering import classify
    kind = classify(u)
    if kind == "diag":
        return Op("diag", tuple(bits), (), np.diag(u).copy())
    return Op(kind, tuple(bits), (), u)


def matrix_instr(u: np.ndarray) -> float:
    """Floating-point instructions per amplitude the generated pass code
    spends on a dense matrix: per output row, each entry that is neither 0
    nor +-1 costs 4 (complex) or 2 (real or imaginary: two products), each
    +-1 entry a complex add (2; none when it comes first), averaged over rows.
    Rows of an identity block cost nothing."""
    u = np.asarray(u)
    nz = u != 0
    unit = (u == 1) | (u == -1)
    cheap = nz & ~unit & ((u.imag == 0) | (u.real == 0))
    general = nz & ~unit & ~cheap
    per_row = 4 * general.sum(axis=1) + 2 * cheap.sum(axis=1) + 2 * unit.sum(axis=1)
    first = np.argmax(nz, axis=1)  # column of each row's first nonzero entry
    first_unit = unit[np.arange(u.shape[0]), first] & nz.any(axis=1)
    per_row = per_row - 2 * first_unit
    return float(per_row.mean())


def op_instr(op: Op) -> float:
    """``matrix_instr`` of an op (controls folded in); diagonals: 4 per
    entry that is not 1 (2 when real or imaginary), averaged; plain
    exchanges cost nothing (the generated code renames registers)."""
    if op.kind == "diag":
        d = np.asarray(op.mat).ravel()
        c = np.where(d == 1, 0, np.where((d.imag == 0) | (d.real == 0), 2, 4))
        return float(c.mean()) * 0.5 ** len(op.cbits)
    if op.kind in ("antidiag", "swap") and _unit_exchange(op):
        return 0.0
    return matrix_instr(op.dense()) * 0.5 ** len(op.cbits)


def _unit_exchange(op: Op) -> bool:
    m = op.mat
    if op.kind == "antidiag":
        return m[0, 1] == 1 and m[1, 0] == 1
    return _unit_swap(op)


def merge_ops(ops: Sequence[Op], tile: frozenset, max_bits: int = 2, max_diag_bits: int = 4,
              cost_aware: bool = True) -> List[Op]:
    """Multiply runs of ops that act on at most `max_bits` tile-resident bits
    into single ops (gate fusion at the matrix level).  Diagonal ops (phases,
    Rz, Rzz, CZ, ...) also merge among themselves into diagonal blocks of up to
    `max_diag_bits` bits on any vector bits: a diagonal costs one complex
    multiply per amplitude whatever its width.

    Open blocks hold disjoint bit sets, so they commute with each other; an op
    that touches several blocks closes them (emits them) first, and an op that
    cannot be merged (bits outside the tile, too many bits, tagged for
    gradients) closes the blocks it touches and is emitted as is.  Order is
    therefore preserved between every pair of ops that share a bit.

    With `cost_aware`, a dense merge happens only when the product costs no
    more floating-point instructions (``matrix_instr``) than the blocks and
    the op apart: a plain exchange, or a real 1-qubit gate such as H or Ry,
    can be cheaper on its own than inside a general 4 x 4 product."""
    out: List[Op] = []
    blocks: List[list] = []  # [bits tuple, matrix, [source ops], all diagonal, instr]

    def close(b):
        blocks.remove(b)
        if len(b[2]) == 1:
            out.append(b[2][0])
        else:
            out.append(_to_op(b[0], b[1]))

    for op in ops:
        S = set(op.tbits) | set(op.cbits)
        hit = [b for b in blocks if S & set(b[0])]
        union = set(S)
        for b in hit:
            union |= set(b[0])
        diag = op.kind == "diag"
        free = op.tag is None
        if free and diag and all(b[3] for b in hit) and len(union) <= max_diag_bits:
            as_diag = True
        elif free and union <= tile and len(union) <= max_bits:
            as_diag = diag and all(b[3] for b in hit)
        else:
            as_diag = None
        merged = None
        if as_diag is not None:
            merged = _merge_blocks(hit, op)
            if cost_aware and not as_diag:
                apart = sum(_block_instr(b) for b in hit) + op_instr(op)
                if matrix_instr(merged[1]) > apart:
                    merged = None
        if merged is None:
            for b in hit:
                close(b)
            if free and ((diag and len(S) <= max_diag_bits) or (S <= tile and len(S) <= max_bits)):
                bits, u = _full_matrix(op)
                blocks.append([bits, u, [op], diag])
            else:
                out.append(op)
            continue
        for b in hit:
            blocks.remove(b)
        nb, u, srcs = merged
        blocks.append([nb, u, srcs, as_diag])
    for b in list(blocks):
        close(b)
    return out


def _block_instr(b) -> float:
    """Instructions of an open block as it would be emitted."""
    return op_instr(b[2][0]) if len(b[2]) == 1 else matrix_instr(b[1])


def _merge_blocks(hit, op):
    """(bits, matrix, source ops) of the product of the hit blocks (disjoint,
    commuting) and the op."""
    bits: Tuple[int, ...] = ()
    u = None  # the first factor is taken as is (no product with an identity)
    srcs: List[Op] = []
    for b in hit:
        if u is None:
            bits, u = b[0], b[1]
        else:
            nb = bits + tuple(x for x in b[0] if x not in bits)
            u = _embed(b[1], b[0], nb) @ _embed(u, bits, nb)
            bits = nb
        srcs += b[2]
    ob, ou = _full_matrix(op)
    if u is None:
        return ob, ou, srcs + [op]
    nb = bits + tuple(x for x in ob if x not in bits)
    return nb, _embed(ou, ob, nb) @ _embed(u, bits, nb), srcs + [op]


def op_entries(op: Op) -> int:
    """Matrix entries the op occupies in a pass's on-chip matrix table."""
    if op.kind == "diag" or (op.kind == "expect" and op.is_diag_expect):
        return 1 << op.m
    return 1 << (2 * op.m)


def op_cost(op: Op) -> float:
    """Arithmetic of an op per amplitude, in units of a dense 1q gate (2 complex MACs)."""
    if op.kind == "diag":
        return 0.5
    if op.kind in ("antidiag", "swap"):
        return 0.5 * (1 << op.m) / 2
    return (1 << op.m) / 2.0


class MatrixTable:
    """De-duplicated matrix table for one run (the role of GateMatrixs,
    QuICT/simulation/utils/gate_based.py:38-101): matrices are keyed by content,
    concatenated, and copied to the device once."""

    def __init__(self):
        self._chunks: List[np.ndarray] = []
        self._index: Dict[bytes, int] = {}
        self.size = 0

    def add(self, entries: np.ndarray) -> int:
        a = np.ascontiguousarray(entries, dtype=np.complex128).ravel()
        key = a.tobytes()
        off = self._index.get(key)
        if off is None:
            off = self.size
            self._index[key] = off
            self._chunks.append(a)
            self.size += a.size
        return off

    def add_block(self, block: np.ndarray) -> int:
        """Append a per-instance block (instances x entries) without de-duplication."""
        a = np.ascontiguousarray(block, dtype=np.complex128).ravel()
        off = self.size
        self._chunks.append(a)
        self.size += a.size
        return off

    def array(self) -> np.ndarray:
        if not self._chunks:
            return np.zeros(1, dtype=np.complex128)
        return np.concatenate(self._chunks)


def emit(passes: Sequence[Pass], table: MatrixTable, inst_shift: int = 0, pair: Optional[int] = None):
    """Convert passes into ctypes (qs_pass[], qs_op[]) arrays, filling `table`.
    inst_shift > 0 marks a batched state (instance = index >> inst_shift); ops
    with per-instance tables (``Op.batch``) then get a matrix stride.  `pair`:
    the vector bit separating psi from lam in an adjoint pair vector."""
    cps = (N.qs_pass * max(1, len(passes)))()
    nops = sum(len(p.ops) for p in passes)
    cops = (N.qs_op * max(1, nops))()
    o = 0
    for pi, p in enumerate(passes):
        cp = cps[pi]
        cp.k, cp.nlow = p.k, p.nlow
        for j, h in enumerate(p.hi):
            cp.hi[j] = h
        cp.op_begin, cp.op_count = o, len(p.ops)
        cp.inst_shift = inst_shift
        cp.pair = 0 if pair is None else pair + 1
        local = {b: b for b in range(p.nlow)}
        for j, h in enumerate(p.hi):
            local[h] = p.nlow + j
        for op in p.ops:
            c = cops[o]
            o += 1
            c.m = op.m
            for j, b in enumerate(op.tbits):
                c.gbit[j] = b
                c.tgt[j] = local.get(b, -1)
            for j in range(op.m, 4):
                c.gbit[j] = 0
                c.tgt[j] = -1
            lc, gc = 0, 0
            for b in op.cbits:
                if b in local:
                    lc |= 1 << local[b]
                else:
                    gc |= 1 << b
            c.lctrl, c.gctrl = lc, gc
            c.flags = 0
            if op.batch is not None:
                c.kind = {"mat": N.QS_OP_MAT, "diag": N.QS_OP_DIAG, "antidiag": N.QS_OP_ANTI,
                          "swap": N.QS_OP_SWAP}[op.kind]
                c.mat = table.add_block(op.batch)
                c.mat_stride = op.batch.shape[1]
            elif op.kind == "expect":
                c.kind = N.QS_OP_EXPECT
                c.slot = op.slot
                if op.is_diag_expect:
                    c.flags = N.QS_OPF_DIAG
                    c.mat = table.add(np.diag(op.mat))
                else:
                    c.mat = table.add(op.mat)
            elif op.kind == "diag":
                c.kind = N.QS_OP_DIAG
                c.mat = table.add(op.mat)
            else:
                c.kind = {"mat": N.QS_OP_MAT, "antidiag": N.QS_OP_ANTI, "swap": N.QS_OP_SWAP}[op.kind]
                c.mat = table.add(op.dense())
                if op.kind == "antidiag" and op.mat[0, 1] == 1 and op.mat[1, 0] == 1:
                    c.flags = N.QS_OPF_UNIT
                if (op.kind == "swap" and op.mat[0, 0] == 1 and op.mat[1, 2] == 1 and op.mat[2, 1] == 1
                        and op.mat[3, 3] == 1):
                    c.flags = N.QS_OPF_UNIT
    return cps, len(passes), cops, nops

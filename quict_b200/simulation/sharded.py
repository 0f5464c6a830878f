"""State vector sharded over 2^g processes by its top g bits (one GPU each).

Beyond one GPU's memory (34 qubits in complex128 needs 256 GiB) the vector is
split by its g highest physical bits: rank r holds the 2^(n-g) amplitudes whose
top bits equal r.  The reference simulator has no such mode; this follows the
plain state-vector semantics of ``StateVectorSimulator.run``
(QuICT/simulation/state_vector/statevector_simulator.py:131-166) on a layout
that no single device holds.

A lowered op is placed against the current logical -> physical bit map:

- controls on global (rank) bits are decided per rank: the op runs without
  them where the rank's bit is 1 and is skipped where it is 0;
- a diagonal op with global targets keeps only the entries that match the
  rank's bits (a diagonal on the remaining local targets, or one phase);
- a plain SWAP gate only relabels (the two logical bits trade physical bits);
- any other op with a global target first swaps that global bit with a free
  local bit: the two partner ranks (rank ^ 2^j) exchange the half of their
  shard whose local bit differs from their rank bit, point to point (NCCL
  send/recv over NVLink on GPUs), and the bit map records the swap, so no
  data moves back.

Local ops run in order through the fused-pass engine between exchanges.  No
kernel waits on another rank: the exchange is a library send/recv pair.
"""
from __future__ import annotations

import bisect
from typing import List, Optional, Sequence

import numpy as np
import torch
import torch.distributed as dist

from .. import _native as N
from .fusion import _unit_swap
from .lowering import Op, lower_gate

_SWAP = np.eye(4, dtype=np.complex128)[[0, 2, 1, 3]]


class ShardedStateVector:
    """An n-qubit state vector over all ranks of `group` (a power of two);
    without an initialised process group, one unsplit vector on this device.

    ``backend`` runs the local work on one shard: ``apply_ops(vec, n, ops)``,
    ``prob0(vec, n, bit)``, ``norm2(vec, n)``, ``collapse``, ``reset`` and
    ``sample_indices`` -- by default the CUDA engine of this package on
    ``device``.  ``chunk_bytes`` bounds the staging buffers
    of one exchange (the half-shard is sent in pieces of at most that size).
    """

    def __init__(self, n: int, precision: str = "double", group=None, device: Optional[torch.device] = None,
                 backend=None, chunk_bytes: int = 1 << 28, seed: Optional[int] = None):
        self.group = group
        # without a process group the vector is one unsplit shard on this device
        self.solo = group is None and not dist.is_initialized()
        self.world = 1 if self.solo else dist.get_world_size(group)
        self.rank = 0 if self.solo else dist.get_rank(group)
        if self.world & (self.world - 1):
            raise ValueError(f"the number of ranks must be a power of two, got {self.world}")
        self.g = self.world.bit_length() - 1
        if n - self.g < 2:
            raise ValueError(f"{n} qubits over {self.world} ranks leaves fewer than 2 local bits")
        self.n = n
        self.nl = n - self.g
        self.dtype = torch.complex128 if precision == "double" else torch.complex64
        if backend is None:
            from .engine import Engine, require_cuda
            device = device or require_cuda(torch.cuda.current_device() if torch.cuda.is_available() else 0)
            backend = Engine(device)
        self.backend = backend
        self.device = device if device is not None else torch.device("cpu")
        self.chunk_bytes = int(chunk_bytes)
        self.where = list(range(n))  # logical vector bit -> physical bit
        self.exchanges = 0           # half-shard exchanges issued by this rank
        self.rng = np.random.default_rng(seed)  # measurement draws (rank 0's are used)
        self.local = torch.zeros(1 << self.nl, dtype=self.dtype, device=self.device)
        if self.rank == 0:
            self.local[0] = 1

    # ---- bit bookkeeping ----------------------------------------------------------------
    def _rank_bit(self, p: int) -> int:
        """Value of global physical bit p on this rank."""
        return (self.rank >> (p - self.nl)) & 1

    def _swap_roles(self, p: int, q: int):
        a, b = self.where.index(p), self.where.index(q)
        self.where[a], self.where[b] = q, p

    # ---- the exchange -----------------------------------------------------------------------
    def exchange(self, gbit: int, lbit: int):
        """Swap global physical bit `gbit` with local physical bit `lbit`: each
        rank sends the half of its shard whose `lbit` differs from its own
        `gbit` value to its partner and receives the partner's half in its
        place.  Afterwards the two physical bits have traded logical bits."""
        if not (self.nl <= gbit < self.n and 0 <= lbit < self.nl):
            raise ValueError(f"exchange needs a global and a local bit, got {gbit}, {lbit}")
        j = gbit - self.nl
        partner = self.rank ^ (1 << j)
        peer = partner if self.group is None else dist.get_global_rank(self.group, partner)
        keep = self._rank_bit(gbit)
        v = self.local.view(1 << (self.nl - lbit - 1), 2, 1 << lbit)
        half = v[:, 1 - keep, :]  # the slice this rank gives away and refills
        rows, cols = half.shape
        per_elem = half.element_size()
        # pieces of at most chunk_bytes: whole rows when a row fits, else column blocks
        cstep = max(1, min(cols, self.chunk_bytes // per_elem))
        rstep = max(1, self.chunk_bytes // (cols * per_elem)) if cstep == cols else 1
        # two pieces in flight: piece k+1 is on the wire while piece k is
        # written back into the shard
        inflight = None
        for r0 in range(0, rows, rstep):
            for c0 in range(0, cols, cstep):
                part = half[r0:r0 + rstep, c0:c0 + cstep]
                # complex data travels as its real view (not every backend takes complex)
                send = torch.view_as_real(part.contiguous())
                recv = torch.empty_like(send)
                reqs = dist.batch_isend_irecv([dist.P2POp(dist.isend, send, peer, self.group),
                                               dist.P2POp(dist.irecv, recv, peer, self.group)])
                if inflight is not None:
                    self._land(*inflight)
                inflight = (reqs, part, recv, send)
        if inflight is not None:
            self._land(*inflight)
        self._swap_roles(gbit, lbit)
        self.exchanges += 1

    @staticmethod
    def _land(reqs, part, recv, send):
        """Wait for one piece's send/recv pair and write the received data
        into its place (`send` is kept alive until its send completed)."""
        for q in reqs:
            q.wait()
        part.copy_(torch.view_as_complex(recv))

    # ---- placing one op -----------------------------------------------------------------
    def _free_local(self, busy: set, at: int = -1) -> int:
        """The local physical bit to trade for a rank bit: not in `busy`, and
        holding the logical bit whose next dense use (after op `at` of the
        current ``apply_ops``) is farthest away, so it can stay on a rank bit
        longest (Belady's rule); ties go to the highest bit, which keeps the
        low, warp-contiguous bits out of the exchanges."""
        uses = getattr(self, "_uses", None)
        best, best_next = -1, -1
        for p in range(self.nl - 1, -1, -1):
            if p in busy:
                continue
            if uses is None:
                return p
            u = uses[self.where.index(p)]
            k = bisect.bisect_right(u, at)
            nxt = u[k] if k < len(u) else 1 << 62
            if nxt > best_next:
                best, best_next = p, nxt
        if best < 0:
            raise ValueError("no free local bit for an exchange: too few local bits for this op")
        return best

    def _place(self, op: Op, pending: List[Op], at: int = -1) -> Optional[Op]:
        """The op in physical local bits for this rank, or None where it does
        nothing here.  Exchanges that the op needs flush `pending` first."""
        if op.kind not in ("mat", "diag", "antidiag", "swap"):
            raise ValueError(f"sharded state vectors apply unitary ops only, not {op.kind}")
        if _unit_swap(op):
            # a plain SWAP only relabels: the two logical bits trade physical bits
            a, b = op.tbits
            self.where[a], self.where[b] = self.where[b], self.where[a]
            return None
        if op.kind != "diag" and any(self.where[b] >= self.nl for b in op.tbits):
            self._flush(pending)
            for b in op.tbits:
                p = self.where[b]
                if p >= self.nl:
                    busy = {self.where[x] for x in op.tbits + op.cbits}
                    self.exchange(p, self._free_local(busy, at))
        tp = [self.where[b] for b in op.tbits]
        cp = [self.where[b] for b in op.cbits]
        if any(p >= self.nl and not self._rank_bit(p) for p in cp):
            return None  # a control on a rank bit that is 0 here
        cloc = tuple(p for p in cp if p < self.nl)
        if op.kind != "diag":
            return Op(op.kind, tuple(tp), cloc, op.mat)
        # diagonal: keep the entries whose global target bits match this rank
        m = len(tp)
        loc = [j for j in range(m) if tp[j] < self.nl]
        base = 0
        for j in range(m):
            if tp[j] >= self.nl and self._rank_bit(tp[j]):
                base |= 1 << (m - 1 - j)
        sel = []
        for i in range(1 << len(loc)):
            idx = base
            for t, j in enumerate(loc):
                if (i >> (len(loc) - 1 - t)) & 1:
                    idx |= 1 << (m - 1 - j)
            sel.append(idx)
        d = np.asarray(op.mat)[sel]
        if loc:
            return Op("diag", tuple(tp[j] for j in loc), cloc, d.copy())
        s = complex(d[0])
        if s == 1:
            return None
        # one phase: on a local control bit (entries 1, s) or on any local bit
        if cloc:
            return Op("diag", (cloc[0],), cloc[1:], np.array([1, s], dtype=np.complex128))
        return Op("diag", (0,), (), np.array([s, s], dtype=np.complex128))

    def _flush(self, pending: List[Op]):
        if pending:
            self.backend.apply_ops(self.local, self.nl, list(pending))
            pending.clear()

    # ---- public surface -------------------------------------------------------------------
    def apply_ops(self, ops: Sequence[Op]):
        """Apply lowered ops (logical vector bits) in order."""
        ops = list(ops)
        # positions where each logical bit is a dense (non-diagonal) target:
        # the lookahead of the exchange choice
        self._uses = [[] for _ in range(self.n)]
        for i, op in enumerate(ops):
            if op.kind != "diag" and not _unit_swap(op):
                for b in op.tbits:
                    self._uses[b].append(i)
        pending: List[Op] = []
        try:
            for i, op in enumerate(ops):
                placed = self._place(op, pending, i)
                if placed is not None:
                    pending.append(placed)
            self._flush(pending)
        finally:
            self._uses = None

    def run(self, circuit) -> "ShardedStateVector":
        """Apply a circuit from the current state (|0...0> at construction).
        Measure and Reset gates act mid-circuit with the reference's rules
        (outcomes are recorded on ``circuit.qubits[q].measured``); Perm gates
        are refused."""
        if int(circuit.width()) != self.n:
            raise ValueError(f"circuit has {circuit.width()} qubits, the vector {self.n}")
        ops: List[Op] = []
        for g in circuit.gates:
            for op in lower_gate(g, self.n):
                if op.kind in ("measure", "reset"):
                    self.apply_ops(ops)
                    ops = []
                    if op.kind == "measure":
                        circuit.qubits[op.qubit].measured = self.measure(op.qubit)
                    else:
                        self.reset(op.qubit)
                else:
                    ops.append(op)
        self.apply_ops(ops)
        return self

    # ---- measurement ------------------------------------------------------------------------
    def _shared_uniform(self) -> float:
        """One uniform, the same on every rank (rank 0 draws it)."""
        u = float(self.rng.random()) if self.rank == 0 else 0.0
        if self.solo:
            return u
        t = torch.tensor([u], dtype=torch.float64, device=self._reduce_dev())
        dist.broadcast(t, 0 if self.group is None else dist.get_global_rank(self.group, 0), group=self.group)
        return float(t.item())

    def measure(self, qubit: int, u: Optional[float] = None) -> int:
        """Measure one qubit with the reference rule: outcome 1 iff u > P(0),
        the kept half scaled by 1/sqrt(p), the other zeroed.  `u`, if given,
        must be the same on every rank."""
        p0 = self.prob0(qubit)
        if u is None:
            u = self._shared_uniform()
        one = int(u > p0)
        scale = 1.0 / np.sqrt((1.0 - p0) if one else p0)
        p = self.where[self.n - 1 - qubit]
        if p < self.nl:
            self.backend.collapse(self.local, self.nl, p, one, scale)
        elif self._rank_bit(p) == one:
            self.local.mul_(scale)
        else:
            self.local.zero_()
        return one

    def reset(self, qubit: int):
        """Reset one qubit to |0> with the reference rule: alpha = sqrt(P(0));
        alpha < 1e-6 moves the |1> half into |0>, else the |0> half is divided
        by alpha; the |1> half becomes 0.  On a rank bit the move is a whole
        shard sent from the bit-1 rank to its bit-0 partner."""
        p0 = self.prob0(qubit)
        p = self.where[self.n - 1 - qubit]
        if p < self.nl:
            self.backend.reset(self.local, self.nl, p, p0)
            return
        alpha = float(np.sqrt(p0))
        mine = self._rank_bit(p)
        if alpha >= 1e-6:
            if mine:
                self.local.zero_()
            else:
                self.local.div_(alpha)
            return
        partner = self.rank ^ (1 << (p - self.nl))
        peer = partner if self.group is None else dist.get_global_rank(self.group, partner)
        buf = torch.view_as_real(self.local)
        if mine:
            dist.send(buf.contiguous(), peer, group=self.group)
            self.local.zero_()
        else:
            recv = torch.empty_like(buf)
            dist.recv(recv, peer, group=self.group)
            self.local.copy_(torch.view_as_complex(recv))

    def canonical(self):
        """Bring every logical bit back to its own physical bit (exchanges for
        the global bits, swap ops for the local ones)."""
        pending: List[Op] = []
        for G in range(self.nl, self.n):
            if self.where[G] == G:
                continue
            p = self.where[G]  # where logical bit G sits now
            if p >= self.nl:   # on another global bit: route it through a local bit
                tmp = self._free_local(set())
                self.exchange(p, tmp)
                p = tmp
            self.exchange(G, p)
        for b in range(self.nl):
            p = self.where[b]
            if p != b:
                pending.append(Op("swap", (p, b), (), _SWAP))
                self._swap_roles(p, b)
        self._flush(pending)

    def _sum_over_ranks(self, x: float) -> float:
        if self.solo:
            return float(x)
        dev = self.device if dist.get_backend(self.group) == "nccl" else torch.device("cpu")
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        dist.all_reduce(t, group=self.group)
        return float(t.item())

    def norm2(self) -> float:
        return self._sum_over_ranks(self.backend.norm2(self.local, self.nl))

    def prob0(self, qubit: int) -> float:
        """P(qubit = 0) over the whole vector (QuICT qubit index)."""
        p = self.where[self.n - 1 - qubit]
        if p < self.nl:
            mine = self.backend.prob0(self.local, self.nl, p)
        else:
            mine = 0.0 if self._rank_bit(p) else self.backend.norm2(self.local, self.nl)
        return self._sum_over_ranks(mine)

    def _reduce_dev(self):
        return self.device if (not self.solo and dist.get_backend(self.group) == "nccl") else torch.device("cpu")

    def sample(self, shots: int, uniforms=None, seed: Optional[int] = None) -> np.ndarray:
        """Basis indices of `shots` samples, one uniform per shot, on every
        rank: the smallest global index i with u * total <= CDF[i] (FP64),
        the rule of ``StateVectorSimulator.sample(mode="cdf")``.  The shot's
        rank comes from the cumulative shard masses (never a rank of zero
        mass); that rank then samples its own shard with the uniform
        (u * total - mass of the ranks before it) / its own mass, which its
        sampler scales back by that mass.  `uniforms`, if given, must be the
        same on every rank; otherwise rank 0 draws them (numpy
        ``default_rng(seed)``) and broadcasts them."""
        self.canonical()
        dev = self._reduce_dev()
        if uniforms is None:
            u = torch.as_tensor(np.random.default_rng(seed).random(shots) if self.rank == 0 else np.zeros(shots),
                                dtype=torch.float64)
            if not self.solo:
                u = u.to(dev)
                dist.broadcast(u, 0 if self.group is None else dist.get_global_rank(self.group, 0), group=self.group)
            u = u.cpu().numpy()
        else:
            u = np.asarray(uniforms, dtype=np.float64).ravel()[:shots]
        mass = torch.tensor([self.backend.norm2(self.local, self.nl)], dtype=torch.float64, device=dev)
        if not self.solo:
            parts = [torch.empty_like(mass) for _ in range(self.world)]
            dist.all_gather(parts, mass, group=self.group)
            mass = torch.cat(parts)
        m = mass.cpu().numpy()
        cdf = np.cumsum(m)
        live = np.flatnonzero(m > 0)
        t = u * cdf[-1]
        owner = np.searchsorted(cdf, t, side="left")
        owner = np.clip(owner, live[0], live[-1]) if live.size else np.zeros_like(owner)
        mine = np.flatnonzero(owner == self.rank)
        out = np.zeros(shots, dtype=np.int64)
        if mine.size:
            before = cdf[self.rank - 1] if self.rank > 0 else 0.0
            ul = torch.as_tensor(np.clip((t[mine] - before) / m[self.rank], 0.0, 1.0), dtype=torch.float64)
            idx = self.backend.sample_indices(self.local, self.nl, ul, N.QS_SAMPLE_CDF)
            out[mine] = (np.asarray(idx.cpu().numpy() if hasattr(idx, "cpu") else idx, dtype=np.int64)
                         + (self.rank << self.nl))
        if self.solo:
            return out
        t = torch.as_tensor(out).to(dev)
        dist.all_reduce(t, group=self.group)  # every shot is filled by exactly one rank
        return t.cpu().numpy()

    def gather(self, dst: int = 0) -> Optional[np.ndarray]:
        """The full vector on rank `dst` (after ``canonical``), None elsewhere;
        for vectors that fit one host."""
        self.canonical()
        if self.solo:
            return self.local.detach().cpu().numpy()
        src = torch.view_as_real(self.local.detach())
        if dist.get_backend(self.group) != "nccl":
            src = src.cpu()
        parts = [torch.empty_like(src) for _ in range(self.world)] if self.rank == dst else None
        dist.gather(src, parts, dst=dst if self.group is None else dist.get_global_rank(self.group, dst),
                    group=self.group)
        return torch.view_as_complex(torch.cat(parts)).cpu().numpy() if self.rank == dst else None

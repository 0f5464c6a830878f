"""Batched expectation values and adjoint-method gradients on the GPU.

B parameter sets of an n-qubit ``ParamCircuit`` are simulated as ONE vector of
2^(n + log2 B') amplitudes (B' = B rounded up to a power of two): instance i
occupies amplitudes [i 2^n, (i+1) 2^n), gates act on the low n bits and each
parameterised gate reads its instance's matrix through a per-instance stride,
so a fused pass advances every instance at once.

  forward   psi = U(theta)|0>                       (fused passes, qs_apply_fused)
            lam = H psi                             (qs_apply_pauli_sum)
            E   = <psi|lam> per instance            (qs_inner_batched, FP64)
  backward  for gates k = L..1 (fused into tile passes, qs_adjoint_pair):
              g_k += scale_k * Im <lam| G_k |psi>   (per-tile FP64 partials)
              psi <- U_k^dagger psi,  lam <- U_k^dagger lam
            partials -> per (gate, instance) sums   (qs_segment_sum)

psi and lam live in the two halves of one vector; the top bit (the "pair
bit") selects the half.  The backward passes run on that vector with the pair
bit in the tile, so the register-tile kernel holds each psi amplitude beside
its lam partner and applies U^dagger to both with one op.  Instances too small
for register tiles use the shared-memory kernel (qs_adjoint_fused) instead.

With U(theta) = exp(-i theta G / 2), dE/dtheta_k = 2 Re <lam_k| dU_k |psi_{k-1}>
= scale_k * Im <lam_k| G_k |psi_k>.  ``parameter_shift`` computes the same
gradient from 2 * P shifted forward runs (the baseline the adjoint is compared
against).
"""
from __future__ import annotations

import ctypes as C
from typing import List, Optional, Sequence, Tuple

import numpy as np
import torch

from .. import _native as N
from ..simulation.engine import Workspace, qs_dtype, require_cuda
from ..simulation.fusion import MatrixTable, Pass, Single, default_tile, emit, plan
from ..simulation.lowering import Op, classify
from .circuit import GENERATORS, ParamCircuit, PauliSum, rotation


def _pow2(b: int) -> int:
    p = 1
    while p < b:
        p <<= 1
    return p


def _batched_rotations(kind, thetas: np.ndarray, inverse: bool = False) -> Tuple[str, np.ndarray]:
    """Per-instance exp(-i t G/2) tables: ("diag", (B, 2^m)) or ("mat", (B, 4^m)).
    `kind`: a GENERATORS key or a generator matrix (diagonal ones may have any
    real eigenvalues; dense ones must square to I)."""
    g = GENERATORS[kind] if isinstance(kind, str) else kind
    t = -thetas if inverse else thetas
    if classify(g) == "diag":
        return "diag", np.exp(-0.5j * t[:, None] * np.diag(g).real[None, :])
    c = np.cos(t / 2)[:, None]
    s = np.sin(t / 2)[:, None]
    eye = np.eye(g.shape[0]).ravel()[None, :]
    return "mat", c * eye - 1j * s * g.ravel()[None, :]


class _Unit:
    """One op of the gradient circuit: a fixed gate, a parameterised gate, or a
    group of gates sharing one parameter that commute: diagonal rotations (e.g.
    the Rzz gates of a QAOA cost layer) merged into one diagonal on at most 4
    qubits, or a pair of one-qubit rotations on different qubits (e.g. two Rx
    of a QAOA mixer), whose unitary is the tensor product of theirs (`pair`)."""

    def __init__(self, entries: List[int], qubits: Tuple[int, ...], gen: Optional[np.ndarray] = None,
                 fixed: Optional[np.ndarray] = None, index: int = -1, scale: float = 1.0,
                 pair: Optional[Tuple[np.ndarray, np.ndarray]] = None):
        self.entries, self.qubits, self.gen, self.fixed = entries, qubits, gen, fixed
        self.index, self.scale, self.pair = index, scale, pair

    def tables(self, thetas: np.ndarray, inverse: bool) -> Tuple[str, np.ndarray]:
        """Per-instance tables of exp(-i theta G / 2) (see _batched_rotations)."""
        if self.pair is None:
            return _batched_rotations(self.gen, thetas, inverse)
        _, a = _batched_rotations(self.pair[0], thetas, inverse)
        _, b = _batched_rotations(self.pair[1], thetas, inverse)
        u = np.einsum("bij,bkl->bikjl", a.reshape(-1, 2, 2), b.reshape(-1, 2, 2)).reshape(-1, 16)
        return "mat", u


def _diag_on(g: np.ndarray, qubits: Sequence[int], into: Sequence[int]) -> np.ndarray:
    """Diagonal of generator g (on `qubits`, big-endian) as a diagonal on `into`."""
    d = np.diag(g).real
    k = len(into)
    out = np.zeros(1 << k)
    for idx in range(1 << k):
        sub = 0
        for q in qubits:
            sub = (sub << 1) | ((idx >> (k - 1 - into.index(q))) & 1)
        out[idx] = d[sub]
    return out


def gate_units(circuit: ParamCircuit, cluster: bool = True, max_qubits: int = 4) -> List[_Unit]:
    """The circuit as gate units.  With `cluster`, each maximal run of
    consecutive diagonal rotations with the same parameter and scale (they
    commute) is split greedily into groups of at most `max_qubits` qubits, and
    each group becomes one diagonal unit whose generator is the sum of the
    group's generators; its gradient term then covers the whole group."""
    E = circuit.entries
    out: List[_Unit] = []
    i = 0
    while i < len(E):
        e = E[i]
        if e.kind == "fixed":
            out.append(_Unit([i], e.qubits, fixed=e.matrix))
            i += 1
            continue
        g = GENERATORS[e.kind]
        j = i + 1
        if cluster and classify(g) == "diag":
            while (j < len(E) and E[j].kind != "fixed" and classify(GENERATORS[E[j].kind]) == "diag"
                   and E[j].index == e.index and E[j].scale == e.scale):
                j += 1
        if cluster and classify(g) != "diag" and len(e.qubits) == 1:
            # one-qubit rotations with the same parameter on different qubits
            # commute: pair them up as tensor products
            seen = {e.qubits[0]}
            while (j < len(E) and E[j].kind != "fixed" and len(E[j].qubits) == 1
                   and classify(GENERATORS[E[j].kind]) != "diag" and E[j].index == e.index
                   and E[j].scale == e.scale and E[j].qubits[0] not in seen):
                seen.add(E[j].qubits[0])
                j += 1
            for t in range(i, j - 1, 2):
                ga, gb = GENERATORS[E[t].kind], GENERATORS[E[t + 1].kind]
                gen = np.kron(ga, np.eye(2)) + np.kron(np.eye(2), gb)
                out.append(_Unit([t, t + 1], E[t].qubits + E[t + 1].qubits, gen=gen, index=e.index,
                                 scale=e.scale, pair=(ga, gb)))
            if (j - i) % 2:
                t = j - 1
                out.append(_Unit([t], E[t].qubits, gen=GENERATORS[E[t].kind], index=e.index, scale=e.scale))
            i = j
            continue
        if j - i == 1:
            out.append(_Unit([i], e.qubits, gen=g, index=e.index, scale=e.scale))
            i = j
            continue
        groups: List[Tuple[set, List[int]]] = []
        for t in range(i, j):
            qs = set(E[t].qubits)
            best, shared = None, -1
            for grp in groups:
                if len(grp[0] | qs) <= max_qubits and len(grp[0] & qs) > shared:
                    best, shared = grp, len(grp[0] & qs)
            if best is None:
                groups.append((set(qs), [t]))
            else:
                best[0].update(qs)
                best[1].append(t)
        for qs, members in groups:
            into = tuple(sorted(qs))
            d = sum(_diag_on(GENERATORS[E[t].kind], E[t].qubits, into) for t in members)
            out.append(_Unit(members, into, gen=np.diag(d).astype(np.complex128), index=e.index, scale=e.scale))
        i = j
    return out


class BatchedAdjoint:
    """Energies and gradients of <psi(theta)|H|psi(theta)> for a batch of theta."""

    def __init__(self, circuit: ParamCircuit, observable: PauliSum, precision: str = "single",
                 device_id: int = 0, tile_bits: Optional[int] = None, pair: bool = True,
                 pair_tile_bits: Optional[int] = None, jit: bool = True):
        if observable.n != circuit.n:
            raise ValueError("observable and circuit act on different qubit counts")
        k0, _ = default_tile(8 if precision == "single" else 16)
        # smallest register tile: 2^(R+5) amplitudes (R = 4 / 5 register bits)
        min_k = 9 if precision == "double" else 10
        if pair_tile_bits is not None and not min_k <= pair_tile_bits <= k0:
            raise ValueError(f"pair_tile_bits must lie in [{min_k}, {k0}] for {precision} precision")
        self.circuit = circuit
        self.obs = observable
        self.n = circuit.n
        self.dev = require_cuda(device_id)
        self.cdtype = torch.complex64 if precision == "single" else torch.complex128
        self.np_dtype = np.complex64 if precision == "single" else np.complex128
        # forward tiles; a small instance still gets a few tiles (CTAs), so
        # that it does not run on one SM alone
        self.k = min(tile_bits or max(min_k, min(k0 - 1, self.n - 3)), self.n)
        self.nlow = min(5, self.k)
        # register-tile backward on the psi/lam pair vector: tile of up to k0
        # bits, one of them the pair bit (two tile buffers of 2^k0 amplitudes
        # fill 128 KB of shared memory: one CTA per SM)
        self.pair_k = pair_tile_bits or min(k0, max(min_k, self.n + 1 - 3))
        self.pair_min_k = min_k
        self.pair = pair and self.pair_min_k <= self.pair_k <= self.n + 1
        # jit: register passes may run as run-time compiled kernels (the
        # library's JIT mode decides when); False keeps the generic kernels
        self.jit = jit
        self.ws = Workspace(self.dev)
        self.launches = 0
        self.pauli = observable.masks()
        self._param_entries = [i for i, e in enumerate(circuit.entries) if e.kind != "fixed"]
        self._units = gate_units(circuit, cluster=True)        # forward / adjoint sweep
        self._units_plain = gate_units(circuit, cluster=False)  # one unit per entry (parameter shift)
        self._param_units = [u for u, un in enumerate(self._units) if un.fixed is None]

    # ---- helpers ---------------------------------------------------------------------------
    @property
    def stream(self):
        return N.stream_ptr(torch.cuda.current_stream(self.dev))

    def _vbits(self, qubits: Sequence[int]) -> Tuple[int, ...]:
        return tuple(self.n - 1 - q for q in qubits)

    def _gate_ops(self, params: np.ndarray, inverse: bool, units: Optional[List[_Unit]] = None
                  ) -> List[Tuple[int, Op]]:
        """[(unit index, op)] in circuit order; per-instance tables for rotations."""
        out = []
        for i, u in enumerate(self._units if units is None else units):
            tb = self._vbits(u.qubits)
            if u.fixed is not None:
                m = np.conj(u.fixed.T) if inverse else u.fixed
                k = classify(m)
                out.append((i, Op("diag", tb, (), np.diag(m).copy()) if k == "diag" else Op(k, tb, (), m.copy())))
            else:
                kind, tab = u.tables(u.scale * params[:, u.index], inverse)
                m0 = tab[0].copy() if kind == "diag" else tab[0].reshape(1 << len(tb), -1)
                out.append((i, Op(kind, tb, (), m0, tag=("param", i), batch=tab)))
        return out

    def _run(self, vec: torch.Tensor, nbits: int, ops: Sequence[Op], lam: Optional[torch.Tensor] = None,
             partials: Optional[torch.Tensor] = None):
        steps = plan(ops, nbits, self.k, self.nlow, merge_bits=0 if lam is not None else 2)
        passes = [s for s in steps if isinstance(s, Pass)]
        if len(passes) != len(steps):
            raise RuntimeError("a gradient-circuit op could not be fused")
        table = MatrixTable()
        cps, npass, cops, nops = emit(passes, table, inst_shift=self.n)
        host = table.array().astype(self.np_dtype)
        mats = torch.from_numpy(host).to(self.dev)
        if lam is None:
            hp = C.c_void_p(host.ctypes.data) if self.jit else None
            N.call("qs_apply_fused_ex", C.c_void_p(vec.data_ptr()), nbits, qs_dtype(vec), cps, npass, cops, nops,
                   C.c_void_p(mats.data_ptr()), hp, int(mats.numel()), self.stream)
        else:
            N.call("qs_adjoint_fused", C.c_void_p(vec.data_ptr()), C.c_void_p(lam.data_ptr()), nbits,
                   qs_dtype(vec), cps, npass, cops, nops, C.c_void_p(mats.data_ptr()), int(mats.numel()),
                   C.c_void_p(partials.data_ptr()), int(partials.numel()), self.stream)
        self.launches += npass
        self._keep = mats

    def _prepare(self, params) -> Tuple[np.ndarray, int, int]:
        p = params.detach().cpu().numpy() if isinstance(params, torch.Tensor) else np.asarray(params)
        p = np.atleast_2d(np.asarray(p, dtype=np.float64))
        if p.shape[1] < self.circuit.num_params:
            raise ValueError(f"expected {self.circuit.num_params} parameters per instance, got {p.shape[1]}")
        b = p.shape[0]
        bp = _pow2(b)
        if bp != b:
            p = np.concatenate([p, np.zeros((bp - b, p.shape[1]))], axis=0)
        return p, b, bp

    def _zero_states(self, bp: int) -> torch.Tensor:
        vec = torch.zeros(bp << self.n, dtype=self.cdtype, device=self.dev)
        vec.view(bp, 1 << self.n)[:, 0] = 1
        return vec

    # ---- public API --------------------------------------------------------------------------
    def states(self, params) -> torch.Tensor:
        """Final states, shape (B, 2^n)."""
        p, b, bp = self._prepare(params)
        nbits = self.n + (bp.bit_length() - 1)
        vec = self._zero_states(bp)
        self._run(vec, nbits, [op for _, op in self._gate_ops(p, False)])
        return vec.view(bp, 1 << self.n)[:b]

    def _energy(self, psi: torch.Tensor, nbits: int, bp: int) -> Tuple[torch.Tensor, torch.Tensor]:
        lam = torch.empty_like(psi)
        x, z, c = self.pauli
        N.call("qs_apply_pauli_sum", C.c_void_p(psi.data_ptr()), C.c_void_p(lam.data_ptr()), nbits,
               qs_dtype(psi), x.ctypes.data_as(C.c_void_p), z.ctypes.data_as(C.c_void_p),
               c.ctypes.data_as(C.c_void_p), len(x), self.stream)
        e = torch.empty(2 * bp, dtype=torch.float64, device=self.dev)
        ws = self.ws.get(16 * bp * 1024 + 256)  # qs_inner_batched: up to 1024 partials per instance
        N.call("qs_inner_batched", C.c_void_p(psi.data_ptr()), C.c_void_p(lam.data_ptr()), nbits, qs_dtype(psi),
               self.n, C.c_void_p(e.data_ptr()), C.c_void_p(ws.data_ptr()), ws.numel(), self.stream)
        self.launches += 2
        return lam, e.view(bp, 2)[:, 0]

    def energies(self, params) -> torch.Tensor:
        p, b, bp = self._prepare(params)
        nbits = self.n + (bp.bit_length() - 1)
        psi = self._zero_states(bp)
        self._run(psi, nbits, [op for _, op in self._gate_ops(p, False)])
        _, e = self._energy(psi, nbits, bp)
        return e[:b]

    def plan_gradient(self, params) -> "GradientPlan":
        """Host work for one gradient evaluation: op tables, pass plans, device
        buffers.  ``launch`` then issues kernels only (so it can be captured in a
        CUDA graph and replayed)."""
        p, b, bp = self._prepare(params)
        nbits = self.n + (bp.bit_length() - 1)
        gp = GradientPlan(b=b, bp=bp, nbits=nbits)
        fwd_ops, ops, gp.nslots, w = self.sweep_ops(p)
        gp.fwd = self._build(nbits, fwd_ops, adjoint=False)
        half = bp << self.n
        # with several instances the tile's non-pair bits must stay below the
        # instance bits, so the tile takes at most n of them
        pk = self.pair_k if bp == 1 else min(self.pair_k, self.n)
        # the pair kernel takes dense ops on at most 2 qubits
        narrow = all(len(u.qubits) <= 2 or (u.fixed is None and classify(u.gen) == "diag")
                     or (u.fixed is not None and classify(u.fixed) == "diag") for u in self._units)
        gp.pair = self.pair and narrow and self.pair_min_k <= pk <= nbits + 1
        if gp.pair:
            ops = [Op(o.kind, o.tbits, o.cbits, o.mat, tag=o.tag, batch=o.batch, slot=o.slot, extra=(nbits,))
                   if o.kind == "expect" else o for o in ops]
            gp.bwd = self._build(nbits + 1, ops, adjoint=True, k=pk, pair=nbits)
            gp.pl = torch.empty(2 * half, dtype=self.cdtype, device=self.dev)
            gp.psi, gp.lam = gp.pl[:half], gp.pl[half:]
            gp.tiles_per_inst = 1 << (self.n + 1 - pk)
        else:
            gp.bwd = self._build(nbits, ops, adjoint=True)
            gp.psi = torch.empty(half, dtype=self.cdtype, device=self.dev)
            gp.lam = torch.empty_like(gp.psi)
            gp.tiles_per_inst = 1 << (self.n - self.k)
        gp.partials = torch.empty(2 * gp.nslots * bp * gp.tiles_per_inst, dtype=torch.float64, device=self.dev)
        gp.sums = torch.empty(2 * gp.nslots * bp, dtype=torch.float64, device=self.dev)
        gp.e = torch.empty(2 * bp, dtype=torch.float64, device=self.dev)
        gp.ws = torch.empty(16 * bp * 1024 + 256, dtype=torch.uint8, device=self.dev)
        gp.weights = torch.from_numpy(w).to(self.dev)
        gp.grads = torch.zeros(self.circuit.num_params, bp, dtype=torch.float64, device=self.dev)
        return gp

    def sweep_ops(self, p: np.ndarray) -> Tuple[List[Op], List[Op], int, np.ndarray]:
        """Op lists of one gradient evaluation of the (padded) parameter rows
        `p`: the forward ops, the backward sweep (inverse gates in reverse
        order, each parameterised unit preceded by its EXPECT op), the number
        of EXPECT slots and the weights W (parameters x slots): gradient =
        W Im<lam|G|psi>, W[param, slot] = the unit's scale, so that gates
        sharing a parameter are summed in a fixed (deterministic) order."""
        fwd = [op for _, op in self._gate_ops(p, False)]
        inv = self._gate_ops(p, True)
        slot_of = {u: s for s, u in enumerate(self._param_units)}
        ops: List[Op] = []
        for ui, op in reversed(inv):
            un = self._units[ui]
            if un.fixed is None:
                ops.append(Op("expect", op.tbits, (), un.gen, tag=("expect", ui), slot=slot_of[ui]))
            ops.append(op)
        nslots = max(1, len(self._param_units))
        w = np.zeros((self.circuit.num_params, nslots))
        for s_, u in enumerate(self._param_units):
            w[self._units[u].index, s_] += self._units[u].scale
        return fwd, ops, nslots, w

    def _build(self, nbits: int, ops: Sequence[Op], adjoint: bool, k: Optional[int] = None,
               pair: Optional[int] = None):
        steps = plan(ops, nbits, k or self.k, self.nlow, merge_bits=0 if adjoint else 2)
        passes = [s for s in steps if isinstance(s, Pass)]
        if len(passes) != len(steps):
            raise RuntimeError("a gradient-circuit op could not be fused")
        table = MatrixTable()
        cps, npass, cops, nops = emit(passes, table, inst_shift=self.n, pair=pair)
        host = table.array().astype(self.np_dtype)
        mats = torch.from_numpy(host).to(self.dev)
        # the host copy lets register passes run as generated kernels
        return (cps, npass, cops, nops, mats, host)

    def launch(self, gp: "GradientPlan", stream=None):
        """Issue the forward, energy and adjoint kernels of a plan on `stream`
        (default: the current stream).  Results land in gp.e and gp.grads."""
        st = N.stream_ptr(stream if stream is not None else torch.cuda.current_stream(self.dev))
        n, bp, nbits = self.n, gp.bp, gp.nbits
        psi, lam = gp.psi, gp.lam
        psi.zero_()
        psi.view(bp, 1 << n)[:, 0] = 1
        cps, npass, cops, nops, mats, host = gp.fwd
        hp = C.c_void_p(host.ctypes.data) if self.jit else None
        N.call("qs_apply_fused_ex", C.c_void_p(psi.data_ptr()), nbits, qs_dtype(psi), cps, npass, cops, nops,
               C.c_void_p(mats.data_ptr()), hp, int(mats.numel()), st)
        x, z, c = self.pauli
        N.call("qs_apply_pauli_sum", C.c_void_p(psi.data_ptr()), C.c_void_p(lam.data_ptr()), nbits,
               qs_dtype(psi), x.ctypes.data_as(C.c_void_p), z.ctypes.data_as(C.c_void_p),
               c.ctypes.data_as(C.c_void_p), len(x), st)
        N.call("qs_inner_batched", C.c_void_p(psi.data_ptr()), C.c_void_p(lam.data_ptr()), nbits, qs_dtype(psi),
               n, C.c_void_p(gp.e.data_ptr()), C.c_void_p(gp.ws.data_ptr()), gp.ws.numel(), st)
        cps, npass2, cops, nops, mats, host = gp.bwd
        if gp.pair:
            hp = C.c_void_p(host.ctypes.data) if self.jit else None
            N.call("qs_adjoint_pair_ex", C.c_void_p(gp.pl.data_ptr()), nbits + 1, qs_dtype(psi), cps, npass2, cops,
                   nops, C.c_void_p(mats.data_ptr()), hp, int(mats.numel()),
                   C.c_void_p(gp.partials.data_ptr()), int(gp.partials.numel()), st)
        else:
            N.call("qs_adjoint_fused", C.c_void_p(psi.data_ptr()), C.c_void_p(lam.data_ptr()), nbits,
                   qs_dtype(psi), cps, npass2, cops, nops, C.c_void_p(mats.data_ptr()), int(mats.numel()),
                   C.c_void_p(gp.partials.data_ptr()), int(gp.partials.numel()), st)
        N.call("qs_segment_sum", C.c_void_p(gp.partials.data_ptr()), gp.nslots * bp, gp.tiles_per_inst,
               C.c_void_p(gp.sums.data_ptr()), st)
        self.launches += npass + npass2 + 3
        im = gp.sums.view(gp.nslots, bp, 2)[:, :, 1]
        torch.matmul(gp.weights, im, out=gp.grads)

    def gradient(self, params) -> Tuple[torch.Tensor, torch.Tensor]:
        """(energies (B,), gradients (B, P)) in FP64."""
        gp = self.plan_gradient(params)
        self.launch(gp)
        return gp.e.view(gp.bp, 2)[: gp.b, 0], gp.grads.t()[: gp.b]

    def parameter_shift(self, params, indices: Optional[Sequence[int]] = None) -> torch.Tensor:
        """Gradient by the two-term shift rule (exact for exp(-i theta G / 2), G^2 = I),
        one pair of batched forward runs per parameter occurrence."""
        p, b, bp = self._prepare(params)
        idx = list(range(self.circuit.num_params)) if indices is None else list(indices)
        grads = torch.zeros(b, len(idx), dtype=torch.float64, device=self.dev)
        for col, k in enumerate(idx):
            occ = [i for i in self._param_entries if self.circuit.entries[i].index == k]
            for entry in occ:
                sc = self.circuit.entries[entry].scale
                for sign in (+1, -1):
                    ops = self._shifted_ops(p, entry, sign * np.pi / 2)
                    nbits = self.n + (bp.bit_length() - 1)
                    psi = self._zero_states(bp)
                    self._run(psi, nbits, ops)
                    _, e = self._energy(psi, nbits, bp)
                    grads[:, col] += sign * 0.5 * sc * e[:b]
        return grads

    def _shifted_ops(self, p: np.ndarray, entry: int, shift: float) -> List[Op]:
        ops = []
        for i, op in self._gate_ops(p, False, self._units_plain):
            if i == entry:
                ent = self.circuit.entries[i]
                kind, tab = _batched_rotations(ent.kind, ent.scale * p[:, ent.index] + shift)
                op = Op(op.kind, op.tbits, (), op.mat, tag=op.tag, batch=tab)
            ops.append(op)
        return ops


class GradientPlan:
    """Device buffers and ctypes pass arrays of one planned gradient evaluation."""

    def __init__(self, b: int, bp: int, nbits: int):
        self.b, self.bp, self.nbits = b, bp, nbits

    @property
    def energies(self) -> torch.Tensor:
        return self.e.view(self.bp, 2)[: self.b, 0]

    @property
    def gradients(self) -> torch.Tensor:
        return self.grads.t()[: self.b]


class _ExpectationFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, params, engine):
        e, g = engine.gradient(params)
        g = g.to(params.device)
        ctx.save_for_backward(g)
        return e.to(device=params.device, dtype=params.dtype if params.is_floating_point() else torch.float64)

    @staticmethod
    def backward(ctx, grad_out):
        (g,) = ctx.saved_tensors
        return (grad_out.to(g.dtype)[:, None] * g).to(grad_out.dtype), None


def expectation(params: torch.Tensor, engine: BatchedAdjoint) -> torch.Tensor:
    """Differentiable batch of energies: torch autograd calls the adjoint sweep
    (computed together with the forward pass)."""
    if params.dim() == 1:
        return _ExpectationFn.apply(params[None, :], engine)[0]
    return _ExpectationFn.apply(params, engine)

"""Device engine: runs lowered ops on a torch-owned state through libqsim.

Torch is the allocator and the stream provider; every kernel launch goes
through the C-ABI in ``quict_b200._native``.  There is no CPU path: a missing
CUDA device or library raises.
"""
from __future__ import annotations

import ctypes as C
from collections import OrderedDict
from typing import List, Optional, Sequence

import numpy as np
import torch

from .. import _native as N
from .autotune import Autotuner, Knobs, default_knobs, tune_key
from .fusion import MatrixTable, Pass, Single, emit, fusable, iter_plan, plan, relabel_swaps
from .lowering import Op

DTYPES = {
    np.complex64: (torch.complex64, N.QS_C64, 8),
    np.complex128: (torch.complex128, N.QS_C128, 16),
}


def qs_dtype(t: torch.Tensor) -> int:
    if t.dtype == torch.complex128:
        return N.QS_C128
    if t.dtype == torch.complex64:
        return N.QS_C64
    raise TypeError(f"state must be complex64 or complex128, got {t.dtype}")


def require_cuda(device_id: int = 0) -> torch.device:
    N.load()
    if not torch.cuda.is_available():
        raise RuntimeError("quict_b200 simulators need a CUDA device; none is visible (no CPU fallback)")
    return torch.device("cuda", device_id)


class _Program:
    """Replayable plan of an op sequence: segments ("passes", qs_pass[],
    npass, qs_op[], nops, host table, pinned copy of the table) for runs of
    fused passes and ("single", op) for ops the per-gate kernels apply."""

    def __init__(self, steps, tdtype: torch.dtype):
        npd = np.complex64 if tdtype == torch.complex64 else np.complex128
        self.segments = []
        run: List[Pass] = []

        def flush():
            if run:
                table = MatrixTable()
                cps, npass, cops, nops = emit(run, table)
                host = table.array().astype(npd)
                self.segments.append(("passes", cps, npass, cops, nops, host, torch.from_numpy(host).pin_memory()))
                run.clear()

        for st in steps:
            if isinstance(st, Pass):
                if st.ops:
                    run.append(st)
            else:
                flush()
                self.segments.append(("single", st.op))
        flush()


class Workspace:
    """Grow-only device scratch owned by torch; handed to libqsim as (ptr, bytes)."""

    def __init__(self, device: torch.device):
        self.device = device
        self.buf: Optional[torch.Tensor] = None

    def get(self, nbytes: int) -> torch.Tensor:
        nbytes = max(int(nbytes), 256)
        if self.buf is None or self.buf.numel() < nbytes:
            self.buf = torch.empty(nbytes, dtype=torch.uint8, device=self.device)
        return self.buf


class Engine:
    """Fused-pass knobs left as None are resolved per (dtype, qubit count) from
    the autotuner's cache (``autotune.Autotuner``), else from its defaults."""

    def __init__(self, device: torch.device, fusion: bool = True, tile_bits: Optional[int] = None,
                 low_bits: Optional[int] = None, max_pass_cost: Optional[float] = None,
                 merge_bits: Optional[int] = None, tune_kind: str = "sv", tuner: Optional[Autotuner] = None):
        self.device = device
        self.merge_bits = merge_bits
        self.fusion = fusion
        self.tile_bits = tile_bits
        self.low_bits = low_bits
        self.max_pass_cost = max_pass_cost
        self.tune_kind = tune_kind
        self.tuner = tuner or Autotuner()
        self._resolved = {}  # (element size, n) -> Knobs from the cache / defaults
        self.ws = Workspace(device)
        self.launches = 0  # libqsim kernel launches issued (per gate or per fused pass)
        self.h2d_bytes = 0  # host->device bytes copied for matrix tables
        self.pass_events = None  # list -> record (start, end, nops) CUDA events per fused pass
        # planned programs of recently applied op sequences (see apply_ops)
        self.programs: "OrderedDict[tuple, _Program]" = OrderedDict()
        self.max_programs = 8

    @property
    def stream(self):
        return N.stream_ptr(torch.cuda.current_stream(self.device))

    # ---- per-gate path -------------------------------------------------------------
    def apply_single(self, vec: torch.Tensor, n: int, op: Op):
        dt = qs_dtype(vec)
        ptr = C.c_void_p(vec.data_ptr())
        cmask = 0
        for b in op.cbits:
            cmask |= 1 << b
        st = self.stream
        if op.m >= 3:
            d = op.dense()
            dm = torch.from_numpy(np.ascontiguousarray(d, dtype=np.complex128)).to(self.device, non_blocking=False)
            bits = (C.c_int32 * op.m)(*op.tbits)
            N.call("qs_apply_kq", ptr, n, dt, op.m, bits, cmask, C.c_void_p(dm.data_ptr()), st)
            self._keep = dm
        elif op.m == 1:
            kind = {"mat": N.QS_K_DENSE, "diag": N.QS_K_DIAG, "antidiag": N.QS_K_ANTIDIAG}[op.kind]
            keep, mp = N.mat_ptr(op.dense())
            N.call("qs_apply_1q", ptr, n, dt, op.tbits[0], cmask, kind, mp, st)
        elif op.m == 2:
            kind = {"mat": N.QS_K_DENSE, "diag": N.QS_K_DIAG, "swap": N.QS_K_SWAP}[op.kind]
            keep, mp = N.mat_ptr(op.dense())
            N.call("qs_apply_2q", ptr, n, dt, op.tbits[0], op.tbits[1], cmask, kind, mp, st)
        else:
            raise ValueError(f"cannot apply op kind {op.kind} with {op.m} targets")
        self.launches += 1

    # ---- fused path -------------------------------------------------------------------
    def knobs(self, vec: torch.Tensor, n: int) -> Knobs:
        """Knobs for a run on `vec` (n qubits): explicit settings win, the rest
        come from the tuning cache for this GPU, dtype and size."""
        esize = vec.element_size()
        kn = self._resolved.get((esize, n))
        if kn is None:
            kn = self.tuner.lookup(tune_key(torch.cuda.get_device_name(self.device), esize, n, self.tune_kind))
            kn = kn or default_knobs(esize)
            self._resolved[(esize, n)] = kn
        return Knobs(self.tile_bits if self.tile_bits is not None else kn.tile_bits,
                     self.low_bits if self.low_bits is not None else kn.low_bits,
                     self.merge_bits if self.merge_bits is not None else kn.merge_bits,
                     self.max_pass_cost if self.max_pass_cost is not None else kn.max_pass_cost)

    def tile_shape(self, vec: torch.Tensor, n: int):
        kn = self.knobs(vec, n)
        return kn.tile_bits, kn.low_bits

    def plan_iter(self, vec: torch.Tensor, n: int, ops: Sequence[Op]):
        """Fused-pass steps of `ops`, yielded as they are planned; plain SWAP
        gates become relabellings (``fusion.relabel_swaps``), so the plan moves
        no data for them."""
        kn = self.knobs(vec, n)
        return iter_plan(relabel_swaps(ops, n), n, kn.tile_bits, kn.low_bits, max_cost=kn.max_pass_cost,
                         merge_bits=kn.merge_bits)

    def plan(self, vec: torch.Tensor, n: int, ops: Sequence[Op]):
        return list(self.plan_iter(vec, n, ops))

    def autotune(self, vec: torch.Tensor, n: int, ops: Sequence[Op], force: bool = False):
        """Tune the knobs on `ops` (overwrites `vec`) unless the cache already
        has an entry for this GPU / dtype / size; returns the knobs in use."""
        key = tune_key(torch.cuda.get_device_name(self.device), vec.element_size(), n, self.tune_kind)
        if force or self.tuner.lookup(key) is None:
            self.tuner.tune(self, vec, n, ops, kind=self.tune_kind)
        self._resolved.pop((vec.element_size(), n), None)
        return self.knobs(vec, n)

    def run_passes(self, vec: torch.Tensor, n: int, passes: List[Pass]):
        if not passes:
            return
        table = MatrixTable()
        cps, npass, cops, nops = emit(passes, table)
        host = table.array().astype(np.complex64 if vec.dtype == torch.complex64 else np.complex128)
        # pinned staging: the copy is queued on the stream without blocking the
        # host behind kernels already in flight
        mats = torch.from_numpy(host).pin_memory().to(self.device, non_blocking=True)
        self.h2d_bytes += mats.numel() * mats.element_size()
        hp = C.c_void_p(host.ctypes.data)  # the same table on the host: generated passes take it as parameters
        if self.pass_events is None:
            N.call("qs_apply_fused_ex", C.c_void_p(vec.data_ptr()), n, qs_dtype(vec), cps, npass, cops, nops,
                   C.c_void_p(mats.data_ptr()), hp, int(mats.numel()), self.stream)
        else:
            # one call per pass, bracketed by CUDA events on the launching stream
            stream = torch.cuda.current_stream(self.device)
            for i in range(npass):
                if passes[i].ops:
                    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    a.record(stream)
                N.call("qs_apply_fused_ex", C.c_void_p(vec.data_ptr()), n, qs_dtype(vec), C.byref(cps[i]), 1,
                       cops, nops, C.c_void_p(mats.data_ptr()), hp, int(mats.numel()), self.stream)
                if passes[i].ops:
                    b.record(stream)
                    self.pass_events.append((a, b, len(passes[i].ops)))
        self._keep = mats
        self.launches += sum(1 for p in passes if p.ops)

    def apply_ops(self, vec: torch.Tensor, n: int, ops: Sequence[Op]):
        """Apply unitary ops (no measure/reset/perm) in order.

        The first time an op sequence is applied, each pass is launched as soon
        as it is planned (the GPU works on it while the host plans the next
        one), and the plan is kept as a program: its passes grouped into
        segments with their packed qs_pass / qs_op arrays and matrix tables.
        Applying the same sequence again (same ops and matrices, qubit count,
        precision and knobs) replays the program: one table upload and one
        library call per segment, no lowering or planning."""
        if not self.fusion:
            for op in ops:
                self.apply_single(vec, n, op)
            return
        key = self._program_key(vec, n, ops)
        prog = self.programs.get(key) if key is not None else None
        if prog is not None:
            self.programs.move_to_end(key)
            self._run_program(vec, n, prog)
            return
        steps = []
        for step in self.plan_iter(vec, n, ops):
            if isinstance(step, Pass):
                self.run_passes(vec, n, [step])
            else:
                self.apply_single(vec, n, step.op)
            steps.append(step)
        if key is not None:
            self.programs[key] = _Program(steps, vec.dtype)
            while len(self.programs) > self.max_programs:
                self.programs.popitem(last=False)

    def _program_key(self, vec: torch.Tensor, n: int, ops: Sequence[Op]):
        """Exact key of an op sequence (None: not kept, e.g. batched or tagged ops)."""
        if not ops:
            return None
        parts = [n, str(vec.dtype), self.knobs(vec, n)]
        for op in ops:
            if op.batch is not None or op.tag is not None or op.kind not in ("mat", "diag", "antidiag", "swap"):
                return None
            parts.append((op.kind, op.tbits, op.cbits, op.mat.tobytes()))
        return tuple(parts)

    def _run_program(self, vec: torch.Tensor, n: int, prog: "_Program"):
        st = self.stream
        for seg in prog.segments:
            if seg[0] == "single":
                self.apply_single(vec, n, seg[1])
                continue
            _, cps, npass, cops, nops, host, pinned = seg
            mats = torch.empty(pinned.shape, dtype=pinned.dtype, device=self.device)
            mats.copy_(pinned, non_blocking=True)
            self.h2d_bytes += mats.numel() * mats.element_size()
            N.call("qs_apply_fused_ex", C.c_void_p(vec.data_ptr()), n, qs_dtype(vec), cps, npass, cops, nops,
                   C.c_void_p(mats.data_ptr()), C.c_void_p(host.ctypes.data), int(mats.numel()), st)
            self.launches += npass
            self._keep = mats

    # ---- reductions / measurement -------------------------------------------------------
    def prob0(self, src: torch.Tensor, n: int, bit: int, src_kind: int = N.QS_SRC_SV) -> float:
        ws = self.ws.get(N.load().qs_reduce_ws_bytes(n))
        res = torch.empty(1, dtype=torch.float64, device=self.device)
        N.call("qs_prob0", C.c_void_p(src.data_ptr()), n, qs_dtype(src), src_kind, bit,
               C.c_void_p(ws.data_ptr()), ws.numel(), C.c_void_p(res.data_ptr()), self.stream)
        return float(res.item())

    def norm2(self, src: torch.Tensor, n: int, src_kind: int = N.QS_SRC_SV) -> float:
        ws = self.ws.get(N.load().qs_reduce_ws_bytes(n))
        res = torch.empty(1, dtype=torch.float64, device=self.device)
        N.call("qs_norm2", C.c_void_p(src.data_ptr()), n, qs_dtype(src), src_kind,
               C.c_void_p(ws.data_ptr()), ws.numel(), C.c_void_p(res.data_ptr()), self.stream)
        return float(res.item())

    def collapse(self, vec: torch.Tensor, n: int, bit: int, outcome: int, scale: float):
        N.call("qs_collapse", C.c_void_p(vec.data_ptr()), n, qs_dtype(vec), bit, int(outcome), float(scale),
               self.stream)

    def reset(self, vec: torch.Tensor, n: int, bit: int, p0: float):
        N.call("qs_reset", C.c_void_p(vec.data_ptr()), n, qs_dtype(vec), bit, float(p0), self.stream)

    def sample_indices(self, src: torch.Tensor, n: int, uniforms: torch.Tensor, mode: int,
                       src_kind: int = N.QS_SRC_SV) -> torch.Tensor:
        """Device int64 tensor of sampled basis indices (one per shot)."""
        lib = N.load()
        wsb = lib.qs_sample_ws_bytes(n)
        ws = self.ws.get(wsb)
        u = uniforms.to(device=self.device, dtype=torch.float64).contiguous()
        shots = u.numel() if mode == N.QS_SAMPLE_CDF else u.numel() // n
        out = torch.empty(max(shots, 1), dtype=torch.int64, device=self.device)
        st = self.stream
        N.call("qs_sample_prepare", C.c_void_p(src.data_ptr()), n, qs_dtype(src), src_kind,
               C.c_void_p(ws.data_ptr()), ws.numel(), st)
        N.call("qs_sample", C.c_void_p(src.data_ptr()), n, qs_dtype(src), src_kind, C.c_void_p(ws.data_ptr()),
               ws.numel(), C.c_void_p(u.data_ptr()), shots, mode, C.c_void_p(out.data_ptr()), st)
        return out[:shots]

    def histogram(self, idx: torch.Tensor, ncounts: int) -> torch.Tensor:
        counts = torch.zeros(ncounts, dtype=torch.int64, device=self.device)
        N.call("qs_histogram", C.c_void_p(idx.data_ptr()), idx.numel(), C.c_void_p(counts.data_ptr()), ncounts,
               self.stream)
        return counts

    def counts_list(self, idx: torch.Tensor, ncounts: int) -> list:
        """Histogram of sample indices as a Python list of length `ncounts`.
        With few shots per bin only the nonzero bins cross to the host, and the
        list is a zero list with those entries set (a full ``tolist`` of 2^20
        counts costs several ms)."""
        counts = self.histogram(idx, ncounts)
        if ncounts <= 4 * idx.numel():
            return counts.cpu().numpy().tolist()
        nz = torch.nonzero(counts).flatten()
        where, vals = nz.cpu().tolist(), counts[nz].cpu().tolist()
        out = [0] * ncounts
        for i, c in zip(where, vals):
            out[i] = c
        return out

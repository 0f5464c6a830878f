"""Many gradient problems in ONE persistent kernel launch.

``PersistentBatch`` takes problems of uneven size -- each an n-qubit
``BatchedAdjoint`` engine (circuit + observable) and one parameter row -- and
plans them all into one work list for ``qs_batch_launch``: per problem, its
forward register passes (the first starts from |0...0>), lam = H psi with the
energy, its adjoint pair passes and a final reduction to the energy and the
gradient.  Persistent CTAs take the work items in list order; an item waits
(bounded) until its problem's earlier stages are done, so small and large
problems share the GPU without one launch per pass.  A replay is a control-
word memset plus the kernel, and can be captured in a CUDA graph.

The tile widths (forward, pair) are capped per batch; ``tune`` times the
candidate caps on the batch itself and keeps the fastest (the autotuner cache
stores it under kind "batch").
"""
from __future__ import annotations

import ctypes as C
from typing import List, Optional, Sequence, Tuple

import numpy as np
import torch

from .. import _native as N
from ..simulation.autotune import Autotuner, tune_key
from ..simulation.engine import require_cuda
from ..simulation.fusion import MatrixTable, Pass, emit, plan
from ..simulation.lowering import Op, classify
from .adjoint import BatchedAdjoint

# (forward cap, pair cap) candidates of ``PersistentBatch.tune``, by precision
CAP_CANDIDATES = {
    "single": [(13, 13), (12, 12), (12, 13), (11, 12)],
    "double": [(11, 11), (11, 12), (10, 11), (12, 12), (10, 10)],
}
DEFAULT_CAPS = {"single": (13, 13), "double": (11, 11)}  # measured on the 512-instance QAOA batch (B200)


def _min_k(precision: str) -> int:
    """Smallest register tile: 2^(R + 5) amplitudes (R = 4 / 5 register bits)."""
    return 9 if precision == "double" else 10


class PersistentBatch:
    """problems: [(engine, params)] with params one row of the engine's
    circuit parameters.  Every engine must have the batch's precision and
    device, n >= 10 (complex64) / 9 (complex128) qubits, and a circuit whose
    units act densely on at most 2 qubits (the pair-pass rule)."""

    def __init__(self, problems: Sequence[Tuple[BatchedAdjoint, np.ndarray]], precision: str = "single",
                 device_id: int = 0, caps: Optional[Tuple[int, int]] = None, tiles_per_item: int = 16,
                 amps_per_ham_item: int = 1 << 14, timeout_s: float = 10.0, jit_min_qubits: int = 20):
        if not problems:
            raise ValueError("an empty batch")
        self.dev = require_cuda(device_id)
        self.precision = precision
        self.caps = tuple(caps or DEFAULT_CAPS[precision])
        self.timeout_s = float(timeout_s)
        self.dtype = N.QS_C64 if precision == "single" else N.QS_C128
        self.cdtype = torch.complex64 if precision == "single" else torch.complex128
        np_dtype = np.complex64 if precision == "single" else np.complex128
        min_k = _min_k(precision)
        table = MatrixTable()
        passes: List[N.qs_pass] = []
        ops: List[N.qs_op] = []
        insts = (N.qs_batch_inst * len(problems))()
        xs, zs, cs, ws = [], [], [], []
        self.nparams: List[int] = []
        for i, (eng, prm) in enumerate(problems):
            if eng.cdtype != self.cdtype:
                raise ValueError(f"problem {i}: precision differs from the batch's")
            n = eng.n
            if n < min_k:
                raise ValueError(f"problem {i}: {n} qubits; the batch kernel needs >= {min_k}")
            if not all(len(u.qubits) <= 2 or classify(u.gen if u.fixed is None else u.fixed) == "diag"
                       for u in eng._units):
                raise ValueError(f"problem {i}: a unit acts densely on more than 2 qubits")
            p = np.atleast_2d(np.asarray(prm, dtype=np.float64))
            if p.shape[0] != 1:
                raise ValueError(f"problem {i}: one parameter row per problem")
            fwd_ops, bwd_ops, nslots, w = eng.sweep_ops(p)
            bwd_ops = [Op(o.kind, o.tbits, o.cbits, o.mat, tag=o.tag, batch=o.batch, slot=o.slot, extra=(n,))
                       if o.kind == "expect" else o for o in bwd_ops]
            kf = max(min_k, min(self.caps[0], n))
            kb = max(min_k, min(self.caps[1], n + 1))
            q = insts[i]
            q.n = n
            for d, (oplist, nbits, k, adj) in enumerate(((fwd_ops, n, kf, False), (bwd_ops, n + 1, kb, True))):
                steps = plan(oplist, nbits, k, min(5, k), merge_bits=0 if adj else 2)
                ps = [s for s in steps if isinstance(s, Pass)]
                if len(ps) != len(steps):
                    raise RuntimeError(f"problem {i}: an op could not be fused")
                cps, npass, cops, nops = emit(ps, table, inst_shift=n, pair=n if adj else None)
                begin = len(passes)
                for j in range(npass):
                    cp = cps[j]
                    cp.op_begin += len(ops)
                    passes.append(cp)
                for j in range(nops):
                    ops.append(cops[j])
                if adj:
                    q.bwd_begin, q.nbwd = begin, npass
                else:
                    q.fwd_begin, q.nfwd = begin, npass
            x, z, c = eng.pauli
            q.term_begin, q.nterms = len(xs), len(x)
            xs += list(x)
            zs += list(z)
            cs += list(c)
            q.nslots = nslots
            q.nparams = w.shape[0]
            q.w_begin = len(ws)
            ws += list(w.ravel())
            self.nparams.append(w.shape[0])
        self.npasses = len(passes)
        cpass = (N.qs_pass * len(passes))(*passes)
        cop = (N.qs_op * len(ops))(*ops)
        host = table.array().astype(np_dtype)
        xa = np.array(xs, dtype=np.uint64)
        za = np.array(zs, dtype=np.uint64)
        ca = np.array(cs, dtype=np.float64)
        wa = np.array(ws if ws else [0.0], dtype=np.float64)
        sizes = N.qs_batch_sizes()
        offs = (C.c_int64 * len(problems))()
        self.jit_min_qubits = jit_min_qubits
        args = (self.dtype, insts, len(problems), cpass, len(passes), cop, len(ops), host.size,
                C.c_void_p(host.ctypes.data) if host.size else None, int(jit_min_qubits),
                xa.ctypes.data_as(C.c_void_p), za.ctypes.data_as(C.c_void_p), ca.ctypes.data_as(C.c_void_p), len(xa),
                wa.ctypes.data_as(C.c_void_p), len(ws), int(tiles_per_item), int(amps_per_ham_item))
        N.call("qs_batch_plan", *args, None, 0, C.byref(sizes), offs)
        blob = np.zeros(int(sizes.blob_bytes), dtype=np.uint8)
        N.call("qs_batch_plan", *args, blob.ctypes.data_as(C.c_void_p), blob.nbytes, C.byref(sizes), offs)
        self.sizes = sizes
        self.state_off = [int(v) for v in offs]
        self.ns = [eng.n for eng, _ in problems]
        dev = self.dev
        # device buffers, owned here (the library allocates nothing)
        self.blob = torch.from_numpy(blob).to(dev)
        self.mats = torch.from_numpy(host if host.size else np.zeros(1, np_dtype)).to(dev)
        self.states = torch.empty(int(sizes.state_elems), dtype=self.cdtype, device=dev)
        self.partials = torch.empty(int(sizes.partial_doubles), dtype=torch.float64, device=dev)
        self.energies = torch.empty(int(sizes.energy_doubles), dtype=torch.float64, device=dev)
        self.grads = torch.empty(int(sizes.grad_doubles), dtype=torch.float64, device=dev)
        self.ctrl = torch.zeros(int(sizes.ctrl_bytes) // 8, dtype=torch.int64, device=dev)
        self.graph = None
        self.launches = 0
        self.linked = False

    # ---- running -------------------------------------------------------------------
    def launch(self, stream=None) -> bool:
        """Issue the batch (control-word memset + one kernel) on `stream`;
        True when the kernel linked with the generated stage functions ran,
        False for the generic one."""
        st = N.stream_ptr(stream if stream is not None else torch.cuda.current_stream(self.dev))
        rc = N.call("qs_batch_launch", C.byref(self.sizes), C.c_void_p(self.blob.data_ptr()),
               C.c_void_p(self.states.data_ptr()), C.c_void_p(self.mats.data_ptr()),
               C.c_void_p(self.partials.data_ptr()), C.c_void_p(self.energies.data_ptr()),
               C.c_void_p(self.grads.data_ptr()), C.c_void_p(self.ctrl.data_ptr()), self.ctrl.numel() * 8,
               self.timeout_s, st)
        self.launches += 1
        self.linked = rc == 1
        return self.linked

    def capture(self) -> "torch.cuda.CUDAGraph":
        """Eager runs first (the generated stage functions finish compiling
        and the linked kernel is loaded outside capture), then the launch
        captured into a CUDA graph."""
        self.launch()
        if self.sizes.jit_fns > 0:
            N.jit_wait(1800)
            self.launch()
        torch.cuda.synchronize(self.dev)
        self.check()
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph):
            self.launch()
        return self.graph

    def replay(self) -> None:
        if self.graph is None:
            self.capture()
        self.graph.replay()

    def check(self) -> None:
        """Raise if the last run's bounded waits gave up (control word 1)."""
        err = int(self.ctrl[1].item())
        if err != 0:
            raise N.QsimError("qs_batch_launch", N.QS_ETIMEOUT,
                              f"work item {err & 0xffffffff} waited longer than {self.timeout_s} s")

    def results(self) -> List[Tuple[float, np.ndarray]]:
        """[(energy, gradient)] per problem (host copies), after checking the
        control word."""
        torch.cuda.synchronize(self.dev)
        self.check()
        e = self.energies.view(-1, 2)[:, 0].cpu().numpy()
        g = self.grads.cpu().numpy()
        out, at = [], 0
        for i, k in enumerate(self.nparams):
            out.append((float(e[i]), g[at:at + k].copy()))
            at += k
        return out

    def state(self, i: int) -> torch.Tensor:
        """psi of problem i after the last run (the backward sweep runs psi
        back to |0...0>, so this is the state the sweep ended on)."""
        return self.states[self.state_off[i]:self.state_off[i] + (1 << self.ns[i])]


def tune(make_batch, precision: str, key: Optional[str] = None, tuner: Optional[Autotuner] = None,
         reps: int = 3, store: bool = True):
    """Time `make_batch(caps)` for every candidate cap pair and return
    (best caps, ms, trials); stored under `key` (kind "batch") when given."""
    import math
    import time as _time
    tuner = tuner or Autotuner()
    trials = {}
    best, best_ms = None, math.inf
    for caps in CAP_CANDIDATES[precision]:
        b = make_batch(caps)
        b.capture()  # compiles and links the generated stage functions, if any
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        for _ in range(reps):
            b.launch()
        e.record()
        torch.cuda.synchronize(b.dev)
        b.check()
        t = s.elapsed_time(e) / reps
        trials[f"caps={caps[0]},{caps[1]}"] = t
        if t < best_ms:
            best, best_ms = caps, t
        del b
        torch.cuda.empty_cache()
    if store and key is not None:
        import json
        import os
        from ..simulation.autotune import _load
        d = _load(tuner.cache_path)
        d[key] = {"knobs": {"tile_bits": best[0], "pair_tile_bits": best[1]}, "ms": best_ms, "trials": trials,
                  "when": _time.strftime("%Y-%m-%dT%H:%M:%SZ", _time.gmtime())}
        os.makedirs(os.path.dirname(os.path.abspath(tuner.cache_path)), exist_ok=True)
        tmp = tuner.cache_path + ".tmp"
        with open(tmp, "w") as f:
            json.dump(d, f, indent=1, sort_keys=True)
        os.replace(tmp, tuner.cache_path)
    return best, best_ms, trials


def batch_key(device_name: str, precision: str, label: str) -> str:
    """Autotuner key of a persistent batch workload (e.g. label "qaoa512")."""
    return tune_key(device_name, 8 if precision == "single" else 16, 0, f"batch-{label}")

"""Uneven-size batched QAOA MaxCut: energies and adjoint gradients of many
instances with different qubit counts, graphs and depths, replayed as ONE
CUDA-graph launch.

Every instance is planned once on the host (``BatchedAdjoint.plan_gradient``:
gate tables, fused-pass plans, device buffers).  Its kernel chain (forward
passes, lam = C psi, FP64 energy, adjoint sweep, partial sums) is then
captured into one graph.  Instances are spread over several capture streams,
so their chains are independent branches that the GPU runs concurrently:
small instances (2^10 amplitudes = one tile) fill the SMs side by side, and
large ones (2^24) use the whole GPU.
"""
from __future__ import annotations

from typing import List, Optional, Sequence, Tuple

import numpy as np
import torch

from ..simulation.autotune import Autotuner, tune_key
from .adjoint import BatchedAdjoint, GradientPlan
from .circuit import maxcut_observable, qaoa_circuit, random_regular_graph


def qaoa_instances(count: int = 512, sizes: Sequence[int] = tuple(range(10, 25, 2)), depths=(1, 6),
                   seed: int = 4) -> List[Tuple[int, List[Tuple[int, int]], int, np.ndarray]]:
    """Seeded (n, edges, p, params) tuples: n uniform over `sizes`, p uniform in
    depths, a random 3-regular graph, gammas and betas uniform in [0, pi)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        n = int(sizes[rng.integers(len(sizes))])
        p = int(rng.integers(depths[0], depths[1] + 1))
        edges = random_regular_graph(n, 3, rng)
        params = rng.uniform(0, np.pi, 2 * p)
        out.append((n, edges, p, params))
    return out


def _tile_maker(n, edges, p, precision, device_id, jit):
    def make(fk, pk):
        return BatchedAdjoint(qaoa_circuit(n, edges, p), maxcut_observable(n, edges), precision, device_id,
                              tile_bits=fk, pair_tile_bits=pk, jit=jit)
    make.precision, make.n = precision, n
    return make


def tune_qaoa_size(tuner: Autotuner, n: int, precision: str, device_id: int = 0, seed: int = 11):
    """Tune the forward / pair tile widths of n-qubit MaxCut QAOA gradients
    (a seeded depth-6 instance) and store them under kind "qaoa"."""
    (nn, edges, p, prm), = qaoa_instances(1, sizes=(n,), depths=(6, 6), seed=seed)
    dev = torch.device("cuda", device_id)
    key = tune_key(torch.cuda.get_device_name(dev), 8 if precision == "single" else 16, n, "qaoa")
    return tuner.tune_adjoint(_tile_maker(n, edges, p, precision, device_id, True), np.asarray(prm)[None, :], key)


class UnevenQAOABatch:
    """Two ways to run the batch:

    mode="persistent": every instance's whole gradient (forward passes,
      lam = C psi and the energy, adjoint sweep, final sums) is planned into
      the work list of ONE persistent kernel launch (``PersistentBatch``);
      a replay is a control-word memset plus that launch.  `caps` (forward,
      pair tile-width caps) come from the autotuner's "batch" entry for this
      workload, else the defaults; ``tune_caps`` measures them.
    mode="graph": each instance runs its own kernel chain; the chains are
      captured over several streams into one CUDA graph.  `jit_min_qubits`:
      instances of at least that many qubits run their register passes as
      run-time compiled kernels (their kernels dominate the replay); smaller
      ones keep the generic kernels, whose per-instance compilation would not
      pay off.  Tile widths come per qubit count from the autotuner's "qaoa"
      entries (`autotune=True` tunes sizes it has none for, on the first
      instance of that size)."""

    def __init__(self, instances, precision: str = "single", device_id: int = 0, streams: int = 16,
                 jit_min_qubits: int = 22, autotune: bool = False, tuner: Optional[Autotuner] = None,
                 mode: str = "graph", caps: Optional[Tuple[int, int]] = None, label: Optional[str] = None):
        if mode not in ("graph", "persistent"):
            raise ValueError(f"mode must be 'graph' or 'persistent', not {mode!r}")
        self.instances = instances
        self.mode = mode
        self.jit_min_qubits = jit_min_qubits
        self.captured_launches = 0
        self.graph = None
        if mode == "persistent":
            from .persistent import PersistentBatch, batch_key
            tuner = tuner or Autotuner()
            dev = torch.device("cuda", device_id)
            self.caps = caps
            if self.caps is None and label is not None:
                self.caps = tuner.lookup_adjoint(batch_key(torch.cuda.get_device_name(dev), precision, label))
            self.engines = [BatchedAdjoint(qaoa_circuit(n, edges, p), maxcut_observable(n, edges), precision,
                                           device_id) for n, edges, p, _ in instances]
            self.persistent = PersistentBatch([(e, np.asarray(prm)) for e, (_, _, _, prm) in
                                               zip(self.engines, instances)], precision, device_id, caps=self.caps,
                                              jit_min_qubits=jit_min_qubits)
            self.caps = self.persistent.caps
            self.dev = self.persistent.dev
            return
        tuner = tuner or Autotuner()
        dev = torch.device("cuda", device_id)
        esize = 8 if precision == "single" else 16
        self.tiles = {}  # n -> (forward tile bits, pair tile bits) or None (engine defaults)
        for n, edges, p, prm in instances:
            if n in self.tiles:
                continue
            key = tune_key(torch.cuda.get_device_name(dev), esize, n, "qaoa")
            kn = tuner.lookup_adjoint(key)
            if kn is None and autotune:
                kn, _, _ = tuner.tune_adjoint(_tile_maker(n, edges, p, precision, device_id, n >= jit_min_qubits),
                                              np.asarray(prm)[None, :], key)
            self.tiles[n] = kn
        self.engines = [BatchedAdjoint(qaoa_circuit(n, edges, p), maxcut_observable(n, edges), precision, device_id,
                                       tile_bits=self.tiles[n][0] if self.tiles[n] else None,
                                       pair_tile_bits=self.tiles[n][1] if self.tiles[n] else None,
                                       jit=n >= jit_min_qubits)
                        for n, edges, p, _ in instances]
        self.captured_launches = 0  # kernel launches recorded in the graph
        self.plans: List[GradientPlan] = [eng.plan_gradient(np.asarray(prm)[None, :])
                                          for eng, (_, _, _, prm) in zip(self.engines, instances)]
        self.dev = self.engines[0].dev if self.engines else torch.device("cuda", device_id)
        self.nstreams = streams
        self.graph = None

    def tune_caps(self, label: str, tuner: Optional[Autotuner] = None):
        """Persistent mode: time every tile-width cap candidate on this batch,
        store the fastest under the "batch" key of `label` and rebuild the
        batch with it; returns (caps, ms, trials)."""
        from .persistent import PersistentBatch, batch_key, tune
        if self.mode != "persistent":
            raise ValueError("tune_caps applies to mode='persistent'")
        prec = self.persistent.precision
        probs = [(e, np.asarray(prm)) for e, (_, _, _, prm) in zip(self.engines, self.instances)]
        key = batch_key(torch.cuda.get_device_name(self.dev), prec, label)
        self.persistent = None
        jm = self.jit_min_qubits
        best, ms, trials = tune(lambda caps: PersistentBatch(probs, prec, self.dev.index, caps=caps,
                                                             jit_min_qubits=jm), prec, key, tuner)
        self.persistent = PersistentBatch(probs, prec, self.dev.index, caps=best, jit_min_qubits=jm)
        self.caps = best
        self.graph = None
        return best, ms, trials

    @property
    def num_gradients(self) -> int:
        return sum(2 * p for _, _, p, _ in self.instances)

    def _launch_all(self, streams):
        cur = torch.cuda.current_stream(self.dev)
        for s in streams:
            s.wait_stream(cur)
        # largest instances first so they start early
        order = sorted(range(len(self.plans)), key=lambda i: -self.instances[i][0])
        for j, i in enumerate(order):
            st = streams[j % len(streams)]
            with torch.cuda.stream(st):
                self.engines[i].launch(self.plans[i], st)
        for s in streams:
            cur.wait_stream(s)

    def run_eager(self):
        streams = [torch.cuda.Stream(self.dev) for _ in range(self.nstreams)]
        self._launch_all(streams)

    def capture(self):
        """Warm up (first-launch configuration and the compilation of the
        generated pass kernels happen outside capture), then capture every
        instance's chain (mode "graph") or the persistent launch into one
        CUDA graph."""
        from .. import _native as N
        if self.mode == "persistent":
            self.graph = self.persistent.capture()
            self.captured_launches = 1  # the kernel (plus a memset node of the control words)
            return self.graph
        self.run_eager()
        N.jit_wait(900)
        self.run_eager()  # loads the compiled kernels on this device
        torch.cuda.synchronize(self.dev)
        self.graph = torch.cuda.CUDAGraph()
        streams = [torch.cuda.Stream(self.dev) for _ in range(self.nstreams)]
        before = sum(e.launches for e in self.engines)
        with torch.cuda.graph(self.graph):
            self._launch_all(streams)
        self.captured_launches = sum(e.launches for e in self.engines) - before
        return self.graph

    def replay(self):
        if self.graph is None:
            self.capture()
        self.graph.replay()

    def results(self) -> List[Tuple[float, np.ndarray]]:
        """[(energy, gradient (2p,))] per instance (host copies)."""
        if self.mode == "persistent":
            return self.persistent.results()
        out = []
        for gp in self.plans:
            out.append((float(gp.energies[0]), gp.gradients[0].cpu().numpy()))
        return out

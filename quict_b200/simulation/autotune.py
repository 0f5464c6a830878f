"""Autotuner for the fused-pass knobs (tile shape, gate-merging width, pass cost bound).

The knobs of a fused run are

  * ``tile_bits`` (k): amplitudes per on-chip tile, 2^k;
  * ``low_bits`` (nlow): how many of them are the contiguous low vector bits;
  * ``merge_bits``: widest block runs of gates are multiplied into (0 = off);
  * ``max_pass_cost``: bound on a pass's arithmetic (inf = fuse as much as fits).

They are chosen per (GPU model, complex dtype, qubit count, workload kind) by
timing candidate settings on the caller's own circuit and state buffer, with
successive halving: every candidate runs a prefix of the circuit, the best few
run it whole, and the fastest is stored in a JSON cache.  Lookups read the
user cache first (``QUICT_B200_TUNE_CACHE`` or ``~/.cache/quict_b200/tune.json``)
and then the table shipped with the package (``tuned_b200.json``, produced by
``python -m quict_b200.simulation.autotune`` on a B200).

QuICT has no tuner: its GPU simulator launches one fixed-shape kernel per gate
(QuICT/simulation/state_vector/statevector_simulator.py:155-164).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import time
from dataclasses import asdict, dataclass, field
from typing import Callable, Dict, List, Optional, Sequence, Tuple

PACKAGED = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tuned_b200.json")

# register-kernel tile widths per element size: 2^R amplitudes per thread and
# 64..256 threads per tile (tile_bits = R + 6 .. R + 8); narrower tiles run
# several CTAs per SM.  k = R + 8 is the default when the cache has no entry.
_TILE_CHOICES = {16: (10, 11, 12), 8: (11, 12, 13)}


@dataclass(frozen=True)
class Knobs:
    tile_bits: int
    low_bits: int
    merge_bits: int
    max_pass_cost: float = math.inf

    def to_json(self) -> dict:
        d = asdict(self)
        d["max_pass_cost"] = None if math.isinf(self.max_pass_cost) else self.max_pass_cost
        return d

    @staticmethod
    def from_json(d: dict) -> "Knobs":
        c = d.get("max_pass_cost")
        return Knobs(int(d["tile_bits"]), int(d["low_bits"]), int(d["merge_bits"]),
                     math.inf if c is None else float(c))


def default_knobs(esize: int) -> Knobs:
    """Settings used when the cache has no entry (k = 12 / 13, 32-amplitude runs, 2-bit merging)."""
    return Knobs(12 if esize == 16 else 13, 5, 2)


def candidates(esize: int, n: int) -> List[Knobs]:
    out = []
    for k in _TILE_CHOICES[esize]:
        for nlow in (5, 6):
            for mb in (0, 2, 3):
                if k <= n and nlow <= k:
                    out.append(Knobs(k, nlow, mb))
    return out


def adjoint_candidates(precision: str, n: int) -> List[Tuple[int, int]]:
    """(forward tile bits, pair tile bits) for an n-qubit adjoint gradient: the
    register tiles from the smallest (64-thread CTAs) to 64 KiB; a pair tile
    holds the psi/lam bit besides n qubit bits."""
    k0 = 12 if precision == "double" else 13
    min_k = 9 if precision == "double" else 10
    fwd = sorted({k for k in (min_k, min_k + 1, k0 - 1) if k <= n}) or [min(min_k, n)]
    pair = [k for k in range(min_k, k0 + 1) if k <= n + 1]
    return [(f, p) for f in fwd for p in pair]


def tune_key(device_name: str, esize: int, n: int, kind: str) -> str:
    return f"{device_name}|{'c128' if esize == 16 else 'c64'}|n{n}|{kind}"


def user_cache_path() -> str:
    return os.environ.get("QUICT_B200_TUNE_CACHE") or os.path.join(
        os.path.expanduser("~"), ".cache", "quict_b200", "tune.json")


def _load(path: str) -> Dict[str, dict]:
    try:
        with open(path) as f:
            d = json.load(f)
        return d if isinstance(d, dict) else {}
    except (OSError, ValueError):
        return {}


@dataclass
class TuneResult:
    knobs: Knobs
    ms: float
    trials: Dict[str, float] = field(default_factory=dict)


class Autotuner:
    def __init__(self, cache_path: Optional[str] = None, packaged_path: str = PACKAGED):
        self.cache_path = cache_path or user_cache_path()
        self.packaged_path = packaged_path

    # ---- cache -------------------------------------------------------------------
    def lookup(self, key: str) -> Optional[Knobs]:
        for path in (self.cache_path, self.packaged_path):
            e = _load(path).get(key)
            if e is not None:
                return Knobs.from_json(e["knobs"])
        return None

    def store(self, key: str, res: TuneResult, path: Optional[str] = None) -> None:
        path = path or self.cache_path
        d = _load(path)
        d[key] = {"knobs": res.knobs.to_json(), "ms": res.ms, "trials": res.trials,
                  "when": time.strftime("%Y-%m-%dT%H:%M:%SZ", time.gmtime())}
        os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
        tmp = path + ".tmp"
        with open(tmp, "w") as f:
            json.dump(d, f, indent=1, sort_keys=True)
        os.replace(tmp, path)

    def lookup_adjoint(self, key: str) -> Optional[Tuple[int, int]]:
        """(forward tile bits, pair tile bits) of an adjoint-gradient entry."""
        for path in (self.cache_path, self.packaged_path):
            e = _load(path).get(key)
            if e is not None and "pair_tile_bits" in e.get("knobs", {}):
                return int(e["knobs"]["tile_bits"]), int(e["knobs"]["pair_tile_bits"])
        return None

    def tune_adjoint(self, make_engine: Callable[[int, int], object], params, key: str, reps: int = 3,
                     store: bool = True) -> Tuple[Tuple[int, int], float, Dict[str, float]]:
        """Time every (forward tile, pair tile) candidate of an adjoint
        gradient on `params` (``adjoint_candidates``), each after its generated
        kernels are compiled; store and return the fastest."""
        import torch

        from .. import _native as N
        trials: Dict[str, float] = {}
        best, best_ms = None, math.inf
        for fk, pk in adjoint_candidates(make_engine.precision, make_engine.n):
            eng = make_engine(fk, pk)
            gp = eng.plan_gradient(params)
            eng.launch(gp)
            N.jit_wait(600)
            eng.launch(gp)
            torch.cuda.synchronize(eng.dev)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            for _ in range(reps):
                eng.launch(gp)
            b.record()
            torch.cuda.synchronize(eng.dev)
            t = a.elapsed_time(b) / reps
            trials[f"tile_bits={fk} pair_tile_bits={pk}"] = t
            if t < best_ms:
                best, best_ms = (fk, pk), t
            del gp, eng
        if store:
            d = _load(self.cache_path)
            d[key] = {"knobs": {"tile_bits": best[0], "pair_tile_bits": best[1]}, "ms": best_ms, "trials": trials,
                      "when": time.strftime("%Y-%m-%dT%H:%M:%SZ", time.gmtime())}
            os.makedirs(os.path.dirname(os.path.abspath(self.cache_path)), exist_ok=True)
            tmp = self.cache_path + ".tmp"
            with open(tmp, "w") as f:
                json.dump(d, f, indent=1, sort_keys=True)
            os.replace(tmp, self.cache_path)
        return best, best_ms, trials

    # ---- search ------------------------------------------------------------------
    @staticmethod
    def search(cands: Sequence[Knobs], time_prefix: Callable[[Knobs], float],
               time_full: Callable[[Knobs], float], keep: int = 3) -> TuneResult:
        """Successive halving: all candidates on the prefix, the best `keep` on the whole."""
        trials: Dict[str, float] = {}
        scored = []
        for kn in cands:
            t = time_prefix(kn)
            trials[f"prefix {kn.to_json()}"] = t
            scored.append((t, kn))
        scored.sort(key=lambda z: z[0])
        best, best_ms = None, math.inf
        for _, kn in scored[:keep]:
            t = time_full(kn)
            trials[f"full {kn.to_json()}"] = t
            if t < best_ms:
                best, best_ms = kn, t
        return TuneResult(best, best_ms, trials)

    def tune(self, engine, vec, n: int, ops, kind: str = "sv", prefix_ops: int = 250, reps: int = 2,
             store: bool = True) -> TuneResult:
        """Time the candidates on `ops` with `engine` on the buffer `vec` (its
        contents are overwritten: every trial starts from |0...0>)."""
        import torch

        from .. import _native as N
        from .engine import qs_dtype

        esize = vec.element_size()
        dev = vec.device
        saved = (engine.tile_bits, engine.low_bits, engine.merge_bits, engine.max_pass_cost)

        def timed(kn: Knobs, seq) -> float:
            engine.tile_bits, engine.low_bits = kn.tile_bits, kn.low_bits
            engine.merge_bits, engine.max_pass_cost = kn.merge_bits, kn.max_pass_cost

            def once():
                N.call("qs_init_zero", vec.data_ptr(), n, qs_dtype(vec), engine.stream)
                engine.apply_ops(vec, n, seq)

            once()
            N.jit_wait(600)  # the candidate's passes run compiled when they are timed
            once()
            torch.cuda.synchronize(dev)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            for _ in range(reps):
                once()
            b.record()
            torch.cuda.synchronize(dev)
            return a.elapsed_time(b) / reps

        prefix = list(ops)[:prefix_ops]
        try:
            res = self.search(candidates(esize, n), lambda kn: timed(kn, prefix), lambda kn: timed(kn, ops))
        finally:
            engine.tile_bits, engine.low_bits, engine.merge_bits, engine.max_pass_cost = saved
        if store:
            self.store(tune_key(torch.cuda.get_device_name(dev), esize, n, kind), res)
        return res


def main() -> None:
    """Tune the seeded random-circuit workloads and write the results to a cache file."""
    import torch

    from ..workloads import spread_circuit
    from .engine import Engine
    from .lowering import lower_circuit

    ap = argparse.ArgumentParser()
    ap.add_argument("--qubits", type=int, nargs="+", default=[30])
    ap.add_argument("--precision", nargs="+", default=["double", "single"])
    ap.add_argument("--gates", type=int, default=1000)
    ap.add_argument("--out", default=None, help="cache file (default: the user cache)")
    ap.add_argument("--qaoa", action="store_true",
                    help="tune the adjoint-gradient tiles of seeded MaxCut QAOA instances (depth 6) instead")
    a = ap.parse_args()
    dev = torch.device("cuda", 0)
    tuner = Autotuner(cache_path=a.out)
    if a.qaoa:
        from ..differentiation.qaoa import tune_qaoa_size
        for n in a.qubits:
            for prec in a.precision:
                (fk, pk), ms, _ = tune_qaoa_size(tuner, n, prec)
                print(json.dumps({"n": n, "precision": prec, "tile_bits": fk, "pair_tile_bits": pk, "ms": ms}),
                      flush=True)
        return
    for n in a.qubits:
        for prec in a.precision:
            dt = torch.complex128 if prec == "double" else torch.complex64
            vec = torch.empty(1 << n, dtype=dt, device=dev)
            eng = Engine(dev)
            ops = lower_circuit(spread_circuit(n, a.gates, 1).gates, n)
            res = tuner.tune(eng, vec, n, ops)
            print(json.dumps({"n": n, "precision": prec, "knobs": res.knobs.to_json(), "ms": res.ms}), flush=True)
            del vec
            torch.cuda.empty_cache()


if __name__ == "__main__":
    main()

"""Seeded synthetic workloads.

uniform circuit: n qubits, gates uniform over {H, X, Rx, Ry, Rz, U3, CX, CZ,
         Rzz, Swap}, angles uniform in [0, 2 pi), distinct uniform qubits.
spread circuit: the same gate set plus 10% random Haar 2-qubit unitaries;
         every qubit argument is drawn, with probability 1/2 each, from the
         qubits on vector bits < 5 or from those on vector bits >= n - 10
         (targets spread over low and high bits).
noisy density matrix, hardware-efficient ansatz: see their functions.
All generators use numpy.random.default_rng(seed); nothing is read from disk.
"""
from __future__ import annotations

import numpy as np

from .core import GATE_BY_NAME, Circuit, Unitary

GATE_SET = ["h", "x", "rx", "ry", "rz", "u3", "cx", "cz", "rzz", "swap"]


def haar_unitary(rng: np.random.Generator, d: int) -> np.ndarray:
    """Haar-random d x d unitary (QR of a complex Ginibre matrix, phases fixed)."""
    z = (rng.normal(size=(d, d)) + 1j * rng.normal(size=(d, d))) / np.sqrt(2.0)
    q, r = np.linalg.qr(z)
    return q * (np.diag(r) / np.abs(np.diag(r)))


def uniform_circuit(n: int = 20, size: int = 200, seed: int = 0) -> Circuit:
    c = Circuit(n)
    c.random_append(size, seed=seed)
    return c


def spread_circuit(n: int = 30, size: int = 1000, seed: int = 1, haar_frac: float = 0.1) -> Circuit:
    rng = np.random.default_rng(seed)
    c = Circuit(n)
    low = [n - 1 - b for b in range(min(5, n))]                 # qubits on vector bits 0..4
    high = [n - 1 - b for b in range(max(5, n - 10), n)]        # qubits on vector bits >= n-10

    def pick(k):
        out = []
        while len(out) < k:
            grp = low if rng.random() < 0.5 else high
            q = int(grp[rng.integers(len(grp))])
            if q not in out:
                out.append(q)
        return out

    for _ in range(size):
        if rng.random() < haar_frac:
            Unitary(haar_unitary(rng, 4)) | c(pick(2))
            continue
        nm = GATE_SET[rng.integers(len(GATE_SET))]
        g = GATE_BY_NAME[nm]
        if g.params:
            g = g(*[float(x) for x in rng.uniform(0, 2 * np.pi, g.params)])
        g | c(pick(g.controls + g.targets))
    return c


def noisy_dm_problem(n: int = 12, size: int = 150, seed: int = 2, gamma: float = 5e-3, p1: float = 1e-3,
                    p2: float = 1e-2):
    """Noisy density-matrix run: a `size`-gate circuit from the uniform-circuit gate set,
    each gate followed by amplitude damping (gamma) composed with depolarizing
    noise (p1 for 1-qubit gates, p2 for 2-qubit gates) on the touched qubits.
    Returns (circuit, noise_model)."""
    from .core import DampingError, DepolarizingError, NoiseModel
    c = uniform_circuit(n, size, seed)
    one = ["h", "x", "rx", "ry", "rz", "u3"]
    two = ["cx", "cz", "rzz", "swap"]
    amp = DampingError(amplitude_prob=gamma, phase_prob=0)
    nm = NoiseModel(basic_gates=one + two)
    nm.add_noise_for_all_qubits(amp.compose(DepolarizingError(p1, 1)), one)
    nm.add_noise_for_all_qubits(amp.tensor(amp).compose(DepolarizingError(p2, 2)), two)
    return c, nm


def hea_problem(n: int = 16, layers: int = 8, batch: int = 1024, seed: int = 3):
    """Hardware-efficient ansatz (Ry, Rz on every qubit + CZ ring per layer),
    H = sum Z_i Z_{i+1} (open chain) + 0.5 sum X_i, params uniform in [0, 2 pi)."""
    from .differentiation import hardware_efficient_ansatz, ising_observable
    circ = hardware_efficient_ansatz(n, layers)
    obs = ising_observable(n)
    params = np.random.default_rng(seed).uniform(0, 2 * np.pi, (batch, circ.num_params))
    return circ, obs, params


def sharded_run(qubits: int, precision: str, gates: int, seed: int = 1) -> dict:
    """The spread circuit on a vector sharded over every rank of the
    default process group (one GPU per rank, NCCL), device-timed with CUDA
    events and reduced as the max over ranks."""
    import torch
    import torch.distributed as dist

    from .simulation.sharded import ShardedStateVector
    circuit = spread_circuit(qubits, gates, seed)
    sv = ShardedStateVector(qubits, precision, device=torch.device("cuda", torch.cuda.current_device()))
    sv.run(spread_circuit(qubits, 8, seed + 1))  # warm-up: knobs, matrix tables, communicators
    dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ex0 = sv.exchanges
    e0.record()
    sv.run(circuit)
    e1.record()
    torch.cuda.synchronize()
    t = torch.tensor([e0.elapsed_time(e1)], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms = float(t.item())
    return {"workload": f"sv-{qubits}q-{precision}-{gates}g-spread sharded over {sv.world} ranks",
            "ms": ms, "gates_per_s": gates / (ms / 1e3), "exchanges": sv.exchanges - ex0,
            "norm2": sv.norm2()}


def main() -> None:
    """Run one workload (for profiling a single kernel family):

        python -m quict_b200.workloads gradient --batch 256 [--precision single] [--repeat 2]
            [--tile-bits K] [--pair-tile-bits K]                       (cuda:0)
        python -m quict_b200.workloads qaoa-batch --instances 8 --sizes 20,22,24 [--repeat 2]
            [--tiles-per-item T] [--tile-bits K] [--pair-tile-bits K]  (cuda:0; ONE persistent
            launch per repeat, after the warm-up run that compiles and links its stages)
        torchrun --nproc-per-node N -m quict_b200.workloads sharded --qubits Q
            [--precision double] [--gates 1000]                        (one GPU per rank)
    """
    import argparse
    import json
    import os

    import torch

    ap = argparse.ArgumentParser()
    ap.add_argument("workload", choices=["gradient", "sharded", "qaoa-batch"])
    ap.add_argument("--instances", type=int, default=8)
    ap.add_argument("--sizes", default="20,22,24", help="qubit counts of the seeded QAOA instances")
    ap.add_argument("--tiles-per-item", type=int, default=16)
    ap.add_argument("--batch", type=int, default=1024)
    ap.add_argument("--precision", default=None, choices=["single", "double"])
    ap.add_argument("--repeat", type=int, default=2)
    ap.add_argument("--tile-bits", type=int, default=None, help="forward register tile width k")
    ap.add_argument("--pair-tile-bits", type=int, default=None, help="backward pair tile width k")
    ap.add_argument("--qubits", type=int, default=32)
    ap.add_argument("--gates", type=int, default=1000)
    a = ap.parse_args()
    if a.workload == "sharded":
        import datetime

        import torch.distributed as dist
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        try:
            res = sharded_run(a.qubits, a.precision or "double", a.gates)
            if dist.get_rank() == 0:
                print(json.dumps(res))
        finally:
            dist.destroy_process_group()
        return
    a.precision = a.precision or "single"
    if a.workload == "qaoa-batch":
        from .differentiation import BatchedAdjoint, maxcut_observable, qaoa_circuit, qaoa_instances
        from .differentiation.persistent import DEFAULT_CAPS, PersistentBatch
        inst = qaoa_instances(a.instances, sizes=tuple(int(v) for v in a.sizes.split(",")))
        caps = (a.tile_bits or DEFAULT_CAPS[a.precision][0], a.pair_tile_bits or DEFAULT_CAPS[a.precision][1])
        pb = PersistentBatch([(BatchedAdjoint(qaoa_circuit(n, e, p), maxcut_observable(n, e), a.precision), prm)
                              for n, e, p, prm in inst], a.precision, caps=caps, tiles_per_item=a.tiles_per_item,
                             jit_min_qubits=min(int(v) for v in a.sizes.split(",")))
        pb.capture()
        for _ in range(a.repeat):
            pb.launch()
        res = pb.results()
        print(f"qaoa batch {a.instances} {a.precision}: linked={pb.linked} items={pb.sizes.nitems} "
              f"sum E = {sum(e for e, _ in res):.6e}")
        return
    from .differentiation import BatchedAdjoint
    circ, obs, params = hea_problem(16, 8, a.batch)
    eng = BatchedAdjoint(circ, obs, a.precision, tile_bits=a.tile_bits, pair_tile_bits=a.pair_tile_bits)
    gp = eng.plan_gradient(params)
    for _ in range(a.repeat):
        eng.launch(gp)
    torch.cuda.synchronize()
    print(f"gradient batch {a.batch} {a.precision}: |grad|_1 = {float(gp.gradients.abs().sum()):.6e}")


if __name__ == "__main__":
    main()

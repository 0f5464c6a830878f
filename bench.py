"""Benchmark: state-vector gate application at 30 qubits on B200.

Workload (one step): StateVectorSimulator.run of the seeded 1000-gate
spread circuit (gate set {H, X, Rx, Ry, Rz, U3, CX, CZ, Rzz, Swap} + 10% Haar
2-qubit unitaries, qubits spread over vector bits < 5 and >= 20) on a
30-qubit complex128 state (16 GiB): |0...0> initialisation + every gate.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

value   gates/s with the state resident in HBM, device-timed (CUDA events),
        max over ranks; N>1 runs independent replicas (the path does not
        shard: a 30-qubit state fits one GPU), value = N * gates / time.
e2e     the same metric through the public API (StateVectorSimulator.run):
        host planning, matrix-table host->device copy and a device->host read
        of P(qubit 0 = 0) inside every step.
roofline  the fused-pass kernel (qs_pass: each pass compiled at run time; the
        generic k_fused_reg runs a pass until its kernel is ready), bound fp64: algorithmic flops of
        its ops over its CUDA-event time, against cuBLAS DGEMM measured here;
        roofline_hbm: 2 * 2^n * 16 bytes per launch against MEASURED_PEAKS.json.
single_gate_sweep, c64, public_api_runs, adjoint, qaoa  extra sections: per-gate HBM
        fractions, complex64 at 30/32 qubits, the 20-qubit state-vector and 12-qubit
        noisy density-matrix runs, ansatz gradients, the QAOA batch.
cpu_baseline  the numba port of the reference CPU kernels (oracle/ref_port.py)
        on this host's cores: gates of every class of the same circuit timed,
        rate = 1000 / sum over classes (count x mean s/gate);
        cpu_baseline_1thread: the same on one thread (26 qubits, scaled).
"""
from __future__ import annotations

import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_QUBITS = 30
N_GATES = 1000
SEED = 1
METRIC = "gates/s & HBM GB/s at 30q"


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def ncu_traffic(n):
    """dram bytes per fused-pass launch from the committed ncu summary of the
    generated pass kernel (a 26-qubit capture scaled by the amplitudes
    processed), or None."""
    for name in ("qs_pass_spread_c128.txt", "k_fused_reg_spread_c128.txt"):
        p = os.path.join(ROOT, "profiles", name)
        if os.path.exists(p):
            m = re.search(r"traffic_bytes_per_launch_30q:\s*([0-9.eE+]+)", open(p).read())
            if m:
                return float(m.group(1)) * 2.0 ** (n - 30)
    return None


class Clocks:
    """nvidia-smi sampler for the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        # raw samples go to $QS_CLOCKS_DIR (default: the temp directory); the
        # JSON line carries their summary
        d = os.environ.get("QS_CLOCKS_DIR") or tempfile.gettempdir()
        self.path = os.path.join(d, f"clocks_{os.getpid()}.csv")

    def __enter__(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index),
                 "--query-gpu=clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,"
                 "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
                 "clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "100"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            time.sleep(0.25)
            self.proc.terminate()
            self.proc.wait()
            self.f.close()

    def summary(self):
        try:
            rows = [r.split(",") for r in open(self.path).read().strip().splitlines() if r.strip()]
        except Exception:
            rows = []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        sm, mx, reasons = [], [], set()
        for r in rows:
            try:
                sm.append(float(r[0]))
                mx.append(float(r[1]))
                for i, nm in enumerate(names):
                    if r[2 + i].strip().lower().startswith("active"):
                        reasons.add(nm)
            except (ValueError, IndexError):
                continue
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_init(args):
    import torch
    import torch.distributed as dist
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    elif torch.cuda.is_available():
        torch.cuda.set_device(0)
    return ws, rank, local


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x, ws):
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda" if dist.get_backend() == "nccl" else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


class CpuBaseline:
    """Numba port of the reference CPU kernels (oracle/ref_port.py) on a host
    copy of the state; the state is allocated once and reused.

    Estimator: the circuit's gates are grouped by class (gate type; 2-qubit
    Haar unitaries are "unitary").  A sample times whole gates of every class
    in turn; the full circuit's time is estimated as sum over classes of
    (gates of that class) x (mean sampled seconds per gate of that class), and
    the rate is gates / that time -- total gates over total time, with each
    class weighted by its share of the circuit."""

    def __init__(self, circuit, n, threads=None):
        import numpy as np
        from oracle import ref_port
        from quict_b200.simulation.lowering import lower_gate
        if threads is not None:
            import numba
            numba.set_num_threads(int(threads))
        self.np, self.port, self.n = np, ref_port, n
        self.classes = {}
        self.prepared = []
        for g in circuit.gates:
            ops = lower_gate(g, n)
            self.classes.setdefault(g.type.name, []).append(len(self.prepared))
            self.prepared.append(ref_port.prepare(ops, np.complex128))
        self.total = len(self.prepared)
        self.vec = np.zeros(1 << n, dtype=np.complex128)
        self.vec[0] = 1
        self.times = {c: [] for c in self.classes}
        # compile every kernel signature once on a 10-qubit vector
        warm = np.zeros(1 << 10, dtype=np.complex128)
        seen = set()
        for ops in (lower_gate(g, n) for g in circuit.gates):
            for op in ops:
                key = (op.kind, op.m, len(op.cbits))
                if key in seen:
                    continue
                seen.add(key)
                t = tuple(range(op.m))
                c = tuple(range(op.m, op.m + len(op.cbits)))
                ref_port.run(warm, ref_port.prepare([type(op)(op.kind, t, c, op.mat)], np.complex128))

    def sample(self, rounds=1, budget_s=float("inf"), record=True):
        """Time `rounds` gates of every class (the next unsampled occurrences);
        stops early after `budget_s` seconds.  Returns seconds spent."""
        t_all = time.perf_counter()
        for _ in range(rounds):
            for c, idx in self.classes.items():
                k = idx[len(self.times[c]) % len(idx)]
                t0 = time.perf_counter()
                self.port.run(self.vec, self.prepared[k])
                dt = time.perf_counter() - t0
                if record:
                    self.times[c].append(dt)
                if time.perf_counter() - t_all > budget_s:
                    return time.perf_counter() - t_all
        return time.perf_counter() - t_all

    def estimate(self):
        """(gates/s, {class: mean s/gate}, gates timed) from the samples so far."""
        per = {c: sum(t) / len(t) for c, t in self.times.items() if t}
        if len(per) < len(self.classes):
            missing = [c for c in self.classes if c not in per]
            raise RuntimeError(f"no timing sample for gate classes {missing}")
        total_s = sum(len(self.classes[c]) * per[c] for c in self.classes)
        return self.total / total_s, per, sum(len(t) for t in self.times.values())

    def describe(self, gates_timed, seconds):
        counts = {c: len(i) for c, i in self.classes.items()}
        return (f"{gates_timed} gates of the 1000-gate {self.n}q c128 spread circuit timed in {seconds:.1f} s, "
                f"stratified by gate class {counts}; rate = 1000 / sum(count x mean s/gate) "
                f"(numba restatement of QuICT cpu_calculator kernels)")

    @staticmethod
    def threads():
        import numba
        return numba.get_num_threads()


def one_thread_baseline(circuit_fn, n_small=26, n=30):
    """The port on ONE host thread (the reference's own numba kernels are
    single-threaded) at n_small qubits, one gate per class, scaled by
    2^(n - n_small) to n qubits (time per gate is linear in the amplitudes)."""
    cb = CpuBaseline(circuit_fn(n_small), n_small, threads=1)
    secs = cb.sample(rounds=1)
    r, per, k = cb.estimate()
    scale = 2.0 ** (n - n_small)
    import numba
    numba.set_num_threads(numba.config.NUMBA_NUM_THREADS)
    return {"value": r / scale, "unit": "gates/s", "cores": 1, "kind": "port",
            "s_per_gate_by_class": {c: v * scale for c, v in per.items()},
            "sample": f"one gate per class at {n_small} qubits on 1 thread ({secs:.1f} s), "
                      f"scaled by 2^{n - n_small} to {n} qubits (extrapolated)"}


def run_reference(args, ws, rank):
    """--impl reference: the reference CPU algorithm (numba port, every host
    thread) on the same workload; each step times one gate of every class."""
    if rank != 0:
        return
    from quict_b200.workloads import spread_circuit
    circuit = spread_circuit(N_QUBITS, N_GATES, SEED)
    cb = CpuBaseline(circuit, N_QUBITS)
    for _ in range(args.warmup):
        cb.sample(rounds=1, record=False)
    secs = cb.sample(rounds=args.steps)
    v, per, timed = cb.estimate()
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "gates/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "c128", "data": "synthetic (seeded spread circuit)",
        "config": {"workload": f"sv-{N_QUBITS}q-c128-{N_GATES}g-spread", "qubits": N_QUBITS,
                   "gates_per_step": len(cb.classes), "seed": SEED},
        "cpu_baseline": {"value": v, "unit": "gates/s", "cores": cb.threads(), "kind": "port",
                         "s_per_gate_by_class": per, "sample": cb.describe(timed, secs)},
        "e2e": {"value": v, "unit": "gates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    if args.ref_one_thread:
        line["cpu_baseline_1thread"] = one_thread_baseline(lambda q: spread_circuit(q, N_GATES, SEED),
                                                           n=N_QUBITS)
    print(json.dumps(line), flush=True)


def _events_ms(fn, reps):
    import torch
    fn()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(reps):
        fn()
    b.record()
    torch.cuda.synchronize()
    return a.elapsed_time(b) / reps


def sv_rate(n, precision, local, ws, steps=2, warmup=1, merge_bits=None):
    """Device-timed gates/s of the spread circuit at n qubits (extra precisions / sizes)."""
    import torch
    from quict_b200 import _native as N
    from quict_b200.simulation import StateVectorSimulator
    from quict_b200.simulation.fusion import Pass
    from quict_b200.simulation.lowering import lower_circuit
    from quict_b200.workloads import spread_circuit
    circuit = spread_circuit(n, N_GATES, SEED)
    sim = StateVectorSimulator("GPU", precision, gpu_device_id=local, sync=False, merge_bits=merge_bits)
    eng = sim.engine
    ops = lower_circuit(circuit.gates, n)
    sim.initial_circuit(circuit)
    sim.initial_state_vector()
    vec = sim._vector
    plan_ = eng.plan(vec, n, ops)
    dt = N.QS_C128 if precision == "double" else N.QS_C64

    def step():
        N.call("qs_init_zero", vec.data_ptr(), n, dt, eng.stream)
        batch = []
        for st in plan_:
            if isinstance(st, Pass):
                batch.append(st)
            else:
                eng.run_passes(vec, n, batch)
                batch = []
                eng.apply_single(vec, n, st.op)
        eng.run_passes(vec, n, batch)

    for _ in range(warmup):
        step()
    N.jit_wait(600)  # compiled passes ready (no-op with the JIT off)
    step()
    barrier(ws)
    ms = max_over_ranks(_events_ms(step, steps), ws)
    passes = sum(1 for s in plan_ if isinstance(s, Pass) and s.ops)
    knobs = eng.knobs(vec, n).to_json()
    del sim, vec
    torch.cuda.empty_cache()
    return {"workload": f"sv-{n}q-{'c128' if precision == 'double' else 'c64'}-{N_GATES}g-spread",
            "gates_per_s": ws * len(ops) / (ms / 1e3), "ms_per_run": ms, "fused_passes": passes,
            "knobs": knobs,
            "state_bytes": (1 << n) * (16 if precision == "double" else 8)}


def c64_error(n, local):
    """complex64 against complex128 on the spread circuit at n qubits (both
    run by this GPU; the complex128 path is checked against the FP64 oracle
    and the per-gate kernels by the parity tests): max |amplitude error| and
    max error of <Z> on a spread of qubits (FP64 P(0) reductions)."""
    import numpy as np
    import torch
    from quict_b200.simulation import StateVectorSimulator
    from quict_b200.workloads import spread_circuit
    a = StateVectorSimulator("GPU", "double", gpu_device_id=local)
    va = a.run(spread_circuit(n, N_GATES, SEED)).tensor
    b = StateVectorSimulator("GPU", "single", gpu_device_id=local)
    vb = b.run(spread_circuit(n, N_GATES, SEED)).tensor
    amp = 0.0
    for i in range(0, va.numel(), 1 << 27):
        amp = max(amp, float((va[i:i + (1 << 27)] - vb[i:i + (1 << 27)].to(torch.complex128)).abs().max()))
    bits = sorted({0, 1, 4, n // 2, n - 2, n - 1})
    za = np.array([2 * a.engine.prob0(va, n, q) - 1 for q in bits])
    zb = np.array([2 * b.engine.prob0(vb, n, q) - 1 for q in bits])
    out = {"max_abs_amp_err_vs_c128": amp, "max_abs_z_expectation_err_vs_c128": float(np.max(np.abs(za - zb))),
           "z_vector_bits": bits}
    del a, b, va, vb
    torch.cuda.empty_cache()
    return out


def grad_bench(ws, rank, local, batch=1024):
    """Hardware-efficient-ansatz gradients: 16q x 8 layers, 256 params, batch 1024 (split over ranks),
    H = sum ZZ + 0.5 sum X.  Adjoint gradient (c64, c128) vs the same GPU's
    parameter shift (2 parameters timed, scaled to 256)."""
    import torch
    from quict_b200.differentiation import BatchedAdjoint
    from quict_b200.workloads import hea_problem
    circ, obs, params = hea_problem(16, 8, batch)
    from quict_b200.distributed import block_shard
    rows = block_shard(batch, ws, rank)
    per = len(rows)
    mine = params[rows.start:rows.stop]
    out = {"workload": f"hea-16q-8layers-256params-batch{batch}", "observable": "sum Z_i Z_i+1 (open) + 0.5 sum X_i",
           "instances_per_rank": per}
    grads = {}
    from quict_b200 import _native as N
    shift_idx = list(range(0, 256, 16))  # 16 parameters spread over the layers
    for prec in ("single", "double"):
        eng = BatchedAdjoint(circ, obs, prec, local)
        gp = eng.plan_gradient(mine)
        eng.launch(gp)
        eng.parameter_shift(mine, indices=shift_idx[:1])
        N.jit_wait(900)  # both methods run on compiled passes when timed
        barrier(ws)
        ms = max_over_ranks(_events_ms(lambda: eng.launch(gp), 3), ws)
        grads[prec] = gp.gradients.clone()
        ps_ms = max_over_ranks(_events_ms(lambda: eng.parameter_shift(mine, indices=shift_idx), 1), ws)
        ps_ms = ps_ms / len(shift_idx) * 256
        key = "c64" if prec == "single" else "c128"
        out[key] = {"ms": ms, "grads_per_s": ws * per * 256 / (ms / 1e3),
                    "param_shift_ms": ps_ms,
                    "param_shift_note": f"{len(shift_idx)} parameters timed (two shifted batched runs per "
                                        f"occurrence, same GPU kernels), scaled to 256",
                    "speedup_vs_param_shift": ps_ms / ms}
        del gp, eng
        torch.cuda.empty_cache()
    out["max_abs_grad_err_c64_vs_c128"] = float((grads["single"] - grads["double"]).abs().max())
    return out


def qaoa_bench(ws, rank, local, count=512, graph_too=False):
    """Uneven QAOA MaxCut batch (n in 10..24 even, p in 1..6),
    complex64, instances split over ranks by amplitude x depth cost.  Timed:
    ONE persistent launch per rank (qs_batch_launch: every instance's forward
    passes, lam = C psi, energy, adjoint sweep and sums as work items; the
    register stages of instances >= 22 qubits as generated functions linked
    into the kernel), replayed from a CUDA graph (a control-word memset node
    and the kernel node).  graph_too: also the per-instance kernel chains
    captured over 16 streams into one graph, for comparison."""
    import torch
    from quict_b200.differentiation import UnevenQAOABatch, qaoa_instances
    from quict_b200.distributed import balanced_shard
    inst = qaoa_instances(count)
    parts = balanced_shard([float(2 ** n) * (p * (1.5 * n + n)) for n, _, p, _ in inst], ws)
    mine = [inst[i] for i in parts[rank]]
    total_grads = sum(2 * p for _, _, p, _ in inst)
    out = {"workload": f"qaoa-maxcut-{count}instances-n10..24-p1..6", "dtype": "c64"}
    t0 = time.perf_counter()
    batch = UnevenQAOABatch(mine, "single", local, mode="persistent", label=f"qaoa{count}")
    batch.capture()
    setup_s = time.perf_counter() - t0
    barrier(ws)
    ms = max_over_ranks(_events_ms(batch.replay, 3), ws)
    batch.persistent.check()
    sz = batch.persistent.sizes
    out.update({"graph_replay_ms": ms, "grads_per_s": total_grads / (ms / 1e3), "instances_per_s": count / (ms / 1e3),
                "launches_per_replay": 1, "graph_nodes": "memset of the control words + the persistent kernel",
                "linked_generated_stages": bool(batch.persistent.linked), "generated_functions": int(sz.jit_fns),
                "work_items": int(sz.nitems), "cta_threads": int(sz.threads), "caps": list(batch.caps),
                "jit_min_qubits": batch.jit_min_qubits, "setup_s_incl_compile_and_link": setup_s})
    del batch
    torch.cuda.empty_cache()
    if graph_too:
        t0 = time.perf_counter()
        g = UnevenQAOABatch(mine, "single", local, mode="graph")
        g.capture()
        setup_s = time.perf_counter() - t0
        barrier(ws)
        gms = max_over_ranks(_events_ms(g.replay, 3), ws)
        out["per_instance_chains"] = {"graph_replay_ms": gms, "launches_per_replay": g.captured_launches,
                                      "setup_s_incl_compile": setup_s}
    return out


def small_runs_bench(ws, local, reps=3):
    """Configs 0 and 2 through the public API, wall time per call with the
    device synchronised on both sides (host planning and copies included):
    StateVectorSimulator.run of the 20-qubit 200-gate uniform circuit, then
    sample(8192); DensityMatrixSimulator.run of the 12-qubit
    150-gate circuit with composed damping + depolarizing noise per gate."""
    import torch
    from quict_b200.simulation import DensityMatrixSimulator, StateVectorSimulator
    from quict_b200.workloads import uniform_circuit, noisy_dm_problem
    dev = torch.device("cuda", local)

    def wall(fn):
        from quict_b200 import _native as N
        fn()
        N.jit_wait(600)  # the run's passes compiled (first use of their shapes)
        fn()
        torch.cuda.synchronize(dev)
        barrier(ws)
        t0 = time.perf_counter()
        for _ in range(reps):
            fn()
        torch.cuda.synchronize(dev)
        return max_over_ranks((time.perf_counter() - t0) / reps * 1e3, ws)

    c0 = uniform_circuit(20, 200, 0)
    sv = StateVectorSimulator("GPU", "double", gpu_device_id=local)
    run_ms = wall(lambda: sv.run(c0))
    sample_ms = wall(lambda: sv.sample(8192, seed=7))
    c2, nm = noisy_dm_problem(12, 150, 2)
    dm = DensityMatrixSimulator("GPU", "double", accumulated_mode=True, gpu_device_id=local)
    dm_ms = wall(lambda: dm.run(c2, noise_model=nm))
    return {"sv_20q": {"workload": "sv-20q-c128-200g-uniform + 8192 shots", "run_ms": run_ms,
                        "sample_8192_ms": sample_ms, "gates_per_s": ws * 200 / (run_ms / 1e3)},
            "dm_12q": {"workload": "dm-12q-c128-150g-damping+depolarizing", "run_ms": dm_ms,
                        "gates_per_s": ws * 150 / (dm_ms / 1e3)},
            "timing": "wall clock per public call, device synchronised, max over ranks"}


SWEEP_1Q = ("h", "x", "rx", "ry", "rz", "u3")
SWEEP_2Q = ("cx", "cz", "rzz", "swap")


SECTOR = 32  # bytes: the L2 / DRAM sector, the smallest unit a skipped run can save


def op_flops(op):
    """Algorithmic FP64 flops per amplitude of a fused op: a dense m-qubit
    matrix costs, per output, one complex multiply-add (8 flops; the first
    one a multiply, 6) for each entry of its row that is neither 0 nor +-1,
    and one complex add (2; none for the first) for each +-1 entry, averaged
    over the rows; a diagonal one complex multiply (6) on the entries that
    are not 1; plain exchanges (X, CX, Swap) none; each control halves the
    amplitudes touched."""
    import numpy as np
    frac = 0.5 ** len(op.cbits)
    if op.kind == "mat":
        m = np.asarray(op.mat)
        tot = 0.0
        for row in m:
            gen = int(np.sum((row != 0) & (row != 1) & (row != -1)))
            one = int(np.sum((row == 1) | (row == -1)))
            f = 8 * gen + 2 * one
            f -= 2 if gen else (2 if one else 0)  # the first term is a product or a copy
            tot += max(f, 0)
        return tot / m.shape[0] * frac
    if op.kind == "diag":
        d = np.asarray(op.mat).ravel()
        return 6 * float(np.mean(np.abs(d - 1) > 1e-15)) * frac
    m = np.asarray(op.mat)
    unit = op.kind == "antidiag" and abs(m[0, 1] - 1) < 1e-15 and abs(m[1, 0] - 1) < 1e-15
    unit = unit or (op.kind == "swap" and all(abs(m[i, j] - 1) < 1e-15 for i, j in ((0, 0), (1, 2), (2, 1), (3, 3))))
    return 0.0 if unit else 6 * frac


def pass_flops(p_, n):
    return sum(op_flops(op) for op in p_.ops) * (1 << n)


def fp64_peak_tflops(dev):
    """Measured FP64 peak: cuBLAS DGEMM (torch.matmul float64, 8192^3), best of 3.
    On B200 the FP64 tensor path and the FP64 FMA pipe peak alike (~35-37 TFLOP/s)."""
    import torch
    a = torch.randn(8192, 8192, dtype=torch.float64, device=dev)
    b = torch.randn_like(a)
    torch.matmul(a, b)
    torch.cuda.synchronize(dev)
    best = float("inf")
    for _ in range(3):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize(dev)
        best = min(best, e0.elapsed_time(e1))
    del a, b
    torch.cuda.empty_cache()
    return 2 * 8192 ** 3 / (best / 1e3) / 1e12, "measured: cuBLAS DGEMM 8192^3 in bench.py"


def knob_source(eng, vec, n):
    """Where the fused-pass knobs of this run come from."""
    import torch
    from quict_b200.simulation.autotune import tune_key
    explicit = None not in (eng.tile_bits, eng.low_bits, eng.merge_bits, eng.max_pass_cost)
    if explicit:
        return "command line"
    key = tune_key(torch.cuda.get_device_name(eng.device), vec.element_size(), n, eng.tune_kind)
    return "tuning cache" if eng.tuner.lookup(key) else "defaults (no cache entry)"


def sweep_bytes(name, bits, n, esize):
    """Bytes a per-gate kernel must move: every 32-byte sector holding an
    amplitude it changes is read and written once.  CX changes the control=1
    half, Swap the |01>,|10> half and CZ the |11> quarter (entries equal to 1
    are skipped); a skipped half saves traffic only when its runs (2^bit
    amplitudes) span whole sectors.  The other gates change every amplitude."""
    def halves(b):
        return 0.5 if (1 << b) * esize >= SECTOR else 1.0
    if name == "cx":
        frac = halves(bits[0])
    elif name == "cz":
        frac = halves(bits[0]) * halves(bits[1])
    elif name == "swap":
        frac = halves(min(bits))
    else:
        frac = 1.0
    return int(2 * (1 << n) * esize * frac)


def _sweep_bits(n):
    """Target vector bits of the 1q sweep: in-warp (0, 1, 2, 4), the first
    pair-indexed bit (5), middle (10, 20) and the highest."""
    return [(b,) for b in sorted({0, 1, 2, 4, 5, 10, 20, n - 1}) if b < n]


def _sweep_pairs(n):
    """(first, second) vector bits of the 2q sweep: both in-warp, mixed, both
    high, and the highest with the lowest."""
    cand = [(1, 0), (4, 2), (10, 5), (20, 10), (n - 1, n - 2), (n - 1, 0)]
    out = []
    for p in cand:
        if max(p) < n and p[0] != p[1] and p not in out:
            out.append(p)
    return out


def gate_sweep(eng, vec, n, ws, reps=5, warmup=2):
    """Single-gate sweep: each gate class of the spread-circuit gate set applied by
    its per-gate kernel to the resident n-qubit state at vector bits from the
    in-warp ones to the highest (``_sweep_bits`` / ``_sweep_pairs``);
    device-timed per launch; GB/s from ``sweep_bytes`` against the measured
    HBM copy bandwidth."""
    import torch
    from quict_b200.core import GATE_BY_NAME
    from quict_b200.simulation.lowering import lower_gate
    peak, kind = peaks()
    esize = vec.element_size()
    rows = []
    for name in SWEEP_1Q + SWEEP_2Q:
        g = GATE_BY_NAME[name]
        if g.params:
            g = g(*[0.3 + 0.1 * i for i in range(g.params)])
        two = name in SWEEP_2Q
        # (vector bits) -> circuit qubits (qubit q is vector bit n-1-q)
        for bits in (_sweep_pairs(n) if two else _sweep_bits(n)):
            (op,) = lower_gate(g & [n - 1 - b for b in bits], n)
            for _ in range(warmup):
                eng.apply_single(vec, n, op)
            ms = max_over_ranks(_events_ms(lambda: eng.apply_single(vec, n, op), reps), ws)
            gbs = sweep_bytes(name, bits, n, esize) / (ms / 1e3) / 1e9
            rows.append({"gate": name, "vector_bits": list(bits), "ms": round(ms, 4),
                         "gbs": round(gbs, 1), "frac": round(gbs / peak, 4)})
    fr = sorted(r["frac"] for r in rows)
    return {"workload": f"sv-{n}q-{'c128' if esize == 16 else 'c64'} one gate per launch",
            "peak_gbs": peak, "peak_source": kind, "min_frac": fr[0], "median_frac": fr[len(fr) // 2],
            "bytes_rule": "read+write of the 32-byte sectors holding amplitudes the gate changes",
            "rows": rows}


def run_ours(args, ws, rank, local):
    import numpy as np
    import torch
    from quict_b200 import _native as N
    from quict_b200.simulation import StateVectorSimulator
    from quict_b200.simulation.lowering import lower_circuit
    from quict_b200.workloads import spread_circuit

    n = args.qubits
    circuit = spread_circuit(n, N_GATES, SEED)
    sim = StateVectorSimulator("GPU", "double", gpu_device_id=local, sync=False,
                               max_pass_cost=args.max_pass_cost, merge_bits=args.merge_bits,
                               tile_bits=args.tile_bits)
    eng = sim.engine
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream(dev)
    ops = lower_circuit(circuit.gates, n)
    sim.initial_circuit(circuit)
    sim.initial_state_vector()
    vec = sim._vector
    steps_plan = eng.plan(vec, n, ops)
    from quict_b200.simulation.fusion import Pass
    npasses = sum(1 for s in steps_plan if isinstance(s, Pass) and s.ops)
    nsingle = sum(1 for s in steps_plan if not isinstance(s, Pass))

    def device_step():
        N.call("qs_init_zero", vec.data_ptr(), n, N.QS_C128, eng.stream)
        batch = []
        for st in steps_plan:
            if isinstance(st, Pass):
                batch.append(st)
            else:
                eng.run_passes(vec, n, batch)
                batch = []
                eng.apply_single(vec, n, st.op)
        eng.run_passes(vec, n, batch)

    # warm-up; passes run as run-time compiled kernels once their compilation
    # (on host threads, started by the first step) has finished
    jit0 = N.jit_stats()
    t_jit = time.perf_counter()
    device_step()
    if args.jit:
        N.jit_wait(600)
    jit_wall_s = time.perf_counter() - t_jit
    for _ in range(max(0, args.warmup - 1)):
        device_step()
    torch.cuda.synchronize(dev)
    barrier(ws)
    jit1 = N.jit_stats()
    launches0 = eng.launches
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Clocks(local) as clk:
        torch.cuda.synchronize(dev)
        e0.record(stream)
        for _ in range(args.steps):
            device_step()
        e1.record(stream)
        torch.cuda.synchronize(dev)
    barrier(ws)
    ms = e0.elapsed_time(e1) / args.steps
    launches = (eng.launches - launches0) // args.steps + 1  # + qs_init_zero
    jit2 = N.jit_stats()
    jit_info = {"mode": "async" if args.jit else "off",
                "kernels_compiled": jit1["compiled"] - jit0["compiled"],
                "compile_ms_host_threads": jit1["compile_ms"] - jit0["compile_ms"],
                "first_step_wall_s_incl_compile": jit_wall_s,
                "compiled_launches_per_step": (jit2["compiled_launches"] - jit1["compiled_launches"]) / args.steps,
                "generic_launches_per_step": (jit2["generic_launches_while_pending"]
                                              - jit1["generic_launches_while_pending"]) / args.steps}
    ms = max_over_ranks(ms, ws)
    value = ws * len(ops) / (ms / 1e3)

    # per-pass kernel timing for the roofline (separate, events per pass)
    eng.pass_events = []
    device_step()
    torch.cuda.synchronize(dev)
    durs = [a.elapsed_time(b) for a, b, _ in eng.pass_events]
    eng.pass_events = None
    bytes_per_pass = 2 * (1 << n) * 16
    avg_pass_ms = statistics.mean(durs) if durs else float("nan")
    achieved = bytes_per_pass / (avg_pass_ms / 1e3) / 1e9
    peak, peak_kind = peaks()
    # FP64 view: algorithmic flops of the fused passes over their event time
    pass_list = [s for s in steps_plan if isinstance(s, Pass) and s.ops]
    flops = sum(pass_flops(p_, n) for p_ in pass_list)
    fp64_peak, fp64_src = fp64_peak_tflops(dev)
    fp64_achieved = flops / (sum(durs) / 1e3) / 1e12 if durs else float("nan")

    # e2e through the public API: run() + P(q0 = 0) readback each step
    h2d0 = eng.h2d_bytes
    for _ in range(1):
        sim.run(circuit)
        sim.get_measured_prob(n - 1)
    torch.cuda.synchronize(dev)
    barrier(ws)
    h2d0 = eng.h2d_bytes
    t0 = time.perf_counter()
    E = max(1, args.steps // 2)
    for _ in range(E):
        sim.run(circuit)
        p = sim.get_measured_prob(n - 1)
    torch.cuda.synchronize(dev)
    e2e_s = (time.perf_counter() - t0) / E
    e2e_s = max_over_ranks(e2e_s, ws)
    h2d = (eng.h2d_bytes - h2d0) // E

    line = {
        "metric": METRIC, "value": value, "unit": "gates/s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "c128", "data": "synthetic (seeded spread circuit)",
        "config": {"workload": f"sv-{n}q-c128-{N_GATES}g-spread", "qubits": n, "gates": len(ops),
                   "state_bytes": (1 << n) * 16, "fused_passes": npasses, "single_gate_launches": nsingle,
                   "knobs": eng.knobs(vec, n).to_json(), "knobs_source": knob_source(eng, vec, n),
                   "l2": f"inputs larger than L2 ({(1 << n) * 16 / 2**30:g} GiB state vs 126 MB L2)",
                   "parallelism": f"replicas x{ws}" if ws > 1 else "single GPU"},
        "hbm_gbs_effective": npasses * bytes_per_pass / (ms / 1e3) / 1e9,
        "roofline": {"bound": "fp64", "kernel": "qs_pass", "achieved": fp64_achieved, "peak": fp64_peak,
                     "unit": "TFLOP/s", "frac": fp64_achieved / fp64_peak, "peak_source": fp64_src,
                     "traffic": ncu_traffic(n), "algorithmic_flops_per_launch": flops / max(1, len(pass_list)),
                     "avg_launch_ms": avg_pass_ms,
                     "note": "a fused pass applies ~20 merged ops per HBM round trip, so FP64 issue, not HBM, "
                             "bounds it; roofline_hbm gives the HBM view"},
        "roofline_hbm": {"bound": "hbm", "kernel": "qs_pass", "achieved": achieved, "peak": peak,
                         "unit": "GB/s", "frac": achieved / peak, "peak_source": peak_kind, "traffic": ncu_traffic(n),
                         "algorithmic_bytes_per_launch": bytes_per_pass, "avg_launch_ms": avg_pass_ms},
        "e2e": {"value": ws * len(ops) / e2e_s, "unit": "gates/s", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": 8},
        "gpu_launches": int(launches),
        "clocks": clk.summary(),
        "jit": jit_info,
    }
    if not args.no_extra:
        line["single_gate_sweep"] = gate_sweep(eng, vec, n, ws)
    del sim, vec
    torch.cuda.empty_cache()
    if not args.no_extra:
        s64 = StateVectorSimulator("GPU", "single", gpu_device_id=local, sync=False)
        s64.initial_circuit(circuit)
        s64.initial_state_vector()
        line["single_gate_sweep_c64"] = gate_sweep(s64.engine, s64._vector, n, ws)
        del s64
        torch.cuda.empty_cache()
    if not args.no_extra:
        line["c64"] = []
        for nq in (30, 32):
            row = sv_rate(nq, "single", local, ws)
            row.update(c64_error(nq, local))
            line["c64"].append(row)
    if not args.no_extra:
        line["public_api_runs"] = small_runs_bench(ws, local)
    if not args.no_grad:
        line["adjoint"] = grad_bench(ws, rank, local)
        line["qaoa"] = qaoa_bench(ws, rank, local, args.qaoa_instances, graph_too=args.qaoa_graph)
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        torch.cuda.empty_cache()
        cb = CpuBaseline(circuit, n)
        cb.sample(rounds=1, record=False)  # first touch of the host state
        secs = cb.sample(rounds=args.ref_rounds, budget_s=args.ref_budget)
        r, per, timed = cb.estimate()
        line["cpu_baseline"] = {"value": r, "unit": "gates/s", "cores": cb.threads(), "kind": "port",
                                "s_per_gate_by_class": per, "sample": cb.describe(timed, secs)}
        if args.ref_one_thread:
            line["cpu_baseline_1thread"] = one_thread_baseline(lambda q: spread_circuit(q, N_GATES, SEED), n=n)
    if rank == 0:
        # short summaries first: a reader of the line's head sees them
        head = {k: line[k] for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step")}
        for key in ("single_gate_sweep", "single_gate_sweep_c64"):
            if key in line:
                head[key + "_summary"] = {"min_frac": line[key]["min_frac"], "median_frac": line[key]["median_frac"]}
        head.update(line)
        print(json.dumps(head), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--qubits", type=int, default=N_QUBITS)
    ap.add_argument("--ref-rounds", type=int, default=2,
                    help="CPU baseline: gates timed per gate class (one per round)")
    ap.add_argument("--ref-budget", type=float, default=40.0, help="CPU baseline: seconds at most")
    ap.add_argument("--ref-one-thread", type=int, default=1,
                    help="also time the port on one thread (26 qubits, scaled to 30)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-grad", action="store_true", help="skip the gradient sections (ansatz batch, QAOA batch)")
    ap.add_argument("--tile-bits", type=int, default=None, help="fused tile width k (default: the tuning cache)")
    ap.add_argument("--merge-bits", type=int, default=None,
                    help="gate-merging block width (0 disables; default: the tuning cache)")
    ap.add_argument("--no-extra", action="store_true", help="skip the complex64 30q / 32q runs")
    ap.add_argument("--qaoa-instances", type=int, default=512)
    ap.add_argument("--qaoa-graph", action="store_true",
                    help="also time the QAOA batch as per-instance kernel chains in one CUDA graph")
    ap.add_argument("--max-pass-cost", type=float, default=None,
                    help="fusion width: per-pass arithmetic bound in dense-1q-gate units (default: the tuning cache)")
    ap.add_argument("--jit", type=int, default=1,
                    help="1: fused passes run as run-time compiled kernels (compiled during warm-up); 0: generic kernels")
    args = ap.parse_args()
    if args.impl == "reference":
        rank = int(os.environ.get("RANK", "0"))
        run_reference(args, int(os.environ.get("WORLD_SIZE", "1")), rank)
        return
    ws, rank, local = dist_init(args)
    from quict_b200 import _native as N
    N.jit_set_mode(N.QS_JIT_ASYNC if args.jit else N.QS_JIT_OFF)
    try:
        run_ours(args, ws, rank, local)
    finally:
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()

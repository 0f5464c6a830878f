"""bench.py's pure helpers on CPU: the single-gate byte rule, the per-op flop
rule behind the FP64 roofline, the sweep positions and the peak source."""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


def test_sweep_positions_fit_the_vector():
    for n in (12, 26, 30, 32):
        bits = bench._sweep_bits(n)
        assert all(0 <= b < n for (b,) in bits) and len(set(bits)) == len(bits)
        assert (0,) in bits and (n - 1,) in bits
        pairs = bench._sweep_pairs(n)
        assert all(a != b and max(a, b) < n for a, b in pairs) and len(set(pairs)) == len(pairs)
    assert bench._sweep_bits(30) == [(0,), (1,), (2,), (4,), (5,), (10,), (20,), (29,)]


def test_sweep_byte_rule():
    n, s = 30, 16
    full = 2 * (1 << n) * s
    assert bench.sweep_bytes("h", (0,), n, s) == full
    assert bench.sweep_bytes("rzz", (20, 10), n, s) == full
    # CX: the control=1 half is skipped only when its runs fill whole 32-byte sectors
    assert bench.sweep_bytes("cx", (0, 5), n, s) == full          # 1 amplitude (16 B) runs
    assert bench.sweep_bytes("cx", (1, 5), n, s) == full // 2     # 2 amplitudes = 32 B
    assert bench.sweep_bytes("cz", (10, 20), n, s) == full // 4
    assert bench.sweep_bytes("swap", (29, 0), n, s) == full       # lower bit 0: 16 B runs
    assert bench.sweep_bytes("swap", (29, 28), n, s) == full // 2


def test_flop_rule_per_op():
    from quict_b200.core import CX, CZ, H, Rz, Swap, U3, Unitary
    from quict_b200.simulation.lowering import lower_gate
    n = 6
    (h,) = lower_gate(H & 0, n)
    assert bench.op_flops(h) == 8 * 2 - 2
    (cx,) = lower_gate(CX & [0, 1], n)
    assert bench.op_flops(cx) == 0.0                  # a plain exchange
    (cz,) = lower_gate(CZ & [0, 1], n)
    assert bench.op_flops(cz) == 6 * 0.5 * 0.5        # one of two entries != 1, one control
    (rz,) = lower_gate(Rz(0.3) & 2, n)
    assert bench.op_flops(rz) == 6
    (sw,) = lower_gate(Swap & [1, 4], n)
    assert bench.op_flops(sw) == 0.0
    u = np.linalg.qr(np.random.default_rng(0).normal(size=(4, 4)) + 1j)[0]
    (g2,) = lower_gate(Unitary(u) & [0, 3], n)
    assert bench.op_flops(g2) == 8 * 4 - 2
    (u3,) = lower_gate(U3(0.1, 0.2, 0.3) & 5, n)
    assert bench.op_flops(u3) == 14


def test_peak_source_and_plan_of_the_bench_circuit():
    peak, kind = bench.peaks()
    assert peak > 1000 and kind in ("measured", "fallback")
    from quict_b200.simulation.fusion import Pass, plan
    from quict_b200.simulation.lowering import lower_circuit
    from quict_b200.workloads import spread_circuit
    n = 30
    ops = lower_circuit(spread_circuit(n, bench.N_GATES, bench.SEED).gates, n)
    steps = plan(ops, n, 11, 5, merge_bits=2)
    passes = [s for s in steps if isinstance(s, Pass)]
    assert passes and all(bench.pass_flops(p, n) > 0 for p in passes)


def _max_worker(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench as b
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=30))
    try:
        b.barrier(world)
        q.put((rank, b.max_over_ranks(1.5 + rank, world)))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_with_two_gloo_ranks():
    """The timing reduction every multi-rank bench line uses: the max over ranks."""
    import socket
    import torch.multiprocessing as mp
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_max_worker, args=(r, 2, port, q), daemon=True) for r in range(2)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(60)
        assert p.exitcode == 0
    assert res == {0: 2.5, 1: 2.5}
    assert bench.max_over_ranks(3.25, 1) == 3.25

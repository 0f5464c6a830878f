"""Batch sharding over 2 ranks with the gloo backend on CPU: the partition,
the result gather, and a rank that fails mid-run (failure is detected on the
host through a short process-group timeout, not on a GPU)."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from oracle import observe as oobs


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _init(rank, world, port, timeout_s=30):
    import datetime
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=timeout_s))


def _energies_worker(rank, world, port, q):
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    from quict_b200.distributed import run_sharded
    from quict_b200.differentiation import hardware_efficient_ansatz, ising_observable, rotation
    _init(rank, world, port)
    circ, obs = hardware_efficient_ansatz(4, 1), ising_observable(4)
    params = np.random.default_rng(0).uniform(0, 6, (7, circ.num_params))
    h = obs.matrix()

    def fn(idx):
        rows = []
        for i in idx:
            mats = [(e.matrix if e.kind == "fixed" else rotation(e.kind, params[i, e.index]), list(e.qubits))
                    for e in circ.entries]
            rows.append([oobs.energy(mats, 4, h), float(rank)])
        return torch.tensor(rows, dtype=torch.float64).reshape(-1, 2)

    out = run_sharded(fn, costs=[1.0 + (i % 3) for i in range(7)])
    q.put((rank, out.numpy()))
    dist.destroy_process_group()


def test_sharded_energies_gather_in_order():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_energies_worker, args=(r, world, port, q), daemon=True) for r in range(world)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(60)
        assert p.exitcode == 0
    a, b = res[0], res[1]
    np.testing.assert_array_equal(a, b)              # every rank holds the gathered result
    assert set(a[:, 1]) == {0.0, 1.0}                # both ranks computed rows
    from quict_b200.differentiation import hardware_efficient_ansatz, ising_observable, rotation
    circ, obs = hardware_efficient_ansatz(4, 1), ising_observable(4)
    params = np.random.default_rng(0).uniform(0, 6, (7, circ.num_params))
    for i in range(7):
        mats = [(e.matrix if e.kind == "fixed" else rotation(e.kind, params[i, e.index]), list(e.qubits))
                for e in circ.entries]
        assert abs(a[i, 0] - oobs.energy(mats, 4, obs.matrix())) < 1e-12


def test_balanced_and_block_shards_cover_everything():
    from quict_b200.distributed import balanced_shard, block_shard
    costs = [2.0 ** n for n in np.random.default_rng(1).choice(range(10, 25, 2), 512)]
    parts = balanced_shard(costs, 8)
    assert sorted(i for p in parts for i in p) == list(range(512))
    loads = [sum(costs[i] for i in p) for p in parts]
    assert max(loads) <= 1.05 * (sum(costs) / 8) + max(costs)
    blocks = [block_shard(1000, 3, r) for r in range(3)]
    assert [len(b) for b in blocks] == [334, 333, 333] and blocks[2].stop == 1000


def _failing_worker(rank, world, port, q):
    import datetime
    _init(rank, world, port, timeout_s=5)
    try:
        if rank == 1:
            raise RuntimeError("rank 1 fails before the gather")
        t = torch.ones(2)
        dist.all_reduce(t)       # rank 1 never joins: ends with an error after the timeout
        q.put((rank, "no error"))
    except Exception as e:       # noqa: BLE001 - reported to the parent
        q.put((rank, type(e).__name__))


def test_failed_rank_is_detected_by_timeout():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_failing_worker, args=(r, world, port, q), daemon=True) for r in range(world)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(60)
        if p.is_alive():
            p.kill()
    assert res[1] == "RuntimeError"
    assert res[0] != "no error"

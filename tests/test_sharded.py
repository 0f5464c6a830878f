"""State vector sharded by its top bits over 2 and 4 gloo ranks on CPU.

The local shard work runs through a numpy stand-in for the CUDA engine (the
FP64 oracle's matrix application), so these tests check the sharding logic:
op placement against the bit map, rank-bit controls and diagonals, the
pairwise half-shard exchanges, chunked exchanges, the final re-ordering and
the cross-rank reductions, against the oracle on the whole vector.  The CUDA
engine path of the same class is the one the product uses."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


class _NumpyShard:
    """Local backend: ops on one shard with the oracle (vector bits)."""

    def apply_ops(self, vec, n, ops):
        from oracle import sv as osv
        v = vec.numpy().astype(np.complex128)
        for op in ops:
            u = op.dense()
            if op.cbits:
                d = u.shape[0] << len(op.cbits)
                f = np.eye(d, dtype=np.complex128)
                f[d - u.shape[0]:, d - u.shape[0]:] = u
                u = f
            bits = list(op.cbits) + list(op.tbits)
            v = osv.apply_matrix(v, n, u, [n - 1 - b for b in bits])
        vec.copy_(torch.from_numpy(v.astype(vec.numpy().dtype)))

    def norm2(self, vec, n):
        return float(np.sum(np.abs(vec.numpy()) ** 2))

    def prob0(self, vec, n, bit):
        v = vec.numpy()
        idx = np.arange(v.size)
        return float(np.sum(np.abs(v[(idx >> bit) & 1 == 0]) ** 2))

    def collapse(self, vec, n, bit, outcome, scale):
        v = vec.numpy()
        idx = np.arange(v.size)
        hit = ((idx >> bit) & 1) == outcome
        v[hit] *= scale
        v[~hit] = 0

    def reset(self, vec, n, bit, p0):
        v = vec.numpy()
        idx = np.arange(v.size)
        zero, one = idx[((idx >> bit) & 1) == 0], idx[((idx >> bit) & 1) == 1]
        alpha = np.sqrt(p0)
        if alpha < 1e-6:
            v[zero] = v[one]
        else:
            v[zero] /= alpha
        v[one] = 0

    def sample_indices(self, vec, n, uniforms, mode):
        # smallest i with u * (shard mass) <= CDF[i] over this shard's masses
        from oracle import sv as osv
        return torch.as_tensor(osv.sample_cdf(vec.numpy().astype(np.complex128), uniforms.numpy()))


def _circuit(n, seed, size):
    from quict_b200.core import Circuit, GATE_BY_NAME
    from quict_b200.core.gate import GateType
    types = [GateType[nm] for nm, g in GATE_BY_NAME.items()
             if nm not in ("measure", "reset", "barrier", "id", "unitary", "qft", "iqft", "perm", "perm_fx")
             and g.controls + g.targets <= 3]
    c = Circuit(n)
    c.random_append(size, typelist=types, seed=seed)
    return c


def _worker(rank, world, port, n, seed, chunk, q, precision="double"):
    import datetime
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        from quict_b200.simulation.sharded import ShardedStateVector
        sv = ShardedStateVector(n, precision, backend=_NumpyShard(), chunk_bytes=chunk)
        c = _circuit(n, seed, 80)
        sv.run(c)
        probs = [sv.prob0(qb) for qb in range(n)]  # before re-ordering: global and local bits
        norm = sv.norm2()
        ex = sv.exchanges
        shots = sv.sample(500, uniforms=np.random.default_rng(seed + 100).random(500))
        full = sv.gather(0)
        q.put((rank, full, probs, norm, ex, list(sv.where), shots))
    except Exception as e:  # noqa: BLE001 - reported to the parent
        q.put((rank, repr(e), None, None, None, None, None))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,n,seed,chunk,precision", [(2, 5, 0, 1 << 28, "double"), (2, 7, 1, 64, "double"),
                                                          (4, 6, 2, 1 << 28, "double"), (4, 7, 3, 48, "double"),
                                                          (2, 6, 4, 40, "single")])
def test_sharded_vector_matches_the_oracle(world, n, seed, chunk, precision):
    from conftest import oracle_gates
    from oracle import sv as osv
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, n, seed, chunk, q, precision), daemon=True) for r in range(world)]
    for p in procs:
        p.start()
    res = {}
    for _ in procs:
        r = q.get(timeout=180)
        res[r[0]] = r[1:]
    for p in procs:
        p.join(60)
        assert p.exitcode == 0
    for r in range(world):
        assert not isinstance(res[r][0], str), res[r][0]
    c = _circuit(n, seed, 80)
    ref = osv.run(oracle_gates(c), n)
    full, probs, norm, ex, where, shots = res[0]
    tol = 1e-12 if precision == "double" else 1e-5
    np.testing.assert_allclose(full, ref, rtol=0, atol=tol)
    u = np.random.default_rng(seed + 100).random(500)
    want = osv.sample_cdf(ref, u)
    ties = osv.near_ties(ref, u, tol)
    assert np.all((shots == want) | ties)
    for r in range(1, world):
        np.testing.assert_array_equal(res[r][5], shots)  # every rank holds all shots
    assert where == list(range(n))
    assert abs(norm - 1) < 10 * tol
    for qb in range(n):
        b = n - 1 - qb
        want = float(np.sum(np.abs(ref[(np.arange(1 << n) >> b) & 1 == 0]) ** 2))
        assert abs(probs[qb] - want) < 10 * tol
    assert ex > 0  # the circuit moved data across ranks
    for r in range(1, world):
        assert res[r][0] is None and res[r][1] == probs


def test_placement_of_rank_bit_controls_and_diagonals():
    """Without any process group: an op placed on rank 1 of 2 (top bit = 1)."""
    from quict_b200.simulation.lowering import Op
    from quict_b200.simulation.sharded import ShardedStateVector
    sv = ShardedStateVector.__new__(ShardedStateVector)
    sv.n, sv.nl, sv.g, sv.rank, sv.world = 4, 3, 1, 1, 2
    sv.where = list(range(4))
    # control on the rank bit (1 here): the op runs without it
    op = sv._place(Op("antidiag", (0,), (3,), np.array([[0, 1], [1, 0]], dtype=complex)), [])
    assert op.tbits == (0,) and op.cbits == ()
    sv.rank = 0
    assert sv._place(Op("antidiag", (0,), (3,), np.array([[0, 1], [1, 0]], dtype=complex)), []) is None
    # Rzz-like diagonal on (global 3, local 1): entries with the rank bit fixed
    d = np.array([1, 2, 3, 4], dtype=complex)
    op = sv._place(Op("diag", (3, 1), (), d), [])
    assert op.tbits == (1,) and list(op.mat) == [1, 2]
    sv.rank = 1
    op = sv._place(Op("diag", (3, 1), (), d), [])
    assert list(op.mat) == [3, 4]
    # diagonal on the rank bit alone: one phase, on a local control if there is one
    op = sv._place(Op("diag", (3,), (2,), np.array([1, 1j])), [])
    assert op.tbits == (2,) and op.cbits == () and list(op.mat) == [1, 1j]
    op = sv._place(Op("diag", (3,), (), np.array([1, 1j])), [])
    assert op.tbits == (0,) and list(op.mat) == [1j, 1j]
    sv.rank = 0
    assert sv._place(Op("diag", (3,), (), np.array([1, 1j])), []) is None


def test_solo_vector_on_cpu_stand_in():
    """Without a process group: one unsplit vector, same API."""
    from conftest import oracle_gates
    from oracle import sv as osv
    from quict_b200.simulation.sharded import ShardedStateVector
    c = _circuit(6, 9, 50)
    sv = ShardedStateVector(6, backend=_NumpyShard()).run(c)
    ref = osv.run(oracle_gates(c), 6)
    np.testing.assert_allclose(sv.gather(), ref, rtol=0, atol=1e-12)
    assert sv.exchanges == 0 and abs(sv.norm2() - 1) < 1e-12


@pytest.mark.gpu
@pytest.mark.parametrize("precision,tol", [("double", 1e-12), ("single", 1e-5)])
def test_solo_vector_on_the_gpu_engine(cuda_ok, precision, tol):
    """The default backend (the CUDA engine) drives the shard: one process, no
    process group, a 12-qubit circuit with 1-3 qubit gates."""
    from conftest import oracle_gates
    from oracle import sv as osv
    from quict_b200.simulation.sharded import ShardedStateVector
    c = _circuit(12, 4, 120)
    sv = ShardedStateVector(12, precision).run(c)
    ref = osv.run(oracle_gates(c), 12)
    np.testing.assert_allclose(sv.gather(), ref, rtol=0, atol=tol)
    assert abs(sv.norm2() - 1) < 10 * tol
    want = float(np.sum(np.abs(ref[: 1 << 11]) ** 2))  # qubit 0 = vector bit 11
    assert abs(sv.prob0(0) - want) < 10 * tol
    u = np.random.default_rng(8).random(1000)
    shots = sv.sample(1000, uniforms=u)
    ties = osv.near_ties(ref, u, 1e-12 if precision == "double" else 1e-5)
    assert np.all((shots == osv.sample_cdf(ref, u)) | ties)
    # mid-circuit measure (given uniform) and reset through the engine's kernels
    ref, one = osv.measure(ref, 12, 3, 0.37)
    assert sv.measure(3, 0.37) == one
    ref = osv.reset(ref, 12, 5)
    sv.reset(5)
    np.testing.assert_allclose(sv.gather(), ref, rtol=0, atol=10 * tol)


def test_exchange_choice_looks_ahead():
    """Dry run of the placement (bit map only): a rank bit is traded for the
    local bit whose next dense use is farthest away, so a spread
    circuit (targets mostly in the low and high bits) needs about one
    exchange per rank bit instead of one per dense gate on a rank bit."""
    from quict_b200.simulation.lowering import lower_circuit
    from quict_b200.simulation.sharded import ShardedStateVector
    from quict_b200.workloads import spread_circuit

    class Dry(ShardedStateVector):
        def __init__(self, n, world):
            self.n, self.world, self.rank = n, world, 0
            self.g = world.bit_length() - 1
            self.nl = n - self.g
            self.where = list(range(n))
            self.exchanges = 0

        def exchange(self, gbit, lbit):
            self._swap_roles(gbit, lbit)
            self.exchanges += 1

        def _flush(self, pending):
            pending.clear()

    n = 24
    ops = lower_circuit(spread_circuit(n, 600, seed=3).gates, n)
    for world in (2, 8):
        d = Dry(n, world)
        d.apply_ops(ops)
        hits = sum(1 for o in ops if o.kind != "diag" and any(b >= d.nl for b in o.tbits))
        assert 0 < d.exchanges <= 2 * d.g < hits
        assert sorted(d.where) == list(range(n))


def _mr_plan(n, seed):
    """Segments of gates, each followed by a measure or reset of one qubit
    (a measure is sometimes followed by a reset of the same qubit, which
    reaches the |1> -> |0> move when the outcome was 1)."""
    rng = np.random.default_rng(seed)
    plan = []
    for k in range(10):
        seg = _circuit(n, seed * 100 + k, 12)
        q = int(rng.integers(n))
        plan.append((seg, "measure", q))
        if rng.random() < 0.5:
            plan.append((None, "reset", q))
        else:
            plan.append((None, "reset", int(rng.integers(n))))
    return plan


def _mr_worker(rank, world, port, n, seed, q):
    import datetime
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        from quict_b200.simulation.sharded import ShardedStateVector
        sv = ShardedStateVector(n, "double", backend=_NumpyShard(), seed=seed)
        log = []
        for seg, what, qb in _mr_plan(n, seed):
            if seg is not None:
                sv.run(seg)
            on_rank_bit = sv.where[n - 1 - qb] >= sv.nl
            if what == "measure":
                log.append(("measure", qb, sv.measure(qb), on_rank_bit))
            else:
                sv.reset(qb)
                log.append(("reset", qb, None, on_rank_bit))
        q.put((rank, sv.gather(0), log))
    except Exception as e:  # noqa: BLE001 - reported to the parent
        q.put((rank, repr(e), None))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,n,seed", [(2, 5, 11), (4, 6, 12)])
def test_midcircuit_measure_and_reset_across_ranks(world, n, seed):
    from conftest import oracle_gates
    from oracle import sv as osv
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_mr_worker, args=(r, world, port, n, seed, q), daemon=True) for r in range(world)]
    for p in procs:
        p.start()
    res = {}
    for _ in procs:
        r = q.get(timeout=180)
        res[r[0]] = r[1:]
    for p in procs:
        p.join(60)
        assert p.exitcode == 0
    full, log = res[0]
    assert not isinstance(full, str), full
    # replay with the oracle and rank 0's uniform stream
    rng = np.random.default_rng(seed)
    v = osv.zero_state(n)
    for (seg, what, qb), (w2, q2, outcome, _) in zip(_mr_plan(n, seed), log):
        assert (what, qb) == (w2, q2)
        if seg is not None:
            v = osv.run(oracle_gates(seg), n, vec=v)
        if what == "measure":
            v, one = osv.measure(v, n, qb, float(rng.random()))
            assert one == outcome
        else:
            v = osv.reset(v, n, qb)
    np.testing.assert_allclose(full, v, rtol=0, atol=1e-12)
    assert any(flag for *_, flag in log) and not all(flag for *_, flag in log)  # both paths ran
    for r in range(1, world):
        assert res[r][1] == log

"""The persistent batch kernel (qs_batch_plan / qs_batch_launch): many
gradient problems of uneven size in one launch.

GPU: energies and gradients against per-instance complex128 adjoint runs
(themselves pinned to the FP64 oracle's parameter shift in test_grad.py and
test_benchmark_sizes.py), replays in a CUDA graph, and the bounded wait: a
work item whose dependency count can never be reached gives up after the
timeout, records itself in the control words and the launch ends.
CPU: the planner's validation and sizes (no device needed)."""
import ctypes as C

import numpy as np
import pytest

from quict_b200 import _native as N


def _qaoa(ns, seed=1234, depths=(1, 6)):
    from quict_b200.differentiation import qaoa_instances
    inst = []
    for j, n in enumerate(ns):
        inst += qaoa_instances(1, sizes=(n,), depths=depths, seed=seed + 17 * j + n)
    return inst


def _reference(inst):
    from quict_b200.differentiation import BatchedAdjoint, maxcut_observable, qaoa_circuit
    out = []
    for n, edges, p, prm in inst:
        eng = BatchedAdjoint(qaoa_circuit(n, edges, p), maxcut_observable(n, edges), "double")
        e, g = eng.gradient(prm[None, :])
        out.append((float(e[0]), g[0].cpu().numpy()))
    return out


@pytest.mark.gpu
def test_persistent_c64_matches_per_instance_c128_up_to_24_qubits(cuda_ok):
    """Uneven-batch sizes (10..24 qubits, two of 24, depths 1..6) in one launch,
    complex64, against per-instance complex128 gradients."""
    import torch
    from quict_b200.differentiation import UnevenQAOABatch
    inst = _qaoa((10, 12, 14, 16, 18, 20, 22, 24, 24, 10, 12))
    batch = UnevenQAOABatch(inst, "single", mode="persistent")
    batch.capture()
    batch.replay()
    torch.cuda.synchronize()
    res = batch.results()
    assert batch.captured_launches == 1
    # the problems of >= 20 qubits run as generated functions in the linked kernel
    assert batch.persistent.sizes.jit_fns > 0 and batch.persistent.linked
    for (n, edges, p, _), (e, g), (e2, g2) in zip(inst, res, _reference(inst)):
        scale = max(1.0, len(edges))
        assert abs(e - e2) < 1e-5 * scale, (n, p, e, e2)
        np.testing.assert_allclose(g, g2, rtol=0, atol=1e-4 * scale, err_msg=f"n={n} p={p}")


@pytest.mark.gpu
@pytest.mark.parametrize("caps", [(9, 9), (10, 11), (11, 12), (12, 12)])
def test_persistent_c128_matches_per_instance_c128(cuda_ok, caps):
    """complex128 in one launch against per-instance complex128 runs, for
    several tile-width caps (forward, pair): 1e-10."""
    from quict_b200.differentiation import BatchedAdjoint, maxcut_observable, qaoa_circuit
    from quict_b200.differentiation.persistent import PersistentBatch
    inst = _qaoa((10, 12, 14, 16, 18), seed=77)
    engines = [BatchedAdjoint(qaoa_circuit(n, e, p), maxcut_observable(n, e), "double") for n, e, p, _ in inst]
    pb = PersistentBatch([(eng, prm) for eng, (_, _, _, prm) in zip(engines, inst)], "double", caps=caps)
    pb.launch()
    res = pb.results()
    for (n, edges, p, _), (e, g), (e2, g2) in zip(inst, res, _reference(inst)):
        assert abs(e - e2) < 1e-10 * max(1.0, len(edges)), (n, p)
        np.testing.assert_allclose(g, g2, rtol=0, atol=1e-10 * max(1.0, len(edges)), err_msg=f"n={n} p={p}")


@pytest.mark.gpu
def test_persistent_hea_problems_and_graph_replays_are_identical(cuda_ok):
    """Other circuits than QAOA (the hardware-efficient ansatz with a
    Z/X observable) and bitwise-identical results over graph replays."""
    import torch
    from quict_b200.differentiation import BatchedAdjoint
    from quict_b200.differentiation.persistent import PersistentBatch
    from quict_b200.workloads import hea_problem
    probs, want = [], []
    for n, layers in ((10, 2), (12, 3), (14, 2)):
        circ, obs, params = hea_problem(n, layers, 2)
        ref = BatchedAdjoint(circ, obs, "double")
        e, g = ref.gradient(params[:1])
        want.append((float(e[0]), g[0].cpu().numpy()))
        probs.append((BatchedAdjoint(circ, obs, "single"), params[0]))
    pb = PersistentBatch(probs, "single")
    pb.capture()
    outs = []
    for _ in range(2):
        pb.replay()
        torch.cuda.synchronize()
        outs.append(pb.results())
    for (e, g), (e2, g2) in zip(outs[0], outs[1]):
        assert e == e2 and np.array_equal(g, g2)
    for (e, g), (e2, g2) in zip(outs[0], want):
        assert abs(e - e2) < 1e-4
        np.testing.assert_allclose(g, g2, rtol=0, atol=1e-4)


@pytest.mark.gpu
def test_persistent_linked_c128_every_stage_generated(cuda_ok):
    """complex128 with EVERY register stage generated and linked into the
    kernel (jit_min_qubits below every problem), QAOA and ansatz problems
    together: the linked kernel runs, and matches per-instance complex128
    runs to 1e-10."""
    import torch
    from quict_b200.differentiation import BatchedAdjoint, maxcut_observable, qaoa_circuit
    from quict_b200.differentiation.persistent import PersistentBatch
    from quict_b200.workloads import hea_problem
    inst = _qaoa((10, 12, 14), seed=91)
    probs = [(BatchedAdjoint(qaoa_circuit(n, e, p), maxcut_observable(n, e), "double"), prm) for n, e, p, prm in inst]
    want = _reference(inst)
    circ, obs, params = hea_problem(11, 2, 1)
    e, g = BatchedAdjoint(circ, obs, "double").gradient(params[:1])
    want.append((float(e[0]), g[0].cpu().numpy()))
    probs.append((BatchedAdjoint(circ, obs, "double"), params[0]))
    pb = PersistentBatch(probs, "double", caps=(11, 11), jit_min_qubits=9)
    assert pb.sizes.jit_fns > 0
    pb.capture()
    pb.replay()
    torch.cuda.synchronize()
    res = pb.results()
    assert pb.linked
    for (e, g), (e2, g2) in zip(res, want):
        assert abs(e - e2) < 1e-9
        np.testing.assert_allclose(g, g2, rtol=0, atol=1e-9)


@pytest.mark.gpu
def test_persistent_wait_that_cannot_finish_times_out(cuda_ok):
    """Patch the plan so that the last work item waits for more items than
    its problem has: the bounded wait gives up after the timeout, control
    word 1 names the item, and the device stays usable."""
    import time

    import torch
    from quict_b200.differentiation import BatchedAdjoint, maxcut_observable, qaoa_circuit
    from quict_b200.differentiation.persistent import PersistentBatch
    inst = _qaoa((10, 12), seed=5)
    engines = [BatchedAdjoint(qaoa_circuit(n, e, p), maxcut_observable(n, e), "single") for n, e, p, _ in inst]
    pb = PersistentBatch([(eng, prm) for eng, (_, _, _, prm) in zip(engines, inst)], "single", timeout_s=0.5)
    blob = pb.blob.cpu().numpy()
    nitems = int(blob[4:8].view(np.int32)[0])
    off_items = int(blob[32:40].view(np.int64)[0])
    last = off_items + 48 * (nitems - 1)  # BItem: 48 bytes; need at byte 16
    blob[last + 16:last + 24] = np.array([1 << 40], dtype=np.int64).view(np.uint8)
    pb.blob.copy_(torch.from_numpy(blob))
    t0 = time.perf_counter()
    pb.launch()
    torch.cuda.synchronize()
    assert time.perf_counter() - t0 < 30
    err = int(pb.ctrl[1].item())
    assert err == (1 << 32) | (nitems - 1)
    with pytest.raises(N.QsimError):
        pb.results()
    x = torch.ones(4, device="cuda")
    assert float(x.sum()) == 4.0


def _tiny_plan_args(n=10, nterms=2, nslots=1, nparams=1, k=10, bwd_k=10, pair=None):
    """A one-problem plan: one forward pass (one diagonal op), one backward
    pair pass (an EXPECT op and a diagonal), H = sum of Z terms."""
    fwd = N.qs_pass()
    fwd.k, fwd.nlow = k, 5
    for j in range(k - 5):
        fwd.hi[j] = 5 + j
    fwd.op_begin, fwd.op_count, fwd.inst_shift, fwd.pair = 0, 1, 0, 0
    bwd = N.qs_pass()
    bwd.k, bwd.nlow = bwd_k, 5
    his = list(range(5, bwd_k - 1)) + [n]  # the pair bit (n) in the tile
    for j, h in enumerate(his):
        bwd.hi[j] = h
    bwd.op_begin, bwd.op_count, bwd.inst_shift, bwd.pair = 1, 2, 0, (n + 1 if pair is None else pair)
    ops = (N.qs_op * 3)()
    for i, (kind, flags) in enumerate(((N.QS_OP_DIAG, 0), (N.QS_OP_EXPECT, N.QS_OPF_DIAG), (N.QS_OP_DIAG, 0))):
        o = ops[i]
        o.kind, o.m, o.flags, o.mat, o.mat_stride, o.slot = kind, 1, flags, 0, 0, 0
        o.gbit[0], o.tgt[0] = 0, 0
        for j in range(1, 4):
            o.gbit[j], o.tgt[j] = 0, -1
    passes = (N.qs_pass * 2)(fwd, bwd)
    inst = (N.qs_batch_inst * 1)()
    inst[0].n, inst[0].fwd_begin, inst[0].nfwd, inst[0].bwd_begin, inst[0].nbwd = n, 0, 1, 1, 1
    inst[0].term_begin, inst[0].nterms, inst[0].nslots, inst[0].nparams, inst[0].w_begin = 0, nterms, nslots, nparams, 0
    x = np.zeros(nterms, dtype=np.uint64)
    z = np.array([1 << (t % n) for t in range(nterms)], dtype=np.uint64)
    c = np.ones(2 * nterms)
    w = np.ones(max(1, nparams * nslots))
    return inst, passes, ops, x, z, c, w


def _plan(inst, passes, ops, x, z, c, w, tiles=4, amps=4096, blob=None, nbytes=0, mats=4, mats_host=None,
          jit_min_qubits=99):
    sizes = N.qs_batch_sizes()
    lib = N.load()
    rc = lib.qs_batch_plan(N.QS_C64, inst, len(inst), passes, len(passes), ops, len(ops), mats, mats_host,
                           jit_min_qubits,
                           x.ctypes.data_as(C.c_void_p), z.ctypes.data_as(C.c_void_p),
                           c.ctypes.data_as(C.c_void_p), len(x), w.ctypes.data_as(C.c_void_p), len(w), tiles, amps,
                           blob, nbytes, C.byref(sizes), None)
    return rc, sizes


def test_planner_sizes_and_blob_without_a_device():
    inst, passes, ops, x, z, c, w = _tiny_plan_args()
    rc, sz = _plan(inst, passes, ops, x, z, c, w)
    assert rc == 0, N.load().qs_last_error()
    assert sz.state_elems == 2 << 10
    assert sz.threads == 32  # tile 2^10 at 32 amplitudes per thread
    assert sz.energy_doubles == 2 and sz.grad_doubles == 1
    # stages: forward (1 tile), HAM (1 item of 1024 amplitudes), backward (2 tiles of the
    # 2^11-amplitude pair vector, 4 tiles per item -> 1 item), FIN
    assert sz.nitems == 4 and sz.nstages == 2
    # EXPECT partials (2 * 1 slot * 2 tiles) + HAM partials (2 * 1 item)
    assert sz.partial_doubles == 6
    blob = np.zeros(int(sz.blob_bytes), dtype=np.uint8)
    rc, _ = _plan(inst, passes, ops, x, z, c, w, blob=blob.ctypes.data_as(C.c_void_p), nbytes=blob.nbytes)
    assert rc == 0
    assert int(blob[4:8].view(np.int32)[0]) == 4
    rc, _ = _plan(inst, passes, ops, x, z, c, w, blob=blob.ctypes.data_as(C.c_void_p), nbytes=16)
    assert rc == N.QS_EWORKSPACE


@pytest.mark.parametrize("bad", ["tiny_tile", "no_pair", "terms", "weights", "item_size", "bwd_tiles"])
def test_planner_rejects_bad_batches(bad):
    kw = {}
    if bad == "tiny_tile":
        kw = dict(n=9, k=9, bwd_k=10)  # complex64 register tiles start at 2^10
    elif bad == "no_pair":
        kw = dict(pair=0)
    args = list(_tiny_plan_args(**kw))
    extra = {}
    if bad == "terms":
        args[0][0].nterms = 0
    elif bad == "weights":
        args[0][0].nparams = 5  # W needs 5 entries, the array has 1
    elif bad == "item_size":
        extra = dict(tiles=0)
    elif bad == "bwd_tiles":
        args[1][1].pair = 3  # the pair bit of a backward pass must be bit n
    rc, _ = _plan(*args, **extra)
    assert rc < 0


def test_generated_stage_functions_compile_and_link_without_a_device():
    """With the host matrix table, the planner generates the register stages
    as device functions; they compile (NVRTC, relocatable) and link with the
    embedded batch kernel (nvJitLink) here, with torch imported first (it
    brings its own, older libnvJitLink)."""
    import torch  # noqa: F401
    args = _tiny_plan_args()
    mats = np.array([1, 1j, 1, -1], dtype=np.complex64)
    rc, sz = _plan(*args, mats_host=C.c_void_p(mats.ctypes.data), jit_min_qubits=0)
    assert rc == 0 and sz.jit_fns == 2 and sz.jit_key != 0
    blob = np.zeros(int(sz.blob_bytes), dtype=np.uint8)
    rc, sz = _plan(*args, blob=blob.ctypes.data_as(C.c_void_p), nbytes=blob.nbytes,
                   mats_host=C.c_void_p(mats.ctypes.data), jit_min_qubits=0)
    assert rc == 0
    nb = C.c_int64()
    rc = N.load().qs_batch_link_check(C.byref(sz), C.byref(nb))
    assert rc == 0, N.load().qs_last_error()
    assert nb.value > 0


def _items(blob):
    """(kind, inst, need) of every work item in a written plan."""
    nitems = int(blob[4:8].view(np.int32)[0])
    off = int(blob[32:40].view(np.int64)[0])
    rec = blob[off:off + 48 * nitems].reshape(nitems, 48)
    kind = rec[:, 0:4].copy().view(np.int32)[:, 0]
    inst = rec[:, 4:8].copy().view(np.int32)[:, 0]
    need = rec[:, 16:24].copy().view(np.int64)[:, 0]
    return kind, inst, need


@pytest.mark.parametrize("group", ["0", "1", "2"])
def test_planner_orders_every_wait_after_its_items(group, monkeypatch):
    """The invariant the persistent kernel's deadlock freedom rests on, for
    three problems and every interleaving: an item waits for exactly the items
    of its problem's earlier stages, all of them come before it in the list,
    no later item belongs to an earlier stage, and each problem's stages run
    forward passes, lam = H psi, backward passes, final reduction in that
    order."""
    monkeypatch.setenv("QS_BATCH_GROUP", group)
    inst, passes, ops, x, z, c, w = _tiny_plan_args()
    three = (N.qs_batch_inst * 3)(inst[0], inst[0], inst[0])
    rc, sz = _plan(three, passes, ops, x, z, c, w, tiles=1, amps=256)
    assert rc == 0
    blob = np.zeros(int(sz.blob_bytes), dtype=np.uint8)
    rc, sz = _plan(three, passes, ops, x, z, c, w, tiles=1, amps=256, blob=blob.ctypes.data_as(C.c_void_p),
                   nbytes=blob.nbytes)
    assert rc == 0
    kind, inst_of, need = _items(blob)
    assert len(kind) == sz.nitems
    for i in range(3):
        seen = []  # (need, kind) of this problem's items so far, in list order
        for k in np.nonzero(inst_of == i)[0]:
            q = int(need[k])
            assert q <= len(seen)                                   # what it waits for precedes it
            assert sum(1 for p, _ in seen if p < q) == q            # exactly the earlier stages' items
            assert all(p <= q for p, _ in seen)                     # stages never go backwards
            seen.append((q, int(kind[k])))
        stage_kinds = [kd for j, (q, kd) in enumerate(seen) if j == 0 or q != seen[j - 1][0]]
        # forward (0), lam = H psi (1), backward (2), final (3)
        assert stage_kinds == [0, 1, 2, 3]

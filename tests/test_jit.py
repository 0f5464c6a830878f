"""Run-time compiled fused passes (qs_apply_fused_ex with the JIT on).

CPU: the generator emits a source for every register launch of a spread
plan, and NVRTC compiles one for sm_100a.  GPU: with the JIT in SYNC mode
(every register pass runs as its generated kernel) the results match the
FP64 oracle and the generic kernels, for every tuner knob set and at the
benchmark's size; ASYNC mode switches to the compiled kernels once they are
built.  Tolerances: 1e-12 (complex128), 1e-5 (complex64)."""
import ctypes as C

import numpy as np
import pytest

from conftest import build_circuit, oracle_gates
from oracle import sv as osv


def _plan_sources(n, esize, gates=300, knobs=None):
    from quict_b200 import _native as N
    from quict_b200.simulation.autotune import default_knobs
    from quict_b200.simulation.fusion import MatrixTable, Pass, emit, iter_plan, relabel_swaps
    from quict_b200.simulation.lowering import lower_circuit
    from quict_b200.workloads import spread_circuit
    lib = N.load()
    kn = knobs or default_knobs(esize)
    ops = relabel_swaps(lower_circuit(spread_circuit(n, gates, 1).gates, n), n)
    passes = [s for s in iter_plan(ops, n, kn.tile_bits, kn.low_bits, merge_bits=kn.merge_bits)
              if isinstance(s, Pass) and s.ops]
    table = MatrixTable()
    cps, npass, cops, nops = emit(passes, table)
    host = table.array().astype(np.complex128 if esize == 16 else np.complex64)
    dt = N.QS_C128 if esize == 16 else N.QS_C64
    out = []
    for i in range(npass):
        li = 0
        while True:
            ln = C.c_int64(0)
            buf = C.create_string_buffer(1 << 21)
            rc = lib.qs_jit_pass_source(n, dt, C.byref(cps[i]), cops, nops, C.c_void_p(host.ctypes.data), host.size,
                                        li, buf, 1 << 21, C.byref(ln))
            if rc != 0:
                break
            assert ln.value == len(buf.value)
            out.append(buf.value.decode())
            li += 1
    return out


def test_generator_emits_every_register_launch_and_nvrtc_compiles_one():
    from quict_b200 import _native as N
    lib = N.load()
    for esize in (16, 8):
        srcs = _plan_sources(20, esize)
        assert len(srcs) >= 3
        for s in srcs:
            assert 'extern "C" __global__' in s and "qs_pass" in s
    nb = C.c_int64(0)
    rc = lib.qs_jit_compile_check(srcs[0].encode(), C.byref(nb))
    if rc == N.QS_ENOTSUP:
        pytest.skip("NVRTC is not available here")
    assert rc == 0, lib.qs_jit_last_log()
    assert nb.value > 1000


@pytest.mark.parametrize("esize", [16, 8])
def test_longest_generated_sources_compile(esize):
    """3-bit merged blocks give the longest row expressions; the launches
    with the most code of such a plan must compile."""
    from quict_b200 import _native as N
    from quict_b200.simulation.autotune import Knobs
    lib = N.load()
    srcs = sorted(_plan_sources(20, esize, gates=400, knobs=Knobs(12 if esize == 16 else 13, 5, 3)), key=len)
    for src in srcs[-2:]:
        nb = C.c_int64(0)
        rc = lib.qs_jit_compile_check(src.encode(), C.byref(nb))
        if rc == N.QS_ENOTSUP:
            pytest.skip("NVRTC is not available here")
        assert rc == 0, lib.qs_jit_last_log()


def test_jit_mode_and_stats_entry_points():
    from quict_b200 import _native as N
    prev = N.jit_set_mode(N.QS_JIT_OFF)
    try:
        assert N.jit_set_mode(N.QS_JIT_SYNC) == N.QS_JIT_OFF
        with pytest.raises(N.QsimError):
            N.jit_set_mode(7)
        st = N.jit_stats()
        assert set(st) == set(N.JIT_STAT_KEYS) and all(v >= 0 for v in st.values())
    finally:
        N.jit_set_mode(prev)


@pytest.fixture
def jit_sync():
    from quict_b200 import _native as N
    prev = N.jit_set_mode(N.QS_JIT_SYNC)
    yield N
    N.jit_set_mode(prev)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["double", "single"])
def test_compiled_passes_vs_oracle_for_every_tuner_knob(cuda_ok, jit_sync, precision):
    from quict_b200.simulation import StateVectorSimulator
    from quict_b200.simulation.autotune import candidates
    from test_sv_gpu import _every_placement_circuit
    N = jit_sync
    esize = 16 if precision == "double" else 8
    tol = 1e-12 if precision == "double" else 1e-5
    cases = []
    for n in (14, 17):
        gl = _every_placement_circuit(n, seed=200 + n)
        cases.append((n, gl, osv.run(oracle_gates(build_circuit(gl, n)), n)))
    # first round in ASYNC mode: generic kernels run while the pool compiles
    # every pass shape in parallel; the second round (SYNC) runs them compiled
    for mode in (N.QS_JIT_ASYNC, N.QS_JIT_SYNC):
        N.jit_set_mode(mode)
        before = N.jit_stats()
        for n, gl, ref in cases:
            for kn in candidates(esize, n):
                s = StateVectorSimulator("GPU", precision, tile_bits=kn.tile_bits, low_bits=kn.low_bits,
                                         merge_bits=kn.merge_bits)
                v = s.run(build_circuit(gl, n, precision)).get()
                err = float(np.max(np.abs(v - ref)))
                assert err < tol, (mode, n, kn, err)
        N.jit_wait(900)
    after = N.jit_stats()
    assert after["compiled_launches"] > before["compiled_launches"], N.load().qs_jit_last_log()
    assert after["failed"] == before["failed"], N.load().qs_jit_last_log()


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["double", "single"])
def test_compiled_passes_match_generic_kernels_at_26_qubits(cuda_ok, precision):
    """The spread circuit at 26 qubits with the shipped knobs: compiled
    passes against the generic register kernel."""
    import torch
    from quict_b200 import _native as N
    from quict_b200.simulation import StateVectorSimulator
    from quict_b200.workloads import spread_circuit
    tol = 1e-12 if precision == "double" else 1e-5
    prev = N.jit_set_mode(N.QS_JIT_OFF)
    try:
        a = StateVectorSimulator("GPU", precision).run(spread_circuit(26, 1000, 1)).tensor
        N.jit_set_mode(N.QS_JIT_ASYNC)  # queue every pass shape for the compile pool
        StateVectorSimulator("GPU", precision).run(spread_circuit(26, 1000, 1))
        N.jit_wait(900)
        N.jit_set_mode(N.QS_JIT_SYNC)
        before = N.jit_stats()["compiled_launches"]
        b = StateVectorSimulator("GPU", precision).run(spread_circuit(26, 1000, 1)).tensor
        assert N.jit_stats()["compiled_launches"] >= before + 10
    finally:
        N.jit_set_mode(prev)
    d = float((a.to(torch.complex128) - b.to(torch.complex128)).abs().max())
    assert d < tol


@pytest.mark.gpu
def test_async_mode_switches_to_compiled_kernels(cuda_ok):
    from quict_b200 import _native as N
    from quict_b200.simulation import StateVectorSimulator
    from quict_b200.workloads import spread_circuit
    prev = N.jit_set_mode(N.QS_JIT_ASYNC)
    try:
        c = spread_circuit(18, 200, 7)
        ref = osv.run(oracle_gates(c), 18)
        v1 = StateVectorSimulator("GPU").run(spread_circuit(18, 200, 7)).get()
        N.jit_wait(600)
        st = N.jit_stats()
        v2 = StateVectorSimulator("GPU").run(spread_circuit(18, 200, 7)).get()
        assert N.jit_stats()["compiled_launches"] > st["compiled_launches"]
        np.testing.assert_allclose(v1, ref, rtol=0, atol=1e-12)
        np.testing.assert_allclose(v2, ref, rtol=0, atol=1e-12)
    finally:
        N.jit_set_mode(prev)


@pytest.mark.gpu
@pytest.mark.parametrize("precision,tol", [("double", 1e-10), ("single", 1e-4)])
def test_compiled_adjoint_passes_match_generic_kernels(cuda_ok, precision, tol):
    """Batched forward passes (per-instance tables staged in shared memory) and
    adjoint pair passes (EXPECT partials) as generated kernels, against the
    generic kernels: a hardware-efficient-ansatz batch and a QAOA instance."""
    from quict_b200 import _native as N
    from quict_b200.differentiation import (BatchedAdjoint, hardware_efficient_ansatz, ising_observable,
                                            maxcut_observable, qaoa_circuit, random_regular_graph)
    circ, obs = hardware_efficient_ansatz(13, 2), ising_observable(13)
    params = np.random.default_rng(8).uniform(0, 2 * np.pi, (4, circ.num_params))
    edges = random_regular_graph(16, 3, np.random.default_rng(3))
    qc, qo = qaoa_circuit(16, edges, 3), maxcut_observable(16, edges)
    prm = np.random.default_rng(9).uniform(0, 3, (1, qc.num_params))
    prev = N.jit_set_mode(N.QS_JIT_OFF)
    try:
        want = [BatchedAdjoint(circ, obs, precision).gradient(params),
                BatchedAdjoint(qc, qo, precision).gradient(prm)]
        N.jit_set_mode(N.QS_JIT_ASYNC)  # compile every shape on the pool, then run them compiled
        for c, o, p in ((circ, obs, params), (qc, qo, prm)):
            BatchedAdjoint(c, o, precision).gradient(p)
        N.jit_wait(900)
        N.jit_set_mode(N.QS_JIT_SYNC)
        before = N.jit_stats()
        got = [BatchedAdjoint(circ, obs, precision).gradient(params),
               BatchedAdjoint(qc, qo, precision).gradient(prm)]
        after = N.jit_stats()
    finally:
        N.jit_set_mode(prev)
    assert after["compiled_launches"] > before["compiled_launches"] and after["failed"] == before["failed"]
    for (e0, g0), (e1, g1), scale in zip(want, got, (1.0, float(len(edges)))):
        np.testing.assert_allclose(e1.cpu().numpy(), e0.cpu().numpy(), rtol=0, atol=tol * scale)
        np.testing.assert_allclose(g1.cpu().numpy(), g0.cpu().numpy(), rtol=0, atol=4 * tol * scale)

"""Parity at the sizes the benchmark runs (bench.py).

* The 1000-gate spread circuit (10% Haar 2-qubit unitaries): at 30 qubits the
  fused run against the per-gate kernels (independent code paths), complex64
  against complex128, and the first 24 gates against the CPU port of the
  reference kernels on every amplitude; at 32 qubits (amplitude indices past
  2^31) complex64 against complex128 and fused against per-gate.  The fused
  runs use the shipped tuning-cache knobs.
* Every fused-pass knob the autotuner can pick, in both precisions, against
  the FP64 oracle.
* The noisy density matrix in full: 12 qubits, 150 noisy gates, against the
  FP64 superoperator oracle.
* The hardware-efficient-ansatz gradient in full: 16 qubits, 8 layers, 256
  parameters, two parameter sets; energies and adjoint gradients against the
  FP64 oracle's parameter shift.
* The uneven QAOA batch with instances up to 24 qubits: the batched complex64
  graph against per-instance complex128 runs.

Tolerances: amplitudes 1e-12 (c128) / 1e-5 (c64); gradients 1e-10 (c128) /
1e-4 (c64) of the FP64 oracle."""
import os

import numpy as np
import pytest

from conftest import oracle_gates
from oracle import dm as odm
from oracle import observe as oobs
from oracle import sv as osv

pytestmark = pytest.mark.gpu

GiB = 1 << 30


def _max_abs_diff(a, b, chunk=1 << 27):
    """max |a - b| over two device vectors (either precision), in chunks so no
    full-size temporary is made."""
    import torch
    m = 0.0
    for i in range(0, a.numel(), chunk):
        x = a[i:i + chunk].to(torch.complex128)
        y = b[i:i + chunk].to(torch.complex128)
        m = max(m, float((x - y).abs().max()))
    return m


def _free_gpu_bytes():
    import torch
    torch.cuda.empty_cache()
    free, _ = torch.cuda.mem_get_info()
    return free


def _z_expectations(sim, bits):
    """<Z> on the given vector bits, from FP64 P(bit = 0) reductions."""
    return np.array([2 * sim.engine.prob0(sim._vector, sim._qubits, b) - 1 for b in bits])


def _sim(precision="double", **kw):
    from quict_b200.simulation import StateVectorSimulator
    return StateVectorSimulator("GPU", precision, **kw)


def test_spread_30q_fused_vs_per_gate_and_c64_vs_c128(cuda_ok):
    import torch
    from quict_b200.workloads import spread_circuit
    n = 30
    if _free_gpu_bytes() < 40 * GiB:
        pytest.skip("needs 40 GiB of free device memory")
    a = _sim()
    va = a.run(spread_circuit(n, 1000, 1)).tensor
    b = _sim(fusion=False)
    vb = b.run(spread_circuit(n, 1000, 1)).tensor
    assert _max_abs_diff(va, vb) < 1e-12
    del b, vb
    torch.cuda.empty_cache()
    s = _sim("single")
    vs = s.run(spread_circuit(n, 1000, 1)).tensor
    assert _max_abs_diff(va, vs) < 1e-5
    bits = [0, 4, 15, 25, 29]
    dz = np.abs(_z_expectations(a, bits) - _z_expectations(s, bits))
    assert dz.max() < 1e-5
    assert abs(a.get_measured_prob(0, all_measured=True) - 1) < 1e-12


def test_spread_30q_prefix_vs_cpu_port(cuda_ok):
    """The first 24 gates at 30 qubits against the numba port of the reference
    CPU kernels (oracle/ref_port.py) on the host, on all 2^30 amplitudes."""
    import psutil
    from oracle import ref_port
    from quict_b200.core import Circuit
    from quict_b200.simulation.lowering import lower_circuit
    from quict_b200.workloads import spread_circuit
    n = 30
    if psutil.virtual_memory().available < 48 * GiB:
        pytest.skip("needs 48 GiB of free host memory (two 16 GiB vectors)")
    full = spread_circuit(n, 1000, 1)
    pre = Circuit(n)
    pre.gates = full.gates[:24]
    v = _sim().run(pre).get()
    host = osv.zero_state(n)
    ref_port.run(host, ref_port.prepare(lower_circuit(pre.gates, n), np.complex128))
    err = 0.0
    for i in range(0, host.size, 1 << 26):
        err = max(err, float(np.max(np.abs(v[i:i + (1 << 26)] - host[i:i + (1 << 26)]))))
    assert err < 1e-12


def test_spread_32q_c64_vs_c128_and_fused_vs_per_gate(cuda_ok):
    """32 qubits: complex64 (32 GiB) against complex128 (64 GiB), and the
    complex128 fused run against the per-gate kernels (another 64 GiB)."""
    import torch
    from quict_b200.workloads import spread_circuit
    n = 32
    if _free_gpu_bytes() < 140 * GiB:
        pytest.skip("needs 140 GiB of free device memory")
    a = _sim()
    va = a.run(spread_circuit(n, 1000, 1)).tensor
    s = _sim("single")
    vs = s.run(spread_circuit(n, 1000, 1)).tensor
    assert _max_abs_diff(va, vs) < 1e-5
    bits = [0, 4, 16, 27, 31]
    assert np.abs(_z_expectations(a, bits) - _z_expectations(s, bits)).max() < 1e-5
    del s, vs
    torch.cuda.empty_cache()
    b = _sim(fusion=False)
    vb = b.run(spread_circuit(n, 1000, 1)).tensor
    assert _max_abs_diff(va, vb) < 1e-12


@pytest.mark.parametrize("precision", ["double", "single"])
def test_every_tuner_candidate_vs_oracle(cuda_ok, precision):
    """Each knob set autotune.candidates() offers (tile width, low bits, merge
    width), fused, against the FP64 oracle on every gate family."""
    from quict_b200.simulation.autotune import candidates
    from test_sv_gpu import _every_placement_circuit
    from conftest import build_circuit
    esize = 16 if precision == "double" else 8
    tol = 1e-12 if precision == "double" else 1e-5
    for n in (14, 17):
        gl = _every_placement_circuit(n, seed=100 + n)
        ref = osv.run(oracle_gates(build_circuit(gl, n)), n)
        for kn in candidates(esize, n):
            s = _sim(precision, tile_bits=kn.tile_bits, low_bits=kn.low_bits, merge_bits=kn.merge_bits)
            v = s.run(build_circuit(gl, n, precision)).get()
            err = float(np.max(np.abs(v - ref)))
            assert err < tol, (n, kn, err)


def test_noisy_dm_12q_150_gates_vs_oracle(cuda_ok):
    """The benchmark's noisy density matrix in full: 12 qubits, 150 gates,
    each followed by damping composed with depolarizing noise."""
    from quict_b200.simulation import DensityMatrixSimulator
    from quict_b200.workloads import noisy_dm_problem
    c, nm = noisy_dm_problem(12, 150, 2)
    k1, k2 = odm.composed_noise_1q(5e-3, 1e-3), odm.composed_noise_2q(5e-3, 1e-2)
    ref = odm.run(oracle_gates(c), 12, noise=lambda a: k1 if len(a) == 1 else k2, superop=True)
    rho = DensityMatrixSimulator("GPU", accumulated_mode=True).run(c, noise_model=nm).get()
    assert float(np.max(np.abs(rho - ref))) < 1e-12
    c, nm = noisy_dm_problem(12, 150, 2)
    rho = DensityMatrixSimulator("GPU", "single", accumulated_mode=True).run(c, noise_model=nm).get()
    assert float(np.max(np.abs(rho - ref))) < 1e-5


def _param_shift_parallel(circ, params, terms):
    """FP64 parameter-shift gradient of `circ` at `params` for the Pauli sum
    `terms`, split over a spawn process pool (oracle.observe.shift_energies)."""
    import concurrent.futures as cf
    import multiprocessing as mp
    from test_grad import _matrices_fn, _occurrences
    fn = _matrices_fn(circ)
    base = fn(params, {})
    occ = sorted(_occurrences(circ), key=lambda t: t[1])
    shifted = [(i, fn(params, {i: np.pi / 2})[i][0], fn(params, {i: -np.pi / 2})[i][0]) for _, i, _ in occ]
    workers = max(1, min(32, os.cpu_count() or 1))
    chunks = [shifted[j::workers] for j in range(workers)]
    # one BLAS thread per worker: the workers already fill the cores
    saved = {k: os.environ.get(k) for k in ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS", "MKL_NUM_THREADS")}
    os.environ.update({k: "1" for k in saved})
    try:
        with cf.ProcessPoolExecutor(workers, mp_context=mp.get_context("spawn")) as ex:
            parts = list(ex.map(oobs.shift_energies, [base] * workers, [circ.n] * workers, [terms] * workers,
                                chunks))
    finally:
        for k, v in saved.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v
    pm = {}
    for ch, res in zip(chunks, parts):
        for (i, _, _), e in zip(ch, res):
            pm[i] = e
    g = np.zeros(len(params))
    for k, i, scale in occ:
        g[k] += scale * 0.5 * (pm[i][0] - pm[i][1])
    return g, oobs.energy(base, circ.n, terms)


def test_hea_16q_gradients_vs_fp64_parameter_shift(cuda_ok):
    """16 qubits, 8 layers of (Ry, Rz) + CZ ring, 256 parameters, H = sum ZZ +
    0.5 sum X: two parameter sets of the benchmark batch, adjoint gradients in
    both precisions against the FP64 oracle's parameter shift."""
    from quict_b200.differentiation import BatchedAdjoint
    from quict_b200.workloads import hea_problem
    circ, obs, params = hea_problem(16, 8, 1024)
    rows = [0, 517]
    want = [_param_shift_parallel(circ, params[r], obs.terms) for r in rows]
    for precision, tol in (("double", 1e-10), ("single", 1e-4)):
        eng = BatchedAdjoint(circ, obs, precision)
        e, g = eng.gradient(params[rows])
        for j, (gw, ew) in enumerate(want):
            assert abs(float(e[j]) - ew) < tol
            np.testing.assert_allclose(g[j].cpu().numpy(), gw, rtol=0, atol=tol)


def test_uneven_qaoa_batch_up_to_24_qubits(cuda_ok):
    """The batched complex64 QAOA graph with instances of 10..24 qubits
    (two of 24) against per-instance complex128 adjoint runs."""
    import torch
    from quict_b200.differentiation import BatchedAdjoint, UnevenQAOABatch, maxcut_observable, qaoa_circuit, \
        qaoa_instances
    inst = []
    for n in (10, 12, 14, 16, 18, 20, 22, 24, 24):
        inst += qaoa_instances(1, sizes=(n,), depths=(1, 6), seed=900 + n + len(inst))
    batch = UnevenQAOABatch(inst, "single")
    batch.capture()
    batch.replay()
    torch.cuda.synchronize()
    res = batch.results()
    for (n, edges, p, prm), (e, g) in zip(inst, res):
        eng = BatchedAdjoint(qaoa_circuit(n, edges, p), maxcut_observable(n, edges), "double")
        e2, g2 = eng.gradient(prm[None, :])
        scale = max(1.0, len(edges))
        assert abs(e - float(e2[0])) < 1e-5 * scale, (n, p)
        np.testing.assert_allclose(g, g2[0].cpu().numpy(), rtol=0, atol=1e-4 * scale, err_msg=f"n={n} p={p}")

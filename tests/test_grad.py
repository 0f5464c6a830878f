"""Batched energies and adjoint gradients.

Pins: tests/golden/grad.npz holds energies and parameter-shift gradients
computed from the REFERENCE StateVectorSimulator's amplitudes.  Tolerances:
complex128 energies / gradients within 1e-10, complex64 within 1e-4 of the
FP64 oracle."""
import numpy as np
import pytest

from conftest import golden
from oracle import observe as oobs
from oracle import sv as osv


def _hea(n, layers):
    from quict_b200.differentiation import hardware_efficient_ansatz, ising_observable
    return hardware_efficient_ansatz(n, layers), ising_observable(n)


def _matrices_fn(circ):
    from quict_b200.differentiation import rotation

    def fn(params, shifts):
        out = []
        for i, e in enumerate(circ.entries):
            if e.kind == "fixed":
                out.append((e.matrix, list(e.qubits)))
            else:
                out.append((rotation(e.kind, e.scale * params[e.index] + shifts.get(i, 0.0)), list(e.qubits)))
        return out
    return fn


def _occurrences(circ):
    return [(e.index, i, e.scale) for i, e in enumerate(circ.entries) if e.kind != "fixed"]


def test_oracle_gradients_match_reference_fixture():
    d = golden("grad.npz")
    circ, obs = _hea(4, 2)
    fn = _matrices_fn(circ)
    h = obs.matrix()
    th = d["hea_params"]
    assert abs(oobs.energy(fn(th, {}), 4, h) - float(d["hea_energy"])) < 1e-12
    np.testing.assert_allclose(oobs.param_shift(fn, th, 4, h, _occurrences(circ)), d["hea_grad"], atol=1e-12)
    np.testing.assert_allclose(oobs.finite_diff(fn, th, 4, h), d["hea_grad"], atol=1e-8)
    from quict_b200.differentiation import qaoa_circuit, maxcut_observable
    edges = [tuple(e) for e in d["qaoa_edges"]]
    qc = qaoa_circuit(6, edges, 2)
    fq = _matrices_fn(qc)
    hq = maxcut_observable(6, edges).matrix()
    gb = d["qaoa_params"]
    assert abs(oobs.energy(fq(gb, {}), 6, hq) - float(d["qaoa_energy"])) < 1e-12
    np.testing.assert_allclose(oobs.param_shift(fq, gb, 6, hq, _occurrences(qc)), d["qaoa_grad"], atol=1e-11)


def test_pauli_masks_and_dense_matrix_agree():
    from quict_b200.differentiation import PauliSum
    hs = PauliSum(3).add(0.7, {0: "X", 2: "Y"}).add(-1.1, {1: "Z"}).add(0.25, {})
    x, z, c = hs.masks()
    v = np.random.default_rng(0).normal(size=8) + 1j * np.random.default_rng(1).normal(size=8)
    out = np.zeros(8, dtype=np.complex128)
    for t in range(len(x)):
        coeff = complex(c[2 * t], c[2 * t + 1]) * (1j ** bin(int(x[t]) & int(z[t])).count("1"))
        for j in range(8):
            src = j ^ int(x[t])
            out[j] += coeff * (-1) ** bin(int(z[t]) & src).count("1") * v[src]
    np.testing.assert_allclose(out, hs.matrix() @ v, atol=1e-14)


def test_pair_tile_width_range_is_checked_before_the_device():
    """pair_tile_bits outside [smallest register tile, 64 KiB tile] is refused
    on the host, before any device is touched."""
    from quict_b200.differentiation import BatchedAdjoint
    circ, obs = _hea(4, 1)
    for precision, bad in (("double", (8, 13)), ("single", (9, 14))):
        for k in bad:
            with pytest.raises(ValueError, match="pair_tile_bits"):
                BatchedAdjoint(circ, obs, precision, pair_tile_bits=k)


def test_random_regular_graph_is_regular():
    from quict_b200.differentiation import random_regular_graph
    for n in (10, 16, 24):
        es = random_regular_graph(n, 3, np.random.default_rng(n))
        deg = np.bincount(np.array(es).ravel(), minlength=n)
        assert len(es) == 3 * n // 2 and np.all(deg == 3)


# ------------------------------------------------------------------ GPU
pytestmark_gpu = pytest.mark.gpu


@pytest.mark.gpu
@pytest.mark.parametrize("precision,tol", [("double", 1e-10), ("single", 1e-4)])
def test_adjoint_matches_reference_fixture(cuda_ok, precision, tol):
    from quict_b200.differentiation import BatchedAdjoint
    d = golden("grad.npz")
    circ, obs = _hea(4, 2)
    eng = BatchedAdjoint(circ, obs, precision)
    e, g = eng.gradient(d["hea_params"][None, :])
    assert abs(float(e[0]) - float(d["hea_energy"])) < tol
    np.testing.assert_allclose(g[0].cpu().numpy(), d["hea_grad"], atol=tol)


@pytest.mark.gpu
@pytest.mark.parametrize("precision,tol", [("double", 1e-10), ("single", 1e-4)])
def test_adjoint_qaoa_matches_reference_fixture(cuda_ok, precision, tol):
    from quict_b200.differentiation import BatchedAdjoint, qaoa_circuit, maxcut_observable
    d = golden("grad.npz")
    edges = [tuple(int(a) for a in e) for e in d["qaoa_edges"]]
    eng = BatchedAdjoint(qaoa_circuit(6, edges, 2), maxcut_observable(6, edges), precision)
    e, g = eng.gradient(d["qaoa_params"][None, :])
    assert abs(float(e[0]) - float(d["qaoa_energy"])) < tol * 10
    np.testing.assert_allclose(g[0].cpu().numpy(), d["qaoa_grad"], atol=tol * 10)


@pytest.mark.gpu
@pytest.mark.parametrize("n,layers,batch", [(6, 2, 5), (13, 2, 4), (16, 1, 3)])
def test_batched_adjoint_vs_oracle(cuda_ok, n, layers, batch):
    from quict_b200.differentiation import BatchedAdjoint
    circ, obs = _hea(n, layers)
    rng = np.random.default_rng(n)
    params = rng.uniform(0, 2 * np.pi, (batch, circ.num_params))
    fn = _matrices_fn(circ)
    h = obs.matrix() if n <= 10 else None
    for precision, tol in (("double", 1e-10), ("single", 1e-4)):
        eng = BatchedAdjoint(circ, obs, precision)
        e, g = eng.gradient(params)
        states = eng.states(params).cpu().numpy()
        for b in range(batch):
            psi = osv.run(fn(params[b], {}), n)
            np.testing.assert_allclose(states[b], psi, atol=10 * tol)
            if h is not None:
                assert abs(float(e[b]) - oobs.energy(fn(params[b], {}), n, h)) < tol
        if h is not None:
            for b in range(min(batch, 2)):
                want = oobs.param_shift(fn, params[b], n, h, _occurrences(circ))
                np.testing.assert_allclose(g[b].cpu().numpy(), want, atol=tol)
        # GPU parameter shift agrees with the adjoint sweep (same GPU kernels)
        ps = eng.parameter_shift(params, indices=[0, 1, circ.num_params - 1])
        np.testing.assert_allclose(ps.cpu().numpy(), g[:, [0, 1, circ.num_params - 1]].cpu().numpy(), atol=tol)


@pytest.mark.gpu
def test_autograd_function(cuda_ok):
    import torch
    from quict_b200.differentiation import BatchedAdjoint, expectation
    circ, obs = _hea(5, 2)
    eng = BatchedAdjoint(circ, obs, "double")
    p = torch.tensor(np.random.default_rng(3).uniform(0, 6, (3, circ.num_params)), requires_grad=True)
    e = expectation(p, eng)
    e.sum().backward()
    _, g = eng.gradient(p.detach())
    np.testing.assert_allclose(p.grad.numpy(), g.cpu().numpy(), atol=1e-12)


@pytest.mark.gpu
def test_uneven_qaoa_graph_vs_per_instance_c128(cuda_ok):
    """Uneven QAOA batch (small sizes) in one CUDA graph, complex64, against
    per-instance complex128 adjoint runs and, for the smallest, the FP64 oracle."""
    from quict_b200.differentiation import (BatchedAdjoint, UnevenQAOABatch, qaoa_instances, qaoa_circuit,
                                            maxcut_observable)
    inst = qaoa_instances(12, sizes=(6, 8, 10, 12, 14), depths=(1, 3), seed=9)
    batch = UnevenQAOABatch(inst, "single", streams=4)
    batch.capture()
    batch.replay()
    import torch
    torch.cuda.synchronize()
    res = batch.results()
    for (n, edges, p, prm), (e, g) in zip(inst, res):
        eng = BatchedAdjoint(qaoa_circuit(n, edges, p), maxcut_observable(n, edges), "double")
        e2, g2 = eng.gradient(prm[None, :])
        scale = max(1.0, len(edges))
        assert abs(e - float(e2[0])) < 1e-4 * scale
        np.testing.assert_allclose(g, g2[0].cpu().numpy(), atol=1e-4 * scale)
        if n <= 8:
            circ = qaoa_circuit(n, edges, p)
            fn = _matrices_fn(circ)
            h = maxcut_observable(n, edges).matrix()
            np.testing.assert_allclose(g2[0].cpu().numpy(), oobs.param_shift(fn, prm, n, h, _occurrences(circ)),
                                       atol=1e-9)
    # a second replay gives the same results (the graph is reusable)
    batch.replay()
    torch.cuda.synchronize()
    for (e, g), (e3, g3) in zip(res, batch.results()):
        assert e == e3 and np.array_equal(g, g3)


@pytest.mark.gpu
@pytest.mark.parametrize("precision,tol", [("double", 1e-10), ("single", 1e-4)])
def test_pair_vector_backward_matches_shared_memory_path(cuda_ok, precision, tol):
    """The register-tile backward on the psi/lam pair vector (qs_adjoint_pair)
    against the shared-memory backward (qs_adjoint_fused) and the FP64 oracle's
    parameter shift, for a batch (pair bit above the instance bits) and for one
    QAOA instance (pair bit just above the qubits)."""
    from quict_b200.differentiation import BatchedAdjoint, maxcut_observable, qaoa_circuit, random_regular_graph
    n = 10
    circ, obs = _hea(n, 2)
    params = np.random.default_rng(4).uniform(0, 2 * np.pi, (4, circ.num_params))
    fast = BatchedAdjoint(circ, obs, precision)
    slow = BatchedAdjoint(circ, obs, precision, pair=False)
    gp = fast.plan_gradient(params)
    assert gp.pair and not slow.plan_gradient(params).pair
    e1, g1 = fast.gradient(params)
    e2, g2 = slow.gradient(params)
    np.testing.assert_allclose(e1.cpu().numpy(), e2.cpu().numpy(), atol=tol)
    np.testing.assert_allclose(g1.cpu().numpy(), g2.cpu().numpy(), atol=tol)
    fn, h = _matrices_fn(circ), obs.matrix()
    want = oobs.param_shift(fn, params[1], n, h, _occurrences(circ))
    np.testing.assert_allclose(g1[1].cpu().numpy(), want, atol=tol)
    edges = random_regular_graph(n, 3, np.random.default_rng(2))
    qc, qo = qaoa_circuit(n, edges, 2), maxcut_observable(n, edges)
    prm = np.random.default_rng(5).uniform(0, 3, (1, qc.num_params))
    a, b = BatchedAdjoint(qc, qo, precision), BatchedAdjoint(qc, qo, precision, pair=False)
    assert a.plan_gradient(prm).pair
    ea, ga = a.gradient(prm)
    eb, gb = b.gradient(prm)
    assert abs(float(ea[0]) - float(eb[0])) < tol * len(edges)
    np.testing.assert_allclose(ga.cpu().numpy(), gb.cpu().numpy(), atol=tol * len(edges))


@pytest.mark.gpu
@pytest.mark.parametrize("precision,tol,widths", [("double", 1e-10, (9, 10, 11, 12)),
                                                  ("single", 1e-4, (10, 11, 12, 13))])
def test_pair_tile_widths_agree(cuda_ok, precision, tol, widths):
    """Every pair tile width the register backward accepts gives the gradient
    of the shared-memory backward; widths outside that range are refused."""
    from quict_b200.differentiation import BatchedAdjoint
    circ, obs = _hea(13, 2)  # batch of 2: the tile takes up to 13 non-pair bits
    params = np.random.default_rng(6).uniform(0, 2 * np.pi, (2, circ.num_params))
    e0, g0 = BatchedAdjoint(circ, obs, precision, pair=False).gradient(params)
    for k in widths:
        eng = BatchedAdjoint(circ, obs, precision, pair_tile_bits=k)
        assert eng.plan_gradient(params).pair
        e, g = eng.gradient(params)
        np.testing.assert_allclose(e.cpu().numpy(), e0.cpu().numpy(), atol=tol)
        # 13 qubits, 13 Ising terms: the two backward sweeps sum in different orders
        np.testing.assert_allclose(g.cpu().numpy(), g0.cpu().numpy(), atol=4 * tol)
    for k in (widths[0] - 1, widths[-1] + 1):
        with pytest.raises(ValueError):
            BatchedAdjoint(circ, obs, precision, pair_tile_bits=k)


def test_qaoa_cost_layer_units_match_the_gates():
    """Commuting Rzz gates that share a parameter are grouped into diagonal units
    of at most 4 qubits, and Rx gates that share one into pairs; the units'
    product equals the gates' product."""
    from quict_b200.differentiation import maxcut_observable, qaoa_circuit, random_regular_graph
    from quict_b200.differentiation.adjoint import gate_units
    n, p = 8, 2
    edges = random_regular_graph(n, 3, np.random.default_rng(1))
    circ = qaoa_circuit(n, edges, p)
    params = np.random.default_rng(2).uniform(0, 3, circ.num_params)
    units = gate_units(circ)
    assert len(units) < len(circ.entries)
    assert all(len(u.qubits) <= 4 for u in units)
    mats = []
    for u in units:
        if u.fixed is not None:
            mats.append((u.fixed, list(u.qubits)))
        else:
            kind, tab = u.tables(np.array([u.scale * params[u.index]]), False)
            m = np.diag(tab[0]) if kind == "diag" else tab[0].reshape(1 << len(u.qubits), -1)
            mats.append((m, list(u.qubits)))
    np.testing.assert_allclose(osv.run(mats, n), osv.run(circ.matrices(params), n), atol=1e-12)
    plain = gate_units(circ, cluster=False)
    assert len(plain) == len(circ.entries)

"""Autotuner: cache format and precedence, the successive-halving search, and
a tuned run on the GPU checked against the oracle."""
import json
import math

import numpy as np
import pytest

from quict_b200.simulation.autotune import Autotuner, Knobs, TuneResult, candidates, default_knobs, tune_key


def test_knobs_json_round_trip():
    for kn in (Knobs(12, 5, 2), Knobs(13, 6, 0, 48.0)):
        assert Knobs.from_json(json.loads(json.dumps(kn.to_json()))) == kn
    assert Knobs(12, 5, 2).to_json()["max_pass_cost"] is None
    assert math.isinf(Knobs.from_json({"tile_bits": 12, "low_bits": 5, "merge_bits": 2}).max_pass_cost)


def test_candidates_respect_register_tile_widths():
    for esize, ks in ((16, {10, 11, 12}), (8, {11, 12, 13})):
        c = candidates(esize, 30)
        assert {kn.tile_bits for kn in c} == ks
        assert {kn.merge_bits for kn in c} == {0, 2, 3}
        assert default_knobs(esize).tile_bits == max(ks)
    assert all(kn.tile_bits <= 11 for kn in candidates(16, 11))
    assert len(candidates(16, 30)) == 18


def test_cache_precedence_user_over_packaged(tmp_path):
    user, packaged = tmp_path / "user.json", tmp_path / "pkg.json"
    key = tune_key("NVIDIA B200", 16, 30, "sv")
    assert key == "NVIDIA B200|c128|n30|sv"
    t = Autotuner(cache_path=str(user), packaged_path=str(packaged))
    assert t.lookup(key) is None
    t.store(key, TuneResult(Knobs(11, 6, 3), 1.0), path=str(packaged))
    assert t.lookup(key) == Knobs(11, 6, 3)
    t.store(key, TuneResult(Knobs(12, 5, 2), 0.5))
    assert t.lookup(key) == Knobs(12, 5, 2)
    d = json.load(open(user))
    assert d[key]["ms"] == 0.5 and "when" in d[key]
    (tmp_path / "bad.json").write_text("not json")
    assert Autotuner(cache_path=str(tmp_path / "bad.json"), packaged_path=str(packaged)).lookup(key) == Knobs(11, 6, 3)


def test_successive_halving_picks_fastest_full_run():
    cands = [Knobs(12, 5, m) for m in (0, 2, 3)] + [Knobs(11, 5, m) for m in (0, 2, 3)]
    prefix = {c: float(i) for i, c in enumerate(cands)}          # first three look best on the prefix
    full = {cands[0]: 9.0, cands[1]: 3.0, cands[2]: 5.0, cands[3]: 0.1}
    res = Autotuner.search(cands, lambda k: prefix[k], lambda k: full[k], keep=3)
    assert res.knobs == cands[1] and res.ms == 3.0               # cands[3] never reaches the full round
    assert sum(1 for k in res.trials if k.startswith("full")) == 3


@pytest.mark.gpu
def test_autotuned_run_matches_oracle(cuda_ok, tmp_path, monkeypatch):
    from conftest import oracle_gates
    from oracle import sv as osv
    from quict_b200.simulation import StateVectorSimulator
    from quict_b200.workloads import spread_circuit
    monkeypatch.setenv("QUICT_B200_TUNE_CACHE", str(tmp_path / "tune.json"))
    n = 14
    c = spread_circuit(n, 150, seed=3)
    sim = StateVectorSimulator("GPU", "double", autotune=True)
    v = sim.run(c).get()
    np.testing.assert_allclose(v, osv.run(oracle_gates(c), n), atol=1e-12)
    d = json.load(open(tmp_path / "tune.json"))
    (key,) = d.keys()
    assert key.endswith("|c128|n14|sv") and len(d[key]["trials"]) >= len(candidates(16, n))
    # a second simulator reads the cached knobs and does not tune again
    sim2 = StateVectorSimulator("GPU", "double", autotune=True)
    v2 = sim2.run(c).get()
    np.testing.assert_allclose(v2, v, atol=1e-12)
    assert sim2.engine.knobs(sim2._vector, n) == Knobs.from_json(d[key]["knobs"])


def test_adjoint_candidates_and_cache_lookup(tmp_path):
    """Adjoint tile candidates stay inside the register-tile range and the
    pair tile fits the psi/lam vector; "qaoa" entries read back as (forward,
    pair) tile widths and are not mistaken for fused-pass knobs."""
    import json
    from quict_b200.simulation.autotune import Autotuner, adjoint_candidates
    for prec, lo, hi in (("single", 10, 13), ("double", 9, 12)):
        for n in (10, 12, 16, 24):
            c = adjoint_candidates(prec, n)
            assert c and all(lo <= f <= max(lo, min(hi - 1, n)) and lo <= p <= min(hi, n + 1) for f, p in c)
    path = tmp_path / "tune.json"
    path.write_text(json.dumps({"dev|c64|n16|qaoa": {"knobs": {"tile_bits": 11, "pair_tile_bits": 12}, "ms": 1.0},
                                "dev|c64|n16|sv": {"knobs": {"tile_bits": 11, "low_bits": 5, "merge_bits": 2,
                                                             "max_pass_cost": None}, "ms": 1.0}}))
    t = Autotuner(cache_path=str(path), packaged_path=str(tmp_path / "none.json"))
    assert t.lookup_adjoint("dev|c64|n16|qaoa") == (11, 12)
    assert t.lookup_adjoint("dev|c64|n16|sv") is None
    assert t.lookup_adjoint("dev|c64|n18|qaoa") is None

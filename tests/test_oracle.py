"""The C oracle against the reference's own results (CPU only).

The expected values in tests/golden were produced by the reference's
CPU_01_nonparallel code (tests/golden/make_golden.py); these tests pin the
restatement in oracle/rules_oracle.c to them before it is trusted as the
checker of the CUDA engine.
"""
import hashlib

import numpy as np
import pytest

import oracle
from conftest import GOLDEN, fuzz_names, load_fixture, terms_to_ir
from masterthesis_gpu_acceleration_b200 import synth

FIELDS = ("support", "headSize", "headSupport", "bodySize")


def _compare(counts, expected):
    got = [dict(zip(FIELDS, row)) for row in counts.tolist()]
    want = [{k: e[k] for k in FIELDS} for e in expected]
    bad = [(i, g, w) for i, (g, w) in enumerate(zip(got, want)) if g != w]
    assert not bad, f"{len(bad)} rules differ, first: {bad[:3]}"


@pytest.mark.parametrize("cfg", ["c1", "c2", "c2s", "c4s"])
def test_synthetic_graph_is_reproducible(cfg, data_dir):
    fx = load_fixture(f"synthetic_{cfg}.json")
    d = synth.generate(cfg, data_dir / cfg, seed=fx["seed"])
    assert hashlib.sha256((d / "triples.bin").read_bytes()).hexdigest() == fx["triples_sha256"]
    assert synth.read_rules(d) == fx["rules"]


@pytest.mark.parametrize("cfg", ["c1", "c2", "c2s"])
def test_oracle_matches_reference_synthetic(cfg, data_dir):
    fx = load_fixture(f"synthetic_{cfg}.json")
    d = synth.generate(cfg, data_dir / cfg, seed=fx["seed"])
    meta = synth.read_meta(d)
    g = oracle.OracleGraph(synth.read_triples(d), int(meta["predicates"]))
    counts, status = g.evaluate_ir(synth.read_rule_ir(d), len(fx["rules"]))
    assert (status == 0).all()
    _compare(counts, fx["expected"])


def test_oracle_matches_reference_c4s_plain_rules(data_dir):
    """c4s rules 10..49 (the ones that do not cross a hub; the hub rules take
    the oracle minutes and are checked against the same fixture on the GPU)."""
    fx = load_fixture("synthetic_c4s.json")
    d = synth.generate("c4s", data_dir / "c4s", seed=fx["seed"])
    g = oracle.OracleGraph(synth.read_triples(d), int(synth.read_meta(d)["predicates"]))
    ir = np.concatenate(oracle.split_ir(synth.read_rule_ir(d))[10:])
    counts, status = g.evaluate_ir(ir, len(fx["rules"]) - 10)
    assert (status == 0).all()
    _compare(counts, fx["expected"][10:])


@pytest.mark.parametrize("name", fuzz_names())
def test_oracle_matches_reference_fuzz(name):
    fx = load_fixture(name)
    g = oracle.OracleGraph(np.array(fx["triples"], dtype=np.int32), fx["n_pred"])
    ir = terms_to_ir(fx["rule_terms"])
    counts, status = g.evaluate_ir(ir, len(fx["rules"]))
    assert (status == 0).all()
    _compare(counts, fx["expected"])


def test_oracle_measures_follow_final_rule():
    m = oracle.measures(np.array([[3, 6, 6, 4], [0, 0, 0, 0], [2, 5, 5, 0]]))
    assert m[0]["headCoverage"] == 0.5 and m[0]["confidence"] == 0.75
    assert m[1]["headCoverage"] == 0.0 and m[1]["confidence"] == 0.0
    assert m[2]["confidence"] == 0.0


def test_oracle_c3_sample():
    path = GOLDEN / "c3_seed0.npz"
    if not path.exists():
        pytest.skip("c3 fixture not generated")
    z = np.load(path)
    exp = z["expected"]
    import tempfile
    from pathlib import Path
    with tempfile.TemporaryDirectory() as t:
        d = synth.generate("c3", Path(t) / "c3", seed=0)
        assert hashlib.sha256((d / "triples.bin").read_bytes()).hexdigest() == str(z["triples_sha256"])
        meta = synth.read_meta(d)
        g = oracle.OracleGraph(synth.read_triples(d), int(meta["predicates"]))
        rules = oracle.split_ir(synth.read_rule_ir(d))
        # a deterministic sample of cheap rules (small body sizes) keeps this CPU test short
        idx = [i for i in range(len(rules)) if exp[i, 3] < 20000][:400]
        ir = np.concatenate([rules[i] for i in idx])
        counts, _ = g.evaluate_ir(ir, len(idx))
        assert (counts == exp[idx]).all()


def test_c4_hub_fixture_is_well_formed():
    """The full-size c4 hub-rule fixture (reference output) holds the 10 hub
    rules and at least one body size that wrapped past 2^31 in the
    reference's int."""
    fx = load_fixture("c4_seed0_hub.json")
    assert fx["rules_index"] == list(range(10)) and len(fx["rules"]) == len(fx["expected"]) == 10
    assert any(e["bodySize_ref"] < 0 for e in fx["expected"])
    assert all(e["support"] <= e["headSupport"] <= e["headSize"] for e in fx["expected"])

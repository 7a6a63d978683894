"""Parity of the CUDA engine with the reference, through the C ABI.

Expected values come from the reference's CPU_01_nonparallel code
(tests/golden) and, where noted, from the C oracle that those fixtures pin.
Counts are integers and must match exactly; headCoverage and confidence are
the same IEEE double divisions of the same integers, so they must match
exactly as well.
"""
import hashlib

import numpy as np
import pytest

import masterthesis_gpu_acceleration_b200 as eng
import oracle
from conftest import GOLDEN, fuzz_names, load_fixture
from masterthesis_gpu_acceleration_b200 import synth

pytestmark = pytest.mark.gpu

FIELDS = ("support", "headSize", "headSupport", "bodySize", "headCoverage", "confidence")


def _check(results, expected, label=""):
    bad = []
    for i, (r, e) in enumerate(zip(results, expected)):
        got = {f: getattr(r, f) for f in FIELDS}
        want = {f: e[f] for f in FIELDS}
        if got != want:
            bad.append((i, got, want))
    assert not bad, f"{label}: {len(bad)} of {len(expected)} rules differ, first: {bad[:2]}"


@pytest.fixture(scope="module")
def edge_lib(tmp_path_factory):
    fx = load_fixture("edge_cases.json")
    p = tmp_path_factory.mktemp("edge") / "graph.ttl"
    p.write_text(fx["ttl"])
    with eng.GpuRulesLib(p) as lib:
        yield lib, fx


def test_edge_cases_per_rule(edge_lib):
    lib, fx = edge_lib
    for case in fx["cases"]:
        r = lib.evaluate_rule(case["rule"])
        _check([r], [case["expected"]], case["what"])


def test_edge_cases_batch(edge_lib):
    lib, fx = edge_lib
    res, st, _ = lib.evaluate_rules_batch([c["rule"] for c in fx["cases"]])
    assert all(s == 0 for s in st)
    _check(res, [c["expected"] for c in fx["cases"]], "edge batch")


def test_malformed_rules_are_errors(edge_lib):
    lib, _ = edge_lib
    for bad in ["", "(?a <http://x/p> ?b)", "(?a <http://x/p>) => (?a <http://x/p> ?b)",
                "?a <http://x/p> ?b => (?a <http://x/p> ?b)"]:
        with pytest.raises(RuntimeError):
            lib.evaluate_rule(bad)
    res, st, _ = lib.evaluate_rules_batch(["(?x <http://x/p> ?y) => (?y <http://x/p> ?x)", "garbage"])
    assert st == [0, -1]
    assert res[1].support == 0 and res[1].bodySize == 0


def test_unsupported_rule_reports_head_only(edge_lib):
    lib, _ = edge_lib
    body = " ^ ".join(f"(?v{i} <http://x/p> ?v{i+1})" for i in range(9))
    r = lib.evaluate_rule(body + " => (?v0 <http://x/p> ?v9)")
    assert r.support == 0 and r.bodySize == 0 and r.headSize == 6 and r.headSupport == 6


@pytest.mark.parametrize("name", fuzz_names())
def test_fuzz(name, tmp_path):
    fx = load_fixture(name)
    p = tmp_path / "graph.ttl"
    p.write_text(fx["ttl"])
    with eng.GpuRulesLib(p) as lib:
        _check([lib.evaluate_rule(t) for t in fx["rules"]], fx["expected"], "per-rule text")
        res, st, _ = lib.evaluate_rules_batch(fx["rules"])
        assert all(s == 0 for s in st)
        _check(res, fx["expected"], "batch text")
        _check([lib.evaluate_rule_json(j) for j in fx["rules_json"]], fx["expected_json"], "per-rule json")
        res, st, _ = lib.evaluate_rules_batch(fx["rules_json"], is_json=True)
        _check(res, fx["expected_json"], "batch json")


@pytest.mark.parametrize("cfg", ["c1", "c2", "c2s", "c4s"])
def test_synthetic(cfg, data_dir):
    fx = load_fixture(f"synthetic_{cfg}.json")
    d = synth.generate(cfg, data_dir / cfg, seed=fx["seed"])
    assert hashlib.sha256((d / "triples.bin").read_bytes()).hexdigest() == fx["triples_sha256"]
    with eng.GpuRulesLib(d / "graph.ttl") as lib:
        _check([lib.evaluate_rule(t) for t in fx["rules"]], fx["expected"], f"{cfg} per-rule")
        res, st, _ = lib.evaluate_rules_batch(fx["rules"])
        _check(res, fx["expected"], f"{cfg} batch")


def test_c3_full_batch(data_dir):
    path = GOLDEN / "c3_seed0.npz"
    if not path.exists():
        pytest.skip("c3 fixture not generated")
    z = np.load(path)
    exp = z["expected"]
    d = synth.generate("c3", data_dir / "c3", seed=0)
    assert hashlib.sha256((d / "triples.bin").read_bytes()).hexdigest() == str(z["triples_sha256"])
    rules = synth.read_rules(d)
    with eng.GpuRulesLib(d / "graph.ttl") as lib:
        res, st, ms = lib.evaluate_rules_batch(rules)
        got = np.array([[r.support, r.headSize, r.headSupport, r.bodySize] for r in res], dtype=np.int64)
        bad = np.nonzero((got != exp).any(axis=1))[0]
        assert len(bad) == 0, f"{len(bad)} rules differ, first {bad[:5]}: {got[bad[:3]]} vs {exp[bad[:3]]}"
        # the plain one-launch-per-phase form agrees on a sample
        for i in range(0, len(rules), 97):
            r = lib.evaluate_rule(rules[i])
            assert [r.support, r.headSize, r.headSupport, r.bodySize] == exp[i].tolist(), i


def test_batch_equals_alone(tmp_path):
    """Each result is the same alone and in a mixed batch."""
    fx = load_fixture("fuzz_2.json")
    p = tmp_path / "graph.ttl"
    p.write_text(fx["ttl"])
    with eng.GpuRulesLib(p) as lib:
        rules = fx["rules"]
        mixed = rules[::-1] + rules[:20]
        res, _, _ = lib.evaluate_rules_batch(mixed)
        alone = {t: lib.evaluate_rule(t).as_dict() for t in rules}
        for t, r in zip(mixed, res):
            a, b = alone[t], r.as_dict()
            for f in FIELDS:
                assert a[f] == b[f], (t, f)


def test_oracle_agrees_on_c2_skew_batch(data_dir):
    d = synth.generate("c2s", data_dir / "c2s_big", seed=7, n_rules=40)
    meta = synth.read_meta(d)
    g = oracle.OracleGraph(synth.read_triples(d), int(meta["predicates"]))
    rules = synth.read_rules(d)
    counts, _ = g.evaluate_ir(synth.read_rule_ir(d), len(rules))
    with eng.GpuRulesLib(d / "graph.ttl") as lib:
        res, _, _ = lib.evaluate_rules_batch(rules)
    got = np.array([[r.support, r.headSize, r.headSupport, r.bodySize] for r in res], dtype=np.int64)
    assert (got == counts).all()


def test_prepared_batch_replays_exactly(tmp_path):
    fx = load_fixture("fuzz_4.json")
    p = tmp_path / "graph.ttl"
    p.write_text(fx["ttl"])
    with eng.GpuRulesLib(p) as lib:
        with lib.prepare_batch(fx["rules"]) as b:
            info = b.info()
            assert info["h2d_bytes"] > 0 and info["d2h_bytes"] > 0
            for flush in (0, 1 << 20, 0):
                res, st, ms = b.run(flush)
                assert ms >= 0
                _check(res, fx["expected"], f"prepared run flush={flush}")
            assert b.count_bytes() > 0


@pytest.mark.parametrize("name", ["fuzz_0.json", "fuzz_2.json", "fuzz_5.json"])
@pytest.mark.parametrize("block", [128, 256, 512])
def test_fuzz_forced_splitting(name, block, tmp_path):
    """Every root is measured and every root with more than a few candidates
    is split into first-segment slices deduplicated in global rows."""
    fx = load_fixture(name)
    p = tmp_path / "graph.ttl"
    p.write_text(fx["ttl"])
    with eng.GpuRulesLib(p) as lib:
        lib.set_option("block", block)
        lib.set_option("walk_threshold", 0)
        lib.set_option("task_target", 3)
        res, st, _ = lib.evaluate_rules_batch(fx["rules"])
        _check(res, fx["expected"], f"batch split block={block}")
        # per-rule launches on the batch block size, then on 512-thread
        # blocks with plans laid out for the batch block size
        for rule_block in (0, 512):
            lib.set_option("rule_block", rule_block)
            _check([lib.evaluate_rule(t) for t in fx["rules"][:60]], fx["expected"][:60],
                   f"per-rule split block={block} rule_block={rule_block}")


@pytest.mark.parametrize("hub_min,memo_gain", [("1", "0"), ("1", "-1"), ("0", "8")])
def test_hub_rows_everywhere_or_nowhere(hub_min, memo_gain, tmp_path, monkeypatch):
    """Body sizes through hub-row bitmaps and two-step suffix memos (every row
    a hub and every hub memoised; hubs without memos; neither), on the fuzz
    graphs, the edge cases and c2s, against the reference."""
    monkeypatch.setenv("GPU_RULES_HUB_MIN_DEGREE", hub_min)
    monkeypatch.setenv("GPU_RULES_MEMO_GAIN", memo_gain)
    for name in fuzz_names():
        fx = load_fixture(name)
        p = tmp_path / f"{name}.ttl"
        p.write_text(fx["ttl"])
        with eng.GpuRulesLib(p) as lib:
            res, st, _ = lib.evaluate_rules_batch(fx["rules"])
            _check(res, fx["expected"], f"{name} hub_min={hub_min} batch")
            _check([lib.evaluate_rule(t) for t in fx["rules"][:40]], fx["expected"][:40], f"{name} per-rule")
    fx = load_fixture("edge_cases.json")
    p = tmp_path / "edge.ttl"
    p.write_text(fx["ttl"])
    with eng.GpuRulesLib(p) as lib:
        res, _, _ = lib.evaluate_rules_batch([c["rule"] for c in fx["cases"]])
        _check(res, [c["expected"] for c in fx["cases"]], f"edge hub_min={hub_min}")
    fx = load_fixture("synthetic_c2s.json")
    d = synth.generate("c2s", tmp_path / "c2s", seed=fx["seed"])
    with eng.GpuRulesLib(d / "graph.ttl") as lib:
        res, _, _ = lib.evaluate_rules_batch(fx["rules"])
        _check(res, fx["expected"], f"c2s hub_min={hub_min}")


@pytest.mark.parametrize("name", ["fuzz_1.json", "fuzz_3.json"])
def test_graph_file_loads_identically(name, tmp_path):
    """A graph written by save_index and loaded back answers every rule as
    the Turtle load does, per rule and batched."""
    fx = load_fixture(name)
    p = tmp_path / "graph.ttl"
    p.write_text(fx["ttl"])
    f = tmp_path / "graph.bin"
    with eng.GpuRulesLib(p) as lib:
        lib.save_index(f)
    with eng.GpuRulesLib(index_path=f) as lib:
        res, st, _ = lib.evaluate_rules_batch(fx["rules"])
        _check(res, fx["expected"], f"{name} from graph file, batch")
        _check([lib.evaluate_rule(t) for t in fx["rules"][:30]], fx["expected"][:30], f"{name} from graph file, per rule")
    (tmp_path / "cut.bin").write_bytes(f.read_bytes()[:1000])
    with pytest.raises(RuntimeError):
        eng.GpuRulesLib(index_path=tmp_path / "cut.bin")


def test_batch_refuses_a_smaller_block_than_staged(tmp_path):
    """Plans are laid out for the shared pool of the block size they were
    staged at.  After the block size is lowered, a prepared batch replays
    its captured launch unchanged (same counts), while a launch issued anew
    (the instrumented run of profile()) is refused with an error; at the
    staged size it works again."""
    fx = load_fixture("fuzz_0.json")
    p = tmp_path / "graph.ttl"
    p.write_text(fx["ttl"])
    with eng.GpuRulesLib(p) as lib:
        lib.set_option("block", 256)
        b = lib.prepare_batch(fx["rules"])
        b.run()
        want = b.counts().copy()
        lib.set_option("block", 128)
        b.run()
        assert (b.counts() == want).all()
        with pytest.raises(RuntimeError):
            b.profile()
        lib.set_option("block", 256)
        b.profile()
        b.run()
        assert (b.counts() == want).all()
        b.close()

"""The rule miner over the engine: one batched call per level and one call
per candidate (the reference's pattern) mine the same rules with the same
measures, and those equal the C oracle's."""
import pytest

import oracle
from miner_eval import oracle_evaluator, small_graph
import masterthesis_gpu_acceleration_b200 as eng
from masterthesis_gpu_acceleration_b200 import miner

pytestmark = pytest.mark.gpu


def _summary(res):
    return [(s.rule.text(), s.support, s.head_size, s.body_size, s.confidence) for s in res.rules]


def test_batched_mining_matches_per_rule_and_oracle(tmp_path):
    t, ttl = small_graph()
    p = tmp_path / "graph.ttl"
    p.write_text(ttl)
    kw = dict(max_body=2, min_support=5, min_head_coverage=0.01, min_confidence=0.0, max_head_predicates=2)
    with eng.GpuRulesLib(p) as lib:
        preds = lib.predicates()
        assert sorted(n for _, n in preds) == sorted(int((t[:, 1] == k).sum()) for k in range(4))
        batched = miner.mine(miner.gpu_evaluator(lib), preds, **kw)
        single = miner.mine(miner.gpu_evaluator(lib, per_rule=True), preds, **kw)
    # the oracle names predicates by generator id; the library by IRI order of appearance
    want = miner.mine(oracle_evaluator(oracle.OracleGraph(t, 4)), preds, **kw)
    assert batched.levels == single.levels == want.levels
    assert _summary(batched) == _summary(single) == _summary(want)
    assert batched.rules

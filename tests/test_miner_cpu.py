"""The rule miner's refinement, pruning and output rules, scored by the C
oracle on a synthetic graph (CPU only)."""
import oracle
from miner_eval import oracle_evaluator, small_graph
from masterthesis_gpu_acceleration_b200 import miner

P = "http://p/"


def test_refinements_dangling_and_closing():
    r = miner.Rule(("?a", P + "0", "?b"), (("?a", P + "1", "?v0"),))
    refs = miner.refinements(r, [P + "2"], max_vars=4)
    # three variables: 2 dangling atoms each, 2 closing atoms per ordered pair
    assert len(refs) == 3 * 2 + 3 * 2
    assert all(len(x.body) == 2 for x in refs)
    assert sum(x.closed() for x in refs) == 2   # (?b p2 ?v0) and (?v0 p2 ?b) close the chain
    assert not miner.refinements(r, [P + "2"], max_vars=3)[0].closed()


def test_canonical_key_merges_renamings():
    a = miner.Rule(("?a", P + "0", "?b"), (("?a", P + "1", "?v0"), ("?v0", P + "2", "?b")))
    b = miner.Rule(("?a", P + "0", "?b"), (("?v7", P + "2", "?b"), ("?a", P + "1", "?v7")))
    assert a.key() == b.key()
    c = miner.Rule(("?a", P + "0", "?b"), (("?a", P + "2", "?v0"), ("?v0", P + "1", "?b")))
    assert a.key() != c.key()


def test_mining_with_the_oracle():
    t, _ = small_graph()
    g = oracle.OracleGraph(t, 4)
    preds = [(P + str(k), int((t[:, 1] == k).sum())) for k in range(4)]
    res = miner.mine(oracle_evaluator(g), preds, max_body=2, min_support=5, min_head_coverage=0.01,
                     min_confidence=0.0, max_head_predicates=2)
    assert res.levels and res.evaluated == sum(res.levels)
    assert res.rules, "some closed rules pass the thresholds"
    for s in res.rules:
        assert s.rule.closed() and s.support >= 5 and s.head_coverage >= 0.01
    # the output rules re-scored alone give the same measures
    again = oracle_evaluator(g)([s.rule for s in res.rules])
    assert [m["support"] for m in again] == [s.support for s in res.rules]
    assert [m["bodySize"] for m in again] == [s.body_size for s in res.rules]


def test_unclosable_candidates_are_skipped_without_changing_output():
    t, _ = small_graph()
    g = oracle.OracleGraph(t, 4)
    preds = [(P + str(k), int((t[:, 1] == k).sum())) for k in range(4)]
    kw = dict(max_body=2, min_support=5, min_head_coverage=0.01, min_confidence=0.0, max_head_predicates=2)
    pruned = miner.mine(oracle_evaluator(g), preds, **kw)
    full = miner.mine(oracle_evaluator(g), preds, prune_unclosable=False, **kw)
    assert pruned.evaluated < full.evaluated
    key = lambda res: sorted((s.rule.key(), s.support, s.body_size) for s in res.rules)
    assert key(pruned) == key(full)

"""Biomedical-shaped graphs (c4s, c4): hub rules, 64-bit counts, rules split
over workers.

c4s (30k entities, 680k triples) is checked exactly against the reference's
CPU_01 results committed in tests/golden/synthetic_c4s.json.  The full c4
(300k entities, 6.8M triples, 50,000-in-degree hubs) is checked against the
reference too: its 10 hub rules (tests/golden/c4_seed0_hub.json, 23 minutes
of the reference's CPU code on 6 threads; body sizes compared modulo 2^32,
because the reference sums them in an int and the largest exceed 2^31), and
the C oracle on every other rule.  Size-independent properties add to that:
the slices of a split rule summing to the whole, and a rule with its head
reversed ((?b q ?a) for (?a q ?b)) having the same body size although the
engine enumerates it from the other end.
"""
import hashlib

import numpy as np
import pytest

import oracle
from conftest import load_fixture
import masterthesis_gpu_acceleration_b200 as eng
from masterthesis_gpu_acceleration_b200 import synth

INT_MAX = 2**31 - 1
HUB_RULES = range(10)   # the generator's first 10 rules use a hub predicate


def mirrored(rule: str) -> str:
    """The same body with the head's subject and object exchanged."""
    body, head = rule.rsplit("=>", 1)
    head = head.replace("?a", "?_x").replace("?b", "?a").replace("?_x", "?b")
    return body + "=>" + head


def test_mirrored_rule_swaps_head_terms():
    assert mirrored("(?a <p> ?v1) ^ (?v1 <q> ?b) => (?a <r> ?b)") == "(?a <p> ?v1) ^ (?v1 <q> ?b) => (?b <r> ?a)"


@pytest.fixture(scope="module")
def c4s(data_dir):
    fx = load_fixture("synthetic_c4s.json")
    d = synth.generate("c4s", data_dir / "c4s", seed=fx["seed"])
    assert hashlib.sha256((d / "triples.bin").read_bytes()).hexdigest() == fx["triples_sha256"]
    exp = np.array([[e[k] for k in ("support", "headSize", "headSupport", "bodySize")] for e in fx["expected"]],
                   dtype=np.int64)
    with eng.GpuRulesLib(d / "graph.ttl") as lib:
        yield lib, fx["rules"], exp


@pytest.mark.gpu
def test_c4s_batch_counts_match_reference(c4s):
    lib, rules, exp = c4s
    b = lib.prepare_batch(rules)
    res, st, _ = b.run()
    got = b.counts()
    b.close()
    bad = np.nonzero((got != exp).any(axis=1))[0]
    assert len(bad) == 0, f"rules {bad.tolist()} differ: {got[bad].tolist()} vs {exp[bad].tolist()}"
    assert [r.bodySize for r in res] == exp[:, 3].tolist()   # all below INT_MAX here


@pytest.mark.gpu
@pytest.mark.parametrize("n", [2, 3, 8])
def test_c4s_split_rules_sum_to_reference(c4s, n):
    lib, rules, exp = c4s
    for i in list(HUB_RULES) + [42]:
        parts = np.array([lib.evaluate_rule_shard(rules[i], k, n) for k in range(n)])
        assert parts[:, 0].sum() == exp[i, 0] and parts[:, 3].sum() == exp[i, 3], (i, parts.tolist())
        assert (parts[:, 1] == exp[i, 1]).all() and (parts[:, 2] == exp[i, 2]).all()


@pytest.mark.gpu
def test_shard_rejects_bad_arguments(c4s):
    lib, rules, _ = c4s
    for k, n in ((2, 2), (-1, 2), (0, 0)):
        with pytest.raises(RuntimeError):
            lib.evaluate_rule_shard(rules[0], k, n)


@pytest.fixture(scope="module")
def c4(data_dir):
    d = synth.generate("c4", data_dir / "c4", seed=0)
    with eng.GpuRulesLib(d / "graph.ttl") as lib:
        rules = synth.read_rules(d)
        b = lib.prepare_batch(rules)
        res, st, _ = b.run()
        cnt = b.counts()
        b.close()
        yield lib, d, rules, res, cnt


@pytest.mark.gpu
def test_c4_plain_rules_match_oracle(c4):
    """Every rule that does not cross a hub, against the C oracle at full size."""
    lib, d, rules, _, cnt = c4
    g = oracle.OracleGraph(synth.read_triples(d), int(synth.read_meta(d)["predicates"]))
    ir = np.concatenate(oracle.split_ir(synth.read_rule_ir(d))[10:])
    want, status = g.evaluate_ir(ir, len(rules) - 10)
    g.close()
    assert (status == 0).all()
    bad = np.nonzero((cnt[10:] != want).any(axis=1))[0]
    assert len(bad) == 0, f"rules {(bad + 10).tolist()} differ"


@pytest.mark.gpu
def test_c4_hub_rules_exceed_int_and_saturate(c4):
    _, _, _, res, cnt = c4
    big = [i for i in HUB_RULES if cnt[i, 3] > INT_MAX]
    assert big, "the two-sided hub rules reach more than 2^31 body pairs"
    for i in range(len(res)):
        assert res[i].bodySize == min(cnt[i, 3], INT_MAX)


@pytest.mark.gpu
def test_c4_mirrored_heads_have_equal_body_size(c4):
    lib, _, rules, _, cnt = c4
    b = lib.prepare_batch([mirrored(r) for r in rules])
    b.run()
    m = b.counts()
    b.close()
    assert (m[:, 3] == cnt[:, 3]).all(), np.nonzero(m[:, 3] != cnt[:, 3])[0].tolist()


@pytest.mark.gpu
def test_c4_split_hub_rules_sum_to_whole(c4):
    lib, _, rules, _, cnt = c4
    for i in HUB_RULES:
        parts = np.array([lib.evaluate_rule_shard(rules[i], k, 4) for k in range(4)])
        assert parts[:, 0].sum() == cnt[i, 0] and parts[:, 3].sum() == cnt[i, 3], (i, parts.tolist())


def _as_int32(x: int) -> int:
    """x reduced the way the reference's `int` accumulator wraps it."""
    x &= 0xFFFFFFFF
    return x - (1 << 32) if x >= (1 << 31) else x


def test_int32_wrap_helper():
    assert _as_int32(5) == 5 and _as_int32(2**31) == -2**31 and _as_int32(2**32 + 7) == 7
    assert _as_int32(8_800_000_000) == 8_800_000_000 - 2 * 2**32


@pytest.mark.gpu
def test_c4_hub_rules_match_reference(c4):
    """The 10 hub rules of the full c4 graph against the reference's own
    CPU_01 results (tests/golden/c4_seed0_hub.json, run by
    tests/golden/make_golden.py --c4-hub): support and head sizes exactly,
    body sizes exactly modulo 2^32, because CPU_01 sums them in an int
    (SupportCounting.cpp, countBodySize) and the largest exceed 2^31 here."""
    _, d, rules, _, cnt = c4
    fx = load_fixture("c4_seed0_hub.json")
    assert hashlib.sha256((d / "triples.bin").read_bytes()).hexdigest() == fx["triples_sha256"]
    for k, i in enumerate(fx["rules_index"]):
        assert rules[i] == fx["rules"][k]
        e = fx["expected"][k]
        assert [int(cnt[i, 0]), int(cnt[i, 1]), int(cnt[i, 2])] == [e["support"], e["headSize"], e["headSupport"]], i
        assert _as_int32(int(cnt[i, 3])) == e["bodySize_ref"], (i, int(cnt[i, 3]), e["bodySize_ref"])

"""Three-step suffix memos (memo3_* in kernels.cu) against the C oracle.

A body-size plan hS -> x -> v2 -> v3 -> hO whose x is a memoised hub row
answers an item (a, x) from x's memo: the values h reached by paths
x -> v2 -> v3 -> h with x, v2, v3, h distinct, with their path counts, less
the h whose every path runs through a.  The graph below makes that
correction matter: head subjects a are drawn from the same entities as the
hub rows' neighbours v2 and the sparse second and third steps, so a is often
a neighbour of x (a = v2), a value of the second step (a = v3) or both, and
hO values are often neighbours of x too.  Both hub relations and every
orientation of the other body atoms are evaluated with the memos on (every hub row
memoised), off (GPU_RULES_MEMO3=0) and without hub rows; all must give the
oracle's counts exactly.
"""
import itertools

import numpy as np
import pytest

import masterthesis_gpu_acceleration_b200 as eng
from conftest import terms_to_ir

pytestmark = pytest.mark.gpu

COUNT_FIELDS = ("support", "headSize", "headSupport", "bodySize")
P_ROOT, P_HUB, P_HUB_IN, P_STEP2, P_STEP3, P_HEAD = range(6)


def memo3_graph(out_dir, seed=11):
    """Entities 0..9 are hubs x, 10..309 the rest (R).  p0: a -> x (R to
    one or two hubs, and one hub to each of R), p1: x -> v (each hub to 40 of R), p2: v -> x (40 of R into each
    hub), p3: R -> R with out-degree 1-2, p4: R -> R and R -> hub with
    out-degree 1-2, p5 (head): half body pairs of the first rule, half
    random.  Returns (ttl path, rules, int64 counts [n, 4])."""
    import oracle
    rng = np.random.default_rng(seed)
    hubs = np.arange(10)
    rest = 10 + np.arange(300)
    trip = set()
    for a in rest:
        for x in rng.choice(hubs, rng.integers(1, 3), replace=False):
            trip.add((int(a), P_ROOT, int(x)))
        trip.add((int(rng.choice(hubs)), P_ROOT, int(a)))
    for x in hubs:
        for v in rng.choice(rest, 40, replace=False):
            trip.add((int(x), P_HUB, int(v)))
        for v in rng.choice(rest, 40, replace=False):
            trip.add((int(v), P_HUB_IN, int(x)))
    for v in rest:
        for w in rng.choice(rest, rng.integers(1, 3), replace=False):
            if w != v:
                trip.add((int(v), P_STEP2, int(w)))
        pool = np.concatenate([rest, hubs])
        for w in rng.choice(pool, rng.integers(1, 3), replace=False):
            if w != v:
                trip.add((int(v), P_STEP3, int(w)))
    # head pairs: some reachable through the first rule's body, some random
    out = {}
    for s, p, o in trip:
        out.setdefault((p, s), []).append(o)
    heads = set()
    for a in rng.choice(rest, 150, replace=False):
        for x in out.get((P_ROOT, int(a)), []):
            for v2 in out.get((P_HUB, x), [])[:5]:
                for v3 in out.get((P_STEP2, v2), []):
                    for b in out.get((P_STEP3, v3), []):
                        heads.add((int(a), P_HEAD, int(b)))
    while len(heads) < 900:
        heads.add((int(rng.choice(rest)), P_HEAD, int(rng.choice(rest))))
    trip = np.array(sorted(trip | heads), dtype=np.int32)
    out_dir.mkdir(parents=True, exist_ok=True)
    ttl = out_dir / "memo3.ttl"
    with open(ttl, "w") as f:
        for s, p, o in trip.tolist():
            f.write(f"<http://m/e{s}> <http://m/p{p}> <http://m/e{o}> .\n")

    def atom(p, s, o, flip):
        return (p, ("v", o), ("v", s)) if flip else (p, ("v", s), ("v", o))

    rules, terms = [], []
    for hub_pred, flips in itertools.product((P_HUB, P_HUB_IN), itertools.product((0, 1), repeat=3)):
        # the hub step runs x -> v2: through p2 it is written (?v2 p2 ?x)
        body = [atom(P_ROOT, "a", "x", flips[0]), atom(hub_pred, "x", "v2", hub_pred == P_HUB_IN),
                atom(P_STEP2, "v2", "v3", flips[1]), atom(P_STEP3, "v3", "b", flips[2])]
        head = atom(P_HEAD, "a", "b", flips[0] ^ flips[1])
        terms.append(body + [head])

        def text(t):
            p, (_, s), (_, o) = t
            return f"(?{s} <http://m/p{p}> ?{o})"
        rules.append(" ^ ".join(text(t) for t in body) + " => " + text(head))
    g = oracle.OracleGraph(trip, P_HEAD + 1)
    counts, st = g.evaluate_ir(terms_to_ir(terms), len(rules))
    g.close()
    assert (st == 0).all()
    return ttl, rules, counts


def saturating_graph(out_dir, seed=5):
    """One hub x (entity 0) with 500 neighbours v2 among R = 1..600; every
    entity of R has two second-step values in V3 = 401..420 and V3 three
    third-step values in H = 421..430, so about 300 paths reach each h
    (path counts saturate at 255).  Every entity of R is a root a -> x, so
    a is often a neighbour of x and sometimes in V3 or H.  Returns (ttl,
    rules, int64 counts [n, 4])."""
    import oracle
    rng = np.random.default_rng(seed)
    R = np.arange(1, 601)
    V3, H = np.arange(401, 421), np.arange(421, 431)
    trip = {(int(a), P_ROOT, 0) for a in R}
    trip |= {(0, P_HUB, int(v)) for v in R[:500]}
    for v in R:
        for w in rng.choice(V3, 2, replace=False):
            if w != v:
                trip.add((int(v), P_STEP2, int(w)))
    for v in V3:
        for w in rng.choice(H, 3, replace=False):
            trip.add((int(v), P_STEP3, int(w)))
    heads = set()
    while len(heads) < 1500:
        heads.add((int(rng.choice(R)), P_HEAD, int(rng.choice(H))))
    trip = np.array(sorted(trip | heads), dtype=np.int32)
    out_dir.mkdir(parents=True, exist_ok=True)
    ttl = out_dir / "saturating.ttl"
    with open(ttl, "w") as f:
        for s_, p_, o_ in trip.tolist():
            f.write(f"<http://m/e{s_}> <http://m/p{p_}> <http://m/e{o_}> .\n")
    terms = [[(P_ROOT, ("v", "a"), ("v", "x")), (P_HUB, ("v", "x"), ("v", "v2")),
              (P_STEP2, ("v", "v2"), ("v", "v3")), (P_STEP3, ("v", "v3"), ("v", "b")),
              (P_HEAD, ("v", "a"), ("v", "b"))]]
    rules = ["(?a <http://m/p0> ?x) ^ (?x <http://m/p1> ?v2) ^ (?v2 <http://m/p3> ?v3) ^ "
             "(?v3 <http://m/p4> ?b) => (?a <http://m/p5> ?b)"]
    g = oracle.OracleGraph(trip, P_HEAD + 1)
    counts, st = g.evaluate_ir(terms_to_ir(terms), len(rules))
    g.close()
    assert (st == 0).all()
    return ttl, rules, counts


@pytest.fixture(scope="module")
def memo3_case(tmp_path_factory):
    return memo3_graph(tmp_path_factory.mktemp("memo3"))


@pytest.mark.parametrize("memo3", ["1", "0"])
def test_three_step_memo_saturated_counts(tmp_path, memo3, monkeypatch):
    ttl, rules, exp = saturating_graph(tmp_path)
    assert exp[0, 3] > 0
    monkeypatch.setenv("GPU_RULES_MEMO3", memo3)
    monkeypatch.setenv("GPU_RULES_MEMO_GAIN", "0")
    with eng.GpuRulesLib(ttl) as lib:
        got = _counts(lib, rules)
        assert got[0].tolist() == exp[0].tolist()
        r = lib.evaluate_rule(rules[0])
        assert [r.support, r.headSize, r.headSupport, r.bodySize] == exp[0].tolist()


def _counts(lib, rules):
    b = lib.prepare_batch(rules)
    b.run()
    got = b.counts()
    b.close()
    return got


@pytest.mark.parametrize("memo3,hub_min,memo_gain", [("1", "8", "0"), ("1", "8", "0.25"), ("0", "8", "0"),
                                                     ("1", "0", "0")])
def test_three_step_memo_counts(memo3_case, memo3, hub_min, memo_gain, monkeypatch):
    ttl, rules, exp = memo3_case
    monkeypatch.setenv("GPU_RULES_MEMO3", memo3)
    monkeypatch.setenv("GPU_RULES_HUB_MIN_DEGREE", hub_min)
    monkeypatch.setenv("GPU_RULES_MEMO_GAIN", memo_gain)
    with eng.GpuRulesLib(ttl) as lib:
        got = _counts(lib, rules)
        bad = [(i, rules[i], got[i].tolist(), exp[i].tolist()) for i in range(len(rules))
               if not (got[i] == exp[i]).all()]
        assert not bad, f"{len(bad)} of {len(rules)} rules differ, first: {bad[:2]}"
        for i in range(0, len(rules), 5):
            r = lib.evaluate_rule(rules[i])
            assert [r.support, r.headSize, r.headSupport, r.bodySize] == exp[i].tolist(), rules[i]

"""Test helper: scores miner rules with the C oracle (synthetic graphs name
predicate k <http://p/k>)."""
import numpy as np

import oracle


def rule_ir(rule) -> list[int]:
    ids: dict[str, int] = {}

    def var(v):
        if v not in ids:
            ids[v] = len(ids)
        return ids[v]

    body = [[int(p.rsplit("/", 1)[1]), 0, var(s), 0, var(o)] for s, p, o in rule.body]
    hs, hp, ho = rule.head
    head = [int(hp.rsplit("/", 1)[1]), 0, var(hs), 0, var(ho)]
    out = [len(body)] + head
    for a in body:
        out += a
    return out


def oracle_evaluator(graph: "oracle.OracleGraph"):
    def run(rules):
        ir = np.array([x for r in rules for x in rule_ir(r)], dtype=np.int32)
        counts, _ = graph.evaluate_ir(ir, len(rules))
        return oracle.measures(counts)
    return run


def small_graph(seed: int = 3, n_ent: int = 200, n_pred: int = 4, n_triples: int = 2000):
    """A small random graph: (triples int32 [n, 3], Turtle text)."""
    rng = np.random.default_rng(seed)
    t = set()
    while len(t) < n_triples:
        t.add((int(rng.integers(n_ent)), int(rng.integers(n_pred)), int(rng.integers(n_ent))))
    arr = np.array(sorted(t), dtype=np.int32)
    ttl = "".join(f"<http://e/{s}> <http://p/{p}> <http://e/{o}> .\n" for s, p, o in arr.tolist())
    return arr, ttl

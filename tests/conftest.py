import json
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = Path(__file__).resolve().parent / "golden"
sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def load_fixture(name: str) -> dict:
    return json.loads((GOLDEN / name).read_text())


def fuzz_names():
    return sorted(p.name for p in GOLDEN.glob("fuzz_*.json"))


def terms_to_ir(rule_terms, ) -> np.ndarray:
    """Rule IR (oracle input) from the fixture's term lists; variables get
    ids in first-seen order (body atoms, then the head), as the reference's
    parser assigns them; unknown constants keep their distinct negative ids."""
    out = []
    for atoms in rule_terms:
        body, head = atoms[:-1], atoms[-1]
        ids = {}

        def term(t):
            kind, v = t
            if kind == "v":
                if v not in ids:
                    ids[v] = len(ids)
                return [0, ids[v]]
            return [1, v]

        enc_body = []
        for p, s, o in body:
            enc_body.append([p] + term(s) + term(o))
        hp, hs, ho = head
        enc_head = [hp] + term(hs) + term(ho)
        out.append(len(body))
        out.extend(enc_head)
        for a in enc_body:
            out.extend(a)
    return np.array(out, dtype=np.int32)


@pytest.fixture(scope="session")
def data_dir(tmp_path_factory):
    return tmp_path_factory.mktemp("kg")


def wide_domain_graph(out_dir: Path):
    """A graph whose body-size pairs need more than a block's shared memory.

    Predicate p0 links 50 middle entities x to 8,000 distinct objects each
    (400,000 distinct objects: an hO domain of 12,500 bitmap words, above the
    shared pool), p1 and p2 link 100 and 200 head subjects to 3 random x each,
    p3 holds 2,000 head triples (half of them body pairs).  The rules chain
    (?a p1|p2 ?x) ^ (?x p0 ?b) under (?a p3 ?b) and its mirror, so per-phase
    global bitmap rows take 5 MB (p1) and 10 MB (p2).  Expected counts come
    from the C oracle, which the reference's fixtures pin.
    Returns (ttl path, rules, int64 counts [n, 4])."""
    import oracle
    rng = np.random.default_rng(7)
    n_x, per_x = 50, 8000
    xs = np.arange(n_x)
    objs = n_x + np.arange(n_x * per_x)
    t0 = np.stack([np.repeat(xs, per_x), np.zeros(n_x * per_x, dtype=np.int64), objs], axis=1)
    nxt = int(objs[-1]) + 1
    s1 = nxt + np.arange(100)
    s2 = nxt + 100 + np.arange(200)
    rows = [t0]
    for p, subj in ((1, s1), (2, s2)):
        for s in subj:
            for x in rng.choice(n_x, 3, replace=False):
                rows.append(np.array([[s, p, x]]))
    trip = np.concatenate(rows).astype(np.int64)
    # head triples: half of them body pairs of p1, the rest random pairs
    heads = set()
    by_x = {int(x): objs[int(x) * per_x:(int(x) + 1) * per_x] for x in xs}
    a_x = [(int(s), int(x)) for s, p, x in trip if p == 1]
    while len(heads) < 1000:
        s, x = a_x[rng.integers(len(a_x))]
        heads.add((s, int(by_x[x][rng.integers(per_x)])))
    every = np.concatenate([s1, s2])
    while len(heads) < 2000:
        heads.add((int(every[rng.integers(len(every))]), int(objs[rng.integers(len(objs))])))
    trip = np.concatenate([trip, np.array([[s, 3, o] for s, o in sorted(heads)])]).astype(np.int32)
    out_dir.mkdir(parents=True, exist_ok=True)
    ttl = out_dir / "wide.ttl"
    with open(ttl, "w") as f:
        for s, p, o in trip.tolist():
            f.write(f"<http://w/e{s}> <http://w/p{p}> <http://w/e{o}> .\n")
    rules = [
        "(?a <http://w/p1> ?x) ^ (?x <http://w/p0> ?b) => (?a <http://w/p3> ?b)",
        "(?a <http://w/p2> ?x) ^ (?x <http://w/p0> ?b) => (?a <http://w/p3> ?b)",
        "(?a <http://w/p1> ?x) ^ (?x <http://w/p0> ?b) => (?b <http://w/p3> ?a)",
        "(?x <http://w/p0> ?b) ^ (?a <http://w/p2> ?x) => (?a <http://w/p3> ?b)",
    ]
    # IR: variables in first-seen order over the body atoms, then the head
    terms = [
        [(1, ("v", "a"), ("v", "x")), (0, ("v", "x"), ("v", "b")), (3, ("v", "a"), ("v", "b"))],
        [(2, ("v", "a"), ("v", "x")), (0, ("v", "x"), ("v", "b")), (3, ("v", "a"), ("v", "b"))],
        [(1, ("v", "a"), ("v", "x")), (0, ("v", "x"), ("v", "b")), (3, ("v", "b"), ("v", "a"))],
        [(0, ("v", "x"), ("v", "b")), (2, ("v", "a"), ("v", "x")), (3, ("v", "a"), ("v", "b"))],
    ]
    g = oracle.OracleGraph(trip, 4)
    counts, st = g.evaluate_ir(terms_to_ir(terms), len(rules))
    g.close()
    assert (st == 0).all()
    return ttl, rules, counts

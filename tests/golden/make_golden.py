"""Regenerates the golden fixtures under tests/golden/ (run in a checkout
that has the reference sources; needs oracle/_ref/cpu01_harness).

Every expected value here comes from the reference's own CPU_01_nonparallel
code (compiled by oracle/build_ref.sh and driven by oracle/ref_harness.cpp)
run on the Turtle graph and rule file the fixture describes.  Nothing is
computed by the engine or by the C restatement.

Fixtures:
  synthetic_<cfg>.json   c1 / c2 / c2s / c4s, seed 0: the generator's rules
                         and the reference's measures, plus a checksum of the
                         graph (c4s: the biomedical shape at a tenth of the
                         size, hub rules included; generated with --threads)
  c3_seed0.npz           all 10,000 c3 rules: support, headSize, headSupport,
                         bodySize per rule (generated with --threads)
  c4_seed0_hub.json      the 10 hub rules of the full c4 graph (body sizes
                         above 2^31 come out wrapped by the reference's int;
                         run separately with --c4-hub: 23 minutes on 6
                         threads)
  fuzz_<k>.json          small dense graphs with prefixes, literals,
                         self-loops and constants, and random rules that use
                         constants, unknown terms, repeated atoms, empty bodies,
                         shared variables, JSON syntax and '|' suffixes
  edge_cases.json        hand-written rules, each pinning one semantic point
"""
from __future__ import annotations

import hashlib
import json
import random
import sys
import tempfile
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

import oracle  # noqa: E402
from masterthesis_gpu_acceleration_b200 import synth  # noqa: E402

OUT = Path(__file__).resolve().parent


def sha(path: Path) -> str:
    return hashlib.sha256(path.read_bytes()).hexdigest()


def ref_rows(ttl: Path, rules: Path, threads: int = 1):
    rows, _ = oracle.run_reference(ttl, rules, threads=threads)
    return [{k: r[k] for k in ("support", "headSize", "headSupport", "bodySize", "headCoverage", "confidence")}
            for r in rows]


def synthetic(cfg: str, tmp: Path, threads: int = 1):
    d = synth.generate(cfg, tmp / cfg, seed=0)
    fx = {
        "config": cfg, "seed": 0,
        "triples_sha256": sha(d / "triples.bin"),
        "rules": synth.read_rules(d),
        "expected": ref_rows(d / "graph.ttl", d / "rules.txt", threads=threads),
    }
    (OUT / f"synthetic_{cfg}.json").write_text(json.dumps(fx, indent=1))


def c3(tmp: Path):
    d = synth.generate("c3", tmp / "c3", seed=0)
    rows = ref_rows(d / "graph.ttl", d / "rules.txt", threads=8)
    arr = np.array([[r["support"], r["headSize"], r["headSupport"], r["bodySize"]] for r in rows], dtype=np.int64)
    np.savez_compressed(OUT / "c3_seed0.npz", expected=arr,
                        triples_sha256=np.array(sha(d / "triples.bin")),
                        rules_sha256=np.array(sha(d / "rules.txt")))


# ---------------------------------------------------------------- fuzz graphs

class Fuzz:
    """A small dense graph with mixed term spellings."""

    def __init__(self, rnd: random.Random, n_ent: int, n_pred: int, n_triples: int):
        self.rnd = rnd
        self.n_ent, self.n_pred = n_ent, n_pred
        # entity 0..n-1; the last few are literals (object position only)
        self.n_lit = 3
        trip = set()
        while len(trip) < n_triples:
            s = rnd.randrange(n_ent - self.n_lit)
            p = rnd.randrange(n_pred)
            o = rnd.randrange(n_ent)
            if rnd.random() < 0.05:
                o = s  # self-loop
            trip.add((s, p, o))
        self.triples = sorted(trip)

    # spellings in the graph file
    def ent_ttl(self, e: int) -> str:
        if e >= self.n_ent - self.n_lit:
            return f'"lit{e}"'
        return f"ex:e{e}" if e % 3 == 0 else f"<http://x/e{e}>"

    def pred_ttl(self, p: int) -> str:
        return f"ex:p{p}" if p % 2 else f"<http://x/p{p}>"

    def ttl(self) -> str:
        lines = ["@prefix ex: <http://x/> .", "# fuzz graph"]
        by_subj = {}
        for s, p, o in self.triples:
            by_subj.setdefault(s, []).append((p, o))
        for s, po in by_subj.items():
            parts = [f"{self.pred_ttl(p)} {self.ent_ttl(o)}" for p, o in po]
            lines.append(f"{self.ent_ttl(s)} " + " ;\n    ".join(parts) + " .")
        return "\n".join(lines) + "\n"

    # spellings in rules
    def ent_rule(self, e: int) -> str:
        if e < 0:
            return "<http://x/nope>" if e == -1 else "ex:nope2"
        if e >= self.n_ent - self.n_lit:
            return f'"lit{e}"'
        return f"ex:e{e}" if e % 2 else f"<http://x/e{e}>"

    def pred_rule(self, p: int) -> str:
        if p < 0:
            return "<http://x/unknownPred>"
        return f"ex:p{p}" if p % 2 == 0 else f"<http://x/p{p}>"


def rule_text(fz: Fuzz, body, head) -> str:
    def term(t):
        kind, v = t
        return v if kind == "v" else fz.ent_rule(v)

    def atom(a):
        p, s, o = a
        return f"({term(s)} {fz.pred_rule(p)} {term(o)})"

    return " ^ ".join(atom(a) for a in body) + " => " + atom(head)


def rule_json(fz: Fuzz, body, head) -> str:
    def term(t):
        kind, v = t
        if kind == "v":
            return {"type": "variable", "value": v}
        return {"type": "constant", "value": fz.ent_rule(v)}

    def atom(a):
        p, s, o = a
        return {"subject": term(s), "predicate": fz.pred_rule(p), "object": term(o)}

    return json.dumps({"body": [atom(a) for a in body], "head": atom(head)})


def random_rule(fz: Fuzz, rnd: random.Random):
    vars_ = ["?a", "?b", "?c", "?d", "?e"]

    def term():
        r = rnd.random()
        if r < 0.78:
            return ("v", rnd.choice(vars_))
        if r < 0.97:
            return ("c", rnd.randrange(fz.n_ent))
        return ("c", -1 if rnd.random() < 0.5 else -2)

    def pred():
        return -1 if rnd.random() < 0.02 else rnd.randrange(fz.n_pred)

    L = rnd.choice([0, 1, 1, 2, 2, 2, 3, 3, 3, 4, 4, 5])
    if rnd.random() < 0.5:
        # closed chain with random directions, occasionally perturbed
        chain = ["?a"] + [f"?v{i}" for i in range(1, L)] + ["?b"] if L else ["?a", "?b"]
        body = []
        for i in range(L):
            x, y = ("v", chain[i]), ("v", chain[i + 1])
            body.append((pred(), y, x) if rnd.random() < 0.5 else (pred(), x, y))
        if body and rnd.random() < 0.3:
            k = rnd.randrange(len(body))
            p, s, o = body[k]
            body[k] = (p, term(), o) if rnd.random() < 0.5 else (p, s, term())
        head = (pred(), ("v", "?a"), ("v", "?b"))
        if rnd.random() < 0.15:
            head = (head[0], term(), head[2])
        if body and rnd.random() < 0.1:
            body.append(rnd.choice(body))        # repeated atom
        if body and rnd.random() < 0.1:
            body[rnd.randrange(len(body))] = head  # body atom equal to the head
    else:
        body = [(pred(), term(), term()) for _ in range(L)]
        head = (pred(), term(), term())
    return body[:8], head


def fuzz_fixture(k: int, tmp: Path, n_rules: int):
    rnd = random.Random(1000 + k)
    fz = Fuzz(rnd, n_ent=[14, 20, 28][k % 3], n_pred=[2, 3, 4][k % 3], n_triples=[60, 110, 160][k % 3])
    d = tmp / f"fuzz{k}"
    d.mkdir(parents=True, exist_ok=True)
    (d / "graph.ttl").write_text(fz.ttl())
    rules = [random_rule(fz, rnd) for _ in range(n_rules)]
    texts = []
    for i, (b, h) in enumerate(rules):
        t = rule_text(fz, b, h)
        if i % 7 == 3:
            t = "  " + t.replace("(", "( ").replace(")", " )") + "  | 0.5 0.1"
        texts.append(t)
    (d / "rules.txt").write_text("\n".join(texts) + "\n")
    expected = ref_rows(d / "graph.ttl", d / "rules.txt")
    # JSON spelling of the same rules, checked through the reference's JSON reader
    jsons = [rule_json(fz, b, h) for b, h in rules]
    (d / "rules.json").write_text("[\n" + ",\n".join(jsons) + "\n]\n")
    expected_json = ref_rows(d / "graph.ttl", d / "rules.json")
    fx = {
        "ttl": fz.ttl(),
        "rules": texts,
        "rules_json": jsons,
        "triples": [list(t) for t in fz.triples],
        "n_pred": fz.n_pred,
        "n_ent": fz.n_ent,
        "rule_terms": [[[p, list(s), list(o)] for p, s, o in b] + [[h[0], list(h[1]), list(h[2])]] for b, h in rules],
        "expected": expected,
        "expected_json": expected_json,
    }
    (OUT / f"fuzz_{k}.json").write_text(json.dumps(fx))


EDGE_TTL = """@prefix ex: <http://x/> .
ex:a ex:p ex:b , ex:c , ex:a .
ex:b ex:p ex:c ; ex:q ex:d .
ex:c ex:p ex:a ; ex:q "v1" .
ex:d ex:q ex:a ; ex:r ex:d .
<http://x/e> ex:p ex:b ; ex:q ex:b ; ex:r ex:e .
ex:b ex:r ex:b .
"""

EDGE_RULES = [
    ("head repeated in the body: the head triple is used (support 0)",
     "(?x ex:p ?y) => (?x ex:p ?y)"),
    ("two identical body atoms never ground", "(?x ex:p ?y) ^ (?x ex:p ?y) => (?x ex:q ?y)"),
    ("self-loop atom", "(?x ex:r ?x) => (?x ex:p ?x)"),
    ("head with one variable in both positions", "(?x ex:p ?y) ^ (?y ex:p ?x) => (?x ex:r ?x)"),
    ("hO absent from the body counts hS values", "(?x ex:p ?z) => (?x ex:q ?y)"),
    ("hS absent from the body: no seed, body size 0", "(?z ex:p ?y) => (?x ex:q ?y)"),
    ("constant head object", "(?x ex:p ?y) => (?x ex:q ex:b)"),
    ("constant head subject", "(?x ex:p ?y) => (ex:b ex:q ?y)"),
    ("constant head, both terms", "(?x ex:p ?y) => (ex:b ex:q ex:d)"),
    ("constant in the body", "(?x ex:p ?y) ^ (?y ex:q ex:d) => (?x ex:r ?y)"),
    ("constant meets the head variable: runtime used-triple check",
     "(ex:b ex:p ?y) ^ (?x ex:q ?y) => (?x ex:p ?y)"),
    ("literal constant", "(?x ex:q \"v1\") => (?x ex:p ?y)"),
    ("unknown predicate in the body", "(?x <http://x/none> ?y) => (?x ex:p ?y)"),
    ("unknown predicate in the head (body size still counted)", "(?x ex:p ?y) => (?x <http://x/none> ?y)"),
    ("unknown constant", "(?x ex:p <http://x/none>) => (?x ex:p ?y)"),
    ("empty body", " => (?x ex:p ?y)"),
    ("disconnected atom is scanned", "(?u ex:q ?w) ^ (?x ex:p ?y) => (?x ex:r ?y)"),
    ("injectivity across the chain", "(?x ex:p ?z) ^ (?z ex:p ?y) => (?x ex:p ?y)"),
    ("score tail after '|'", "(?x ex:p ?y) => (?y ex:p ?x) | 0.3"),
    ("padded parentheses", "( ?x ex:p ?y ) ^ ( ?y ex:q ?z ) => ( ?x ex:q ?z )"),
    ("full IRIs", "(?x <http://x/p> ?y) => (?x <http://x/q> ?y)"),
    ("eight body atoms",
     "(?a ex:p ?b) ^ (?b ex:p ?c) ^ (?c ex:p ?d) ^ (?d ex:p ?e) ^ (?e ex:p ?f) ^ (?f ex:p ?g) ^ (?g ex:p ?h) ^ (?h ex:p ?i) => (?a ex:p ?i)"),
]


def edge_cases(tmp: Path):
    d = tmp / "edge"
    d.mkdir(parents=True, exist_ok=True)
    (d / "graph.ttl").write_text(EDGE_TTL)
    (d / "rules.txt").write_text("\n".join(r for _, r in EDGE_RULES) + "\n")
    expected = ref_rows(d / "graph.ttl", d / "rules.txt")
    fx = {"ttl": EDGE_TTL, "cases": [{"what": w, "rule": r, "expected": e}
                                     for (w, r), e in zip(EDGE_RULES, expected)]}
    (OUT / "edge_cases.json").write_text(json.dumps(fx, indent=1))


def c4_hub(tmp: Path, threads: int = 6):
    """The 10 hub rules of the full c4 graph (seed 0), run by the reference.

    CPU_01 adds the per-hS pair counts into an `int` (SupportCounting.cpp,
    countBodySize: `int bodySizeResult`), so body sizes above 2^31 come out
    wrapped modulo 2^32; the fixture keeps the reference's value as printed
    (`bodySize_ref`, two's-complement int32) and the engine's 64-bit count is
    compared modulo 2^32.  Support and head sizes fit an int exactly."""
    d = synth.generate("c4", tmp / "c4", seed=0)
    rules = synth.read_rules(d)[:10]
    rf = tmp / "c4_hub_rules.txt"
    rf.write_text("\n".join(rules) + "\n")
    rows, summary = oracle.run_reference(d / "graph.ttl", rf, threads=threads)
    fx = {
        "config": "c4", "seed": 0, "rules_index": list(range(10)),
        "triples_sha256": sha(d / "triples.bin"),
        "rules": rules,
        "expected": [{"support": r["support"], "headSize": r["headSize"], "headSupport": r["headSupport"],
                      "bodySize_ref": r["bodySize"], "supportMs": r["supportMs"], "confidenceMs": r["confidenceMs"]}
                     for r in rows],
        "reference_eval_wall_ms": summary.get("eval_wall_ms"), "threads": threads,
    }
    (OUT / "c4_seed0_hub.json").write_text(json.dumps(fx, indent=1))


def main():
    if not oracle.ref_available():
        oracle.build()
    with tempfile.TemporaryDirectory() as t:
        tmp = Path(t)
        if "--c4-hub" in sys.argv:
            c4_hub(tmp)
            print("fixture written to", OUT / "c4_seed0_hub.json")
            return
        only = [a.split("=", 1)[1] for a in sys.argv if a.startswith("--only=")]
        if only:
            for cfg in only[0].split(","):
                synthetic(cfg, tmp, threads=8)
            print("fixtures written to", OUT)
            return
        for cfg in ("c1", "c2", "c2s"):
            synthetic(cfg, tmp)
        synthetic("c4s", tmp, threads=8)
        edge_cases(tmp)
        for k in range(6):
            fuzz_fixture(k, tmp, n_rules=150)
        if "--no-c3" not in sys.argv:
            c3(tmp)
    print("fixtures written to", OUT)


if __name__ == "__main__":
    main()

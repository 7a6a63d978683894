"""Rule mining around the evaluation path: level-wise candidate generation
with support and head-coverage pruning (the step either side of
gpu_evaluate_rule in RDFRules, which scores one candidate per call,
GPU_03/GpuRulesLib.scala:107-112).

Candidates are Horn rules ``body => (?a p ?b)``.  A rule is refined the way
AMIE-style miners refine it: a *dangling* atom joins one existing variable
to a fresh one, a *closing* atom joins two existing variables.  Support and
head coverage can only fall when an atom is added, so a candidate below
either threshold is not refined further.  A rule is output when it is
closed (every variable occurs at least twice) and its confidence reaches
``min_confidence``.

Every level is scored in one call of ``evaluate`` — by default
``GpuRulesLib.evaluate_rules_batch``, one batched device launch per level —
instead of one call per candidate; ``per_rule=True`` scores them one by one
(the reference's calling pattern) for comparison.  Scores do not depend on
the mode.
"""
from __future__ import annotations

import itertools
from dataclasses import dataclass, field
from typing import Callable, Sequence

Atom = tuple[str, str, str]   # (subject variable, predicate IRI, object variable)
_RENAMED = tuple(f"?x{i}" for i in range(8))   # canonical names of body-only variables


@dataclass(frozen=True)
class Rule:
    head: Atom
    body: tuple[Atom, ...]

    def text(self) -> str:
        body = " ^ ".join(f"({s} <{p}> {o})" for s, p, o in self.body)
        s, p, o = self.head
        return f"{body} => ({s} <{p}> {o})"

    def variables(self) -> list[str]:
        seen: list[str] = []
        for s, _, o in (self.head,) + self.body:
            for v in (s, o):
                if v not in seen:
                    seen.append(v)
        return seen

    def closed(self) -> bool:
        return self.singletons() == 0

    def singletons(self) -> int:
        """Variables that occur once (head included).  A dangling atom never
        lowers the count and a closing atom lowers it by at most 2, so a rule
        with more than 2 x (atoms still to add) of them never closes."""
        count: dict[str, int] = {}
        for s, _, o in (self.head,) + self.body:
            count[s] = count.get(s, 0) + 1
            count[o] = count.get(o, 0) + 1
        return sum(1 for c in count.values() if c == 1)

    def key(self) -> tuple:
        """Canonical form: the smallest sorted atom list over renamings of
        the body-only variables (the head keeps ?a and ?b)."""
        hs, _, ho = self.head
        extra: list[str] = []   # body-only variables in first-occurrence order
        for s, _, o in self.body:
            if s != hs and s != ho and s not in extra:
                extra.append(s)
            if o != hs and o != ho and o not in extra:
                extra.append(o)
        if not extra:
            return (self.head, tuple(sorted(self.body)))
        best = None
        for perm in itertools.permutations(_RENAMED[:len(extra)]):
            ren = dict(zip(extra, perm))
            atoms = tuple(sorted((ren.get(s, s), p, ren.get(o, o)) for s, p, o in self.body))
            if best is None or atoms < best:
                best = atoms
        return (self.head, best)


@dataclass
class Scored:
    rule: Rule
    support: int
    head_size: int
    head_coverage: float
    body_size: int
    confidence: float


@dataclass
class MiningResult:
    rules: list[Scored] = field(default_factory=list)     # output rules
    evaluated: int = 0                                   # candidates scored
    levels: list[int] = field(default_factory=list)      # candidates per level


def refinements(rule: Rule, predicates: Sequence[str], max_vars: int) -> list[Rule]:
    """Dangling and closing refinements of `rule` (one added atom)."""
    vars_ = rule.variables()
    fresh = f"?v{len(vars_) - 1}"
    out = []
    have = set(rule.body) | {rule.head}
    for p in predicates:
        for x in vars_:
            if len(vars_) < max_vars:
                for atom in ((x, p, fresh), (fresh, p, x)):
                    out.append(Rule(rule.head, rule.body + (atom,)))
            for y in vars_:
                if y != x and (x, p, y) not in have:
                    out.append(Rule(rule.head, rule.body + ((x, p, y),)))
    return out


def gpu_evaluator(lib, per_rule: bool = False) -> Callable[[list[Rule]], list[dict]]:
    """Scores rules with the engine: one batched call, or one call per rule."""
    def run(rules: list[Rule]) -> list[dict]:
        texts = [r.text() for r in rules]
        res = [lib.evaluate_rule(t) for t in texts] if per_rule else lib.evaluate_rules_batch(texts)[0]
        return [x.as_dict() for x in res]
    return run


def mine(evaluate: Callable[[list[Rule]], list[dict]], predicates: Sequence[tuple[str, int]],
         max_body: int = 2, min_support: int = 2, min_head_coverage: float = 0.01,
         min_confidence: float = 0.1, max_head_predicates: int | None = None, max_vars: int = 4,
         max_candidates: int = 200_000, prune_unclosable: bool = True) -> MiningResult:
    """Level-wise mining of rules with up to `max_body` body atoms.

    predicates: (IRI, triples) of the graph (GpuRulesLib.predicates()); head
    predicates are those with at least `min_support` triples, the largest
    first, at most `max_head_predicates` of them.  prune_unclosable: skip
    candidates that can no longer become closed within `max_body` atoms
    (they could be neither output nor refined into output rules)."""

    def closable(r: Rule) -> bool:
        return not prune_unclosable or r.singletons() <= 2 * (max_body - len(r.body))

    heads = [p for p, n in sorted(predicates, key=lambda x: -x[1]) if n >= min_support]
    if max_head_predicates is not None:
        heads = heads[:max_head_predicates]
    body_preds = [p for p, _ in predicates]
    result = MiningResult()
    seen: set = set()
    frontier = []
    for p in heads:
        head = ("?a", p, "?b")
        for q in body_preds:
            for atom in (("?a", q, "?b"), ("?b", q, "?a"), ("?a", q, "?v0"), ("?v0", q, "?a"),
                         ("?b", q, "?v0"), ("?v0", q, "?b")):
                if atom == head:
                    continue
                r = Rule(head, (atom,))
                if closable(r) and r.key() not in seen:
                    seen.add(r.key())
                    frontier.append(r)
    for level in range(1, max_body + 1):
        frontier = frontier[:max_candidates]
        if not frontier:
            break
        scores = evaluate(frontier)
        result.evaluated += len(frontier)
        result.levels.append(len(frontier))
        keep = []
        for r, m in zip(frontier, scores):
            if m["support"] < min_support or m["headCoverage"] < min_head_coverage:
                continue   # anti-monotone: no refinement can recover
            if r.closed() and m["confidence"] >= min_confidence:
                result.rules.append(Scored(r, m["support"], m["headSize"], m["headCoverage"], m["bodySize"],
                                           m["confidence"]))
            keep.append(r)
        if level == max_body:
            break
        # only the first max_candidates new refinements are scored, so
        # generation stops there (keys of longer bodies never meet these)
        nxt = []
        for r in keep:
            for c in refinements(r, body_preds, max_vars):
                if not closable(c):
                    continue
                k = c.key()
                if k not in seen:
                    seen.add(k)
                    nxt.append(c)
                    if len(nxt) >= max_candidates:
                        break
            if len(nxt) >= max_candidates:
                break
        frontier = nxt
    return result

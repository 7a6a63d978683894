"""Rule-set sharding over GPUs (one process per GPU).

Rules are independent, so the path shards without a data-path collective:
every rank loads the same graph and evaluates its own rules.  Two layouts:

* weak scaling: rank r evaluates a full rule set of its own (the benchmark
  draws it from rule seed r over the same graph);
* strong scaling: one rule list is split into contiguous, nearly equal
  slices, one per rank (``shard_rules``), and the results are gathered back
  in the original order on the host (``gather_results``).

* one giant rule: every rank evaluates its slice of the rule's roots
  (``gpu_evaluate_rule_shard``: head triples for support, head-subject rows
  for body size, cut for equal estimated work) and one int64 sum all-reduce
  adds the partial support and body-size counts (``evaluate_rule_split``).
  Distinct (hS, hO) pairs of different head subjects never collide, so the
  sum is exact.

Apart from that all-reduce the cross-rank communication is host-side
plumbing through torch.distributed: a barrier, the maximum of the ranks'
timed spans, and, for strong scaling, an object gather of result tuples.
"""
from __future__ import annotations

from typing import Sequence


def rule_seed(rank: int) -> int | None:
    """Rule seed of a rank in the weak-scaling layout (rank 0 keeps the
    configuration's standard rule set)."""
    return None if rank == 0 else rank


def shard_bounds(n: int, rank: int, world: int) -> tuple[int, int]:
    """Contiguous slice [lo, hi) of n items for `rank` of `world`."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError("bad rank/world")
    base, extra = divmod(n, world)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def shard_rules(rules: Sequence[str], rank: int, world: int) -> list[str]:
    lo, hi = shard_bounds(len(rules), rank, world)
    return list(rules[lo:hi])


def gather_results(parts: Sequence[Sequence], n: int, world: int) -> list:
    """Reassembles per-rank result lists (in rank order) into one list."""
    out = []
    for r in range(world):
        lo, hi = shard_bounds(n, r, world)
        if len(parts[r]) != hi - lo:
            raise ValueError(f"rank {r} returned {len(parts[r])} results, expected {hi - lo}")
        out.extend(parts[r])
    return out


def max_over_ranks(x: float, group=None, device=None) -> float:
    """Maximum of a per-rank float over the process group (x itself when
    torch.distributed is not initialised)."""
    import torch
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized():
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device or "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())


def weak_value(rules_per_rank: int, world: int, steps: int, max_ms: float) -> float:
    """Whole-job rules/s of the weak-scaling layout."""
    return world * rules_per_rank * steps / (max_ms / 1e3)


def evaluate_rule_split(evaluate_shard, rule: str, group=None, device=None) -> dict:
    """One rule over all ranks of the process group.

    evaluate_shard(rule, shard, n_shards) returns this rank's int64 counts
    [support part, headSize, headSupport, bodySize part] (e.g.
    ``GpuRulesLib.evaluate_rule_shard``).  The support and body-size parts
    are summed over the ranks with one all-reduce (NCCL when ``device`` is a
    CUDA device, else the group's backend); every rank returns the whole
    rule's measures, derived as FinalRule::setMeasures / setConfidence do
    (CPU_01_nonparallel/FinalRule.cpp:19-41)."""
    import torch
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        rank, world = dist.get_rank(group), dist.get_world_size(group)
    else:
        rank, world = 0, 1
    c = [int(x) for x in evaluate_shard(rule, rank, world)]
    part = torch.tensor([c[0], c[3]], dtype=torch.int64, device=device or "cpu")
    if world > 1:
        dist.all_reduce(part, op=dist.ReduceOp.SUM, group=group)
    sup, body = (int(x) for x in part.tolist())
    hsz, hsup = c[1], c[2]
    return {"support": sup, "headSize": hsz, "headSupport": hsup, "bodySize": body,
            "headCoverage": sup / hsz if hsz > 0 else 0.0,
            "confidence": sup / body if body > 0 else 0.0}

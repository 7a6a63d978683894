"""Open-loop serving measurement: Poisson arrivals into the request loop.

Requests are submitted at exponentially distributed intervals (a Poisson
process of the given rate, seeded) regardless of how fast results come back;
a second thread drains results.  Latency is measured inside the library,
from gpu_serve_submit to completion, so Python's scheduling only shifts
arrival times.  For each offered rate the sweep reports the sustained rate
(completed requests over the span from the first submission to the last
completion) and the p50 / p99 latency.
"""
from __future__ import annotations

import threading
import time

import numpy as np


def run_rate(lib, rules, rate: float, duration: float, seed: int = 0, slots: int = 4,
             max_batch: int = 4096, mem_budget: int = 1 << 30, id_base: int = 0):
    """Offers `rate` requests/s for `duration` seconds (rules cycled in order).

    Returns (summary dict, {request_id: (rule_index, status, GpuRuleResult)})."""
    summ, res = run_rate_multi([(lib, rules)], rate, duration, seed=seed, slots=slots, max_batch=max_batch,
                               mem_budget=mem_budget, id_base=id_base)
    return summ, res[0]


def run_rate_multi(graphs, rate: float, duration: float, seed: int = 0, weights=None, slots: int = 4,
                   max_batch: int = 4096, mem_budget: int = 1 << 30, id_base: int = 0):
    """One Poisson stream of `rate` requests/s for `duration` seconds over
    several resident graphs: `graphs` is a list of (GpuRulesLib, rules), each
    graph gets its own server, and every arrival goes to graph g with
    probability weights[g] (uniform by default), taking that graph's next
    rule in order.

    Returns (summary dict with latencies over all graphs and per graph,
    [{request_id: (rule_index, status, GpuRuleResult)} per graph])."""
    rng = np.random.default_rng(seed)
    n = max(1, int(rate * duration))
    at = np.cumsum(rng.exponential(1.0 / rate, size=n))
    k = len(graphs)
    w = np.full(k, 1.0 / k) if weights is None else np.asarray(weights, dtype=float) / np.sum(weights)
    dest = rng.choice(k, size=n, p=w)
    results = [dict() for _ in range(k)]
    lat = [[] for _ in range(k)]
    done = threading.Event()
    servers = [lib.serve(slots=slots, max_batch=max_batch, mem_budget=mem_budget) for lib, _ in graphs]
    try:
        idx_of = {}   # request id -> rule index within its graph's list

        def drain():
            while True:
                for g, sv in enumerate(servers):
                    for rid, st, res, ms in sv.poll(wait_ms=5 if k > 1 else 20):
                        results[g][rid] = (idx_of[rid], st, res)
                        lat[g].append(ms)
                if done.is_set() and sum(len(r) for r in results) >= n:
                    break
        th = threading.Thread(target=drain, daemon=True)
        next_rule = [0] * k
        t0 = time.perf_counter()
        th.start()
        for i in range(n):
            target = t0 + at[i]
            while True:
                now = time.perf_counter()
                if now >= target:
                    break
                if target - now > 0.002:
                    time.sleep(target - now - 0.001)
            g = int(dest[i])
            rules = graphs[g][1]
            ri = next_rule[g] % len(rules)
            next_rule[g] += 1
            idx_of[id_base + i] = ri
            servers[g].submit(id_base + i, rules[ri])
        t_sub = time.perf_counter() - t0
        done.set()
        th.join(timeout=600)
        t_end = time.perf_counter() - t0
        stats = [sv.stats() for sv in servers]
    finally:
        for sv in servers:
            sv.stop()
    every = np.concatenate([np.array(x) for x in lat if x]) if any(lat) else np.zeros(1)
    completed = sum(len(r) for r in results)
    ok = sum(1 for r in results for v in r.values() if v[1] == 0)
    shed = sum(1 for r in results for v in r.values() if v[1] == -4)
    summ = {
        "offered_rules_per_s": rate,
        "submitted": n,
        "completed_ok": ok,
        "shed_over_time_limits": shed,
        "sustained_rules_per_s": completed / t_end if t_end > 0 else 0.0,
        "achieved_arrival_rate": n / t_sub if t_sub > 0 else 0.0,
        "p50_ms": float(np.percentile(every, 50)),
        "p99_ms": float(np.percentile(every, 99)),
        "max_ms": float(every.max()),
        "launches": sum(s["launches"] for s in stats),
        "device_ms": sum(s["device_ms"] for s in stats),
        "host_prepare_ms": sum(s["host_ms"] for s in stats),
    }
    if k > 1:
        summ["per_graph"] = [{"requests": len(lat[g]),
                              "p50_ms": float(np.percentile(lat[g], 50)) if lat[g] else None,
                              "p99_ms": float(np.percentile(lat[g], 99)) if lat[g] else None} for g in range(k)]
    return summ, results


def sweep(lib, rules, rates, duration: float, seed: int = 0, **kw):
    out, allres = [], {}
    base = 0
    for k, r in enumerate(rates):
        summ, res = run_rate(lib, rules, r, duration, seed + k, id_base=base, **kw)
        out.append(summ)
        allres.update(res)
        base += summ["submitted"]
    return out, allres


def sweep_multi(graphs, rates, duration: float, seed: int = 0, **kw):
    """sweep over several resident graphs (run_rate_multi per rate)."""
    out, allres = [], [dict() for _ in graphs]
    base = 0
    for k, r in enumerate(rates):
        summ, res = run_rate_multi(graphs, r, duration, seed + k, id_base=base, **kw)
        out.append(summ)
        for g, x in enumerate(res):
            allres[g].update(x)
        base += summ["submitted"]
    return out, allres

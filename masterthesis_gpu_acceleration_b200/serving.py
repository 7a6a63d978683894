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
    rng = np.random.default_rng(seed)
    n = max(1, int(rate * duration))
    gaps = rng.exponential(1.0 / rate, size=n)
    at = np.cumsum(gaps)
    results = {}
    lat = []
    done = threading.Event()
    with lib.serve(slots=slots, max_batch=max_batch, mem_budget=mem_budget) as sv:
        def drain():
            while not done.is_set() or len(results) < n:
                for rid, st, res, ms in sv.poll(wait_ms=20):
                    results[rid] = ((rid - id_base) % len(rules), st, res)
                    lat.append(ms)
                if done.is_set() and len(results) >= n:
                    break
        th = threading.Thread(target=drain, daemon=True)
        th.start()
        t0 = time.perf_counter()
        for i in range(n):
            target = t0 + at[i]
            while True:
                now = time.perf_counter()
                if now >= target:
                    break
                if target - now > 0.002:
                    time.sleep(target - now - 0.001)
            sv.submit(id_base + i, rules[i % len(rules)])
        t_sub = time.perf_counter() - t0
        done.set()
        th.join(timeout=600)
        t_end = time.perf_counter() - t0
        stats = sv.stats()
    lat = np.array(lat) if lat else np.zeros(1)
    ok = sum(1 for v in results.values() if v[1] == 0)
    return {
        "offered_rules_per_s": rate,
        "submitted": n,
        "completed_ok": ok,
        "sustained_rules_per_s": len(results) / t_end if t_end > 0 else 0.0,
        "achieved_arrival_rate": n / t_sub if t_sub > 0 else 0.0,
        "p50_ms": float(np.percentile(lat, 50)),
        "p99_ms": float(np.percentile(lat, 99)),
        "max_ms": float(lat.max()),
        "launches": stats["launches"],
        "device_ms": stats["device_ms"],
        "host_prepare_ms": stats["host_ms"],
    }, results


def sweep(lib, rules, rates, duration: float, seed: int = 0, **kw):
    out, allres = [], {}
    base = 0
    for k, r in enumerate(rates):
        summ, res = run_rate(lib, rules, r, duration, seed + k, id_base=base, **kw)
        out.append(summ)
        allres.update(res)
        base += summ["submitted"]
    return out, allres

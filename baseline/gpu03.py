#!/usr/bin/env python
"""Per-rule timing of the reference's own GPU library (GPU_03), built from its
sources by baseline/build_gpu03.sh, on a sample of a rule file.

Run as a separate process (bench.py --gpu03 does), so that the reference
library never shares a process with this repository's engine:

    python baseline/gpu03.py GRAPH.ttl RULES.txt [--stride 20] [--max-seconds 120]

Prints one JSON object: rules evaluated, wall time, the summed device times
the library reports (supportMs + confidenceMs), and the raw results (support,
headSize, headSupport, bodySize per rule).  GPU_03 differs from CPU_01 (and
this engine) on some rules: it reuses the head triple for support, turns
constants into free variables and skips the body size when support is 0, so
its results are reported, not checked.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import sys
import time
from pathlib import Path

HERE = Path(__file__).resolve().parent
LIB = HERE / "_ref" / "gpu03" / "libgpu_rules.so"


class GpuRuleResult(ctypes.Structure):
    # GPU_03/gpu_rules_api.h:21-30
    _fields_ = [("support", ctypes.c_int), ("headSize", ctypes.c_int), ("headSupport", ctypes.c_int),
                ("headCoverage", ctypes.c_double), ("bodySize", ctypes.c_int), ("confidence", ctypes.c_double),
                ("supportMs", ctypes.c_double), ("confidenceMs", ctypes.c_double)]


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("ttl")
    ap.add_argument("rules")
    ap.add_argument("--stride", type=int, default=20)
    ap.add_argument("--max-seconds", type=float, default=120.0)
    a = ap.parse_args()
    if not LIB.exists():
        print(json.dumps({"unavailable": f"{LIB.name} not built (baseline/build_gpu03.sh)"}))
        return 0
    lib = ctypes.CDLL(str(LIB))
    lib.gpu_load_graph.restype = ctypes.c_void_p
    lib.gpu_load_graph.argtypes = [ctypes.c_char_p]
    lib.gpu_evaluate_rule.restype = ctypes.c_int
    lib.gpu_evaluate_rule.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.POINTER(GpuRuleResult)]
    lib.gpu_free_graph.argtypes = [ctypes.c_void_p]
    rules = [r for r in Path(a.rules).read_text().splitlines() if r.strip()][::a.stride]
    t0 = time.perf_counter()
    ctx = lib.gpu_load_graph(a.ttl.encode())
    load_s = time.perf_counter() - t0
    if not ctx:
        print(json.dumps({"unavailable": "gpu_load_graph returned NULL"}))
        return 0
    res = GpuRuleResult()
    lib.gpu_evaluate_rule(ctx, rules[0].encode(), ctypes.byref(res))   # warm-up (lazy head caches)
    rows, dev_ms, n = [], 0.0, 0
    t0 = time.perf_counter()
    for r in rules:
        if lib.gpu_evaluate_rule(ctx, r.encode(), ctypes.byref(res)) != 0:
            rows.append(None)
        else:
            rows.append([res.support, res.headSize, res.headSupport, res.bodySize])
            dev_ms += res.supportMs + res.confidenceMs
        n += 1
        if time.perf_counter() - t0 > a.max_seconds:
            break
    wall = time.perf_counter() - t0
    lib.gpu_free_graph(ctx)
    print(json.dumps({"rules": n, "stride": a.stride, "wall_s": wall, "load_s": load_s,
                      "device_ms": dev_ms, "rules_per_s_wall": n / wall if wall > 0 else None,
                      "rules_per_s_device": n / (dev_ms / 1e3) if dev_ms > 0 else None,
                      "results": rows}))
    return 0


if __name__ == "__main__":
    sys.exit(main())

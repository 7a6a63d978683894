"""gpu_evaluate_rule_noalloc against gpu_evaluate_rule.

The no-allocation entry point exists for callers that may not call
cudaMalloc while they evaluate rules (a host framework with a fixed device
memory budget, a serving loop that cannot afford the device-wide
synchronisation cudaMalloc/cudaFree can cause).  It must give exactly the
results of the allocating entry point, also on the second of two calls in a
row, when the shared scratch array still holds the previous call's data.
This file sorts last so that a stop-at-first-failure run has already run the
other tests.
"""
import numpy as np
import pytest

import masterthesis_gpu_acceleration_b200 as eng
from conftest import load_fixture
from masterthesis_gpu_acceleration_b200 import synth

pytestmark = pytest.mark.gpu

FIELDS = ("support", "headSize", "headSupport", "bodySize", "headCoverage", "confidence")


def _same(a, b):
    return all(getattr(a, f) == getattr(b, f) for f in FIELDS)


def test_noalloc_matches_allocating_entry_point_fuzz(tmp_path):
    fx = load_fixture("fuzz_3.json")
    p = tmp_path / "graph.ttl"
    p.write_text(fx["ttl"])
    with eng.GpuRulesLib(p) as lib:
        for rule in fx["rules"]:
            want = lib.evaluate_rule(rule)
            first = lib.evaluate_rule_noalloc(rule)
            second = lib.evaluate_rule_noalloc(rule)
            assert _same(first, want) and _same(second, want), rule


def test_noalloc_matches_allocating_entry_point_c3(tmp_path):
    d = synth.generate("c3", tmp_path / "c3", seed=0)
    rules = synth.read_rules(d)[::50]
    with eng.GpuRulesLib(d / "graph.ttl") as lib:
        for rule in rules:
            want = lib.evaluate_rule(rule)
            got = [lib.evaluate_rule_noalloc(rule) for _ in range(2)]
            assert all(_same(g, want) for g in got), rule

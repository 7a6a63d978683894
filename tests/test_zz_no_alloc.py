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


def test_noalloc_global_bitmap_in_scratch_and_size_limit(tmp_path):
    """Rules whose pair bitmap cannot sit in shared memory (an hO domain of
    400,000 values) keep it in the scratch array: 100 head subjects need
    5 MB of rows, which fits the 8 MiB array; 200 need 10 MB, which the
    entry point refuses with -1 and the size in gpu_last_error().  Warm
    calls take no device memory."""
    from conftest import wide_domain_graph
    ttl, rules, exp = wide_domain_graph(tmp_path / "wide")
    with eng.GpuRulesLib(ttl) as lib:
        want = lib.evaluate_rule(rules[0])
        assert [want.support, want.headSize, want.headSupport, want.bodySize] == exp[0].tolist()
        got = [lib.evaluate_rule_noalloc(rules[0]) for _ in range(2)]
        assert all(_same(g, want) for g in got)
        before = eng.query_vram()[0]
        for _ in range(3):
            assert _same(lib.evaluate_rule_noalloc(rules[0]), want)
        assert eng.query_vram()[0] == before, "no-allocation calls changed free device memory"
        with pytest.raises(RuntimeError, match="scratch"):
            lib.evaluate_rule_noalloc(rules[1])
        # the array is still usable after a refusal
        assert _same(lib.evaluate_rule_noalloc(rules[0]), want)

"""Body-size deduplication modes, through the C ABI.

A body-size phase counts distinct (hS, hO) pairs.  Pairs go to bitmap rows
in shared memory when a task's rows fit there; otherwise to one global
bitmap row per head subject while all of a launch's rows fit the context's
dedup budget; beyond it either to rows per resident block (memory bounded by
the launch, not by the number of head subjects) or to 64-bit pair keys that
a radix sort on the device orders and counts once each (the reference's
Thrust sort + unique, GPU_03/gpu_rules_lib.cu:485-518).  Every mode must give
the reference's counts exactly: each is forced here on the reference-pinned
fixtures, and chosen automatically under a small budget on a graph whose hO
domain (400,000 values) does not fit shared memory.
"""
import numpy as np
import pytest

import masterthesis_gpu_acceleration_b200 as eng
from conftest import fuzz_names, load_fixture, wide_domain_graph
from masterthesis_gpu_acceleration_b200 import synth

pytestmark = pytest.mark.gpu

MODES = {"rows": 1, "block_rows": 2, "sort": 3}
COUNT_FIELDS = ("support", "headSize", "headSupport", "bodySize")


def _expected(fx):
    return np.array([[e[k] for k in COUNT_FIELDS] for e in fx["expected"]], dtype=np.int64)


def _batch_counts(lib, rules):
    b = lib.prepare_batch(rules)
    b.run()
    got = b.counts()
    modes, keys = b.dedup()
    b.close()
    return got, modes, keys


@pytest.fixture(scope="module")
def wide(tmp_path_factory):
    ttl, rules, exp = wide_domain_graph(tmp_path_factory.mktemp("wide"))
    return ttl, rules, exp


@pytest.mark.parametrize("mode", sorted(MODES))
@pytest.mark.parametrize("name", fuzz_names())
def test_forced_mode_fuzz(tmp_path, name, mode):
    fx = load_fixture(name)
    p = tmp_path / "graph.ttl"
    p.write_text(fx["ttl"])
    exp = np.array([[e[k] for k in COUNT_FIELDS] for e in fx["expected"]], dtype=np.int64)
    with eng.GpuRulesLib(p) as lib:
        lib.set_option("dedup_mode", MODES[mode])
        got, modes, _ = _batch_counts(lib, fx["rules"])
        bad = np.nonzero((got != exp).any(axis=1))[0]
        assert len(bad) == 0, f"{mode}: rules {bad[:5].tolist()} differ"
        assert set(modes[modes >= 0].tolist()) <= {MODES[mode]}
        for i in range(0, len(fx["rules"]), 7):   # the plain per-rule form too
            r = lib.evaluate_rule(fx["rules"][i])
            assert [r.support, r.headSize, r.headSupport, r.bodySize] == exp[i].tolist(), (mode, i)


@pytest.mark.parametrize("mode", sorted(MODES))
@pytest.mark.parametrize("cfg", ["c2s", "c4s"])
def test_forced_mode_synthetic(data_dir, cfg, mode):
    fx = load_fixture(f"synthetic_{cfg}.json")
    d = synth.generate(cfg, data_dir / cfg, seed=fx["seed"])
    exp = _expected(fx)
    with eng.GpuRulesLib(d / "graph.ttl") as lib:
        lib.set_option("dedup_mode", MODES[mode])
        got, modes, keys = _batch_counts(lib, fx["rules"])
        bad = np.nonzero((got != exp).any(axis=1))[0]
        assert len(bad) == 0, f"{cfg} {mode}: rules {bad[:5].tolist()}: {got[bad[:3]].tolist()} vs {exp[bad[:3]].tolist()}"
        assert (modes >= 0).any() and set(modes[modes >= 0].tolist()) == {MODES[mode]}
        if mode == "sort":
            assert keys > 0


def test_sort_keys_overflow_is_rerun_exactly(data_dir):
    """A small budget caps the first key buffer at 65,536 keys; c2s emits
    millions, so the first run overflows and is staged again with the exact
    count taken from the append cursor."""
    fx = load_fixture("synthetic_c2s.json")
    d = synth.generate("c2s", data_dir / "c2s", seed=fx["seed"])
    exp = _expected(fx)
    with eng.GpuRulesLib(d / "graph.ttl") as lib:
        lib.set_option("dedup_mode", MODES["sort"])
        lib.set_option("dedup_budget", 4096)
        got, modes, keys = _batch_counts(lib, fx["rules"])
        assert keys > 65536
        assert (got == exp).all()
        res, st, _ = lib.evaluate_rules_batch(fx["rules"])   # one-shot chunks rerun the same way
        assert [[r.support, r.headSize, r.headSupport, r.bodySize] for r in res] == exp.tolist()
        for i, rule in enumerate(fx["rules"]):
            r = lib.evaluate_rule(rule)
            assert [r.support, r.headSize, r.headSupport, r.bodySize] == exp[i].tolist(), i


def test_wide_domain_automatic_choice(wide):
    ttl, rules, exp = wide
    with eng.GpuRulesLib(ttl) as lib:
        got, modes, _ = _batch_counts(lib, rules)
        assert (got == exp).all()
        # default budget: every global row fits, one row per head subject
        assert modes[0] == 1 and modes[1] == 1 and modes[2] == 0
        lib.set_option("dedup_budget", 1 << 20)   # 1 MiB: rows of 5 and 10 MB no longer fit
        got, modes, _ = _batch_counts(lib, rules)
        assert (got == exp).all()
        assert modes[0] in (2, 3) and modes[1] in (2, 3) and modes[2] == 0
        for i, rule in enumerate(rules):
            r = lib.evaluate_rule(rule)
            assert [r.support, r.headSize, r.headSupport, r.bodySize] == exp[i].tolist(), i


@pytest.mark.parametrize("mode", sorted(MODES))
def test_wide_domain_forced(wide, mode):
    ttl, rules, exp = wide
    with eng.GpuRulesLib(ttl) as lib:
        lib.set_option("dedup_mode", MODES[mode])
        lib.set_option("dedup_budget", 1 << 20)
        got, modes, _ = _batch_counts(lib, rules)
        assert (got == exp).all(), (mode, got.tolist(), exp.tolist())
        assert modes.tolist() == [MODES[mode]] * 4
        parts = np.array([lib.evaluate_rule_shard(rules[1], k, 3) for k in range(3)])
        assert parts[:, 3].sum() == exp[1, 3] and parts[:, 0].sum() == exp[1, 0]


def test_bad_dedup_options_are_rejected(wide):
    ttl, _, _ = wide
    with eng.GpuRulesLib(ttl) as lib:
        for name, v in (("dedup_mode", 4), ("dedup_mode", -1), ("dedup_budget", 100)):
            with pytest.raises(ValueError):
                lib.set_option(name, v)

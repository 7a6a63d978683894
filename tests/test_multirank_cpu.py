"""Multi-rank host logic with two gloo processes on the CPU.

The engine needs a GPU, but everything the multi-GPU layout adds around it
runs on the host: each rank's data (same graph, own rule set), the slice of a
shared rule list, the max-over-ranks timing that the benchmark reports, the
gather of per-rank results back into rule order, and the int64 sum
all-reduce that joins the slices of one rule split over the ranks.  The
split rule goes through the library's own Python wrapper
(GpuRulesLib.evaluate_rule_shard), with only its C function
gpu_evaluate_rule_shard replaced by a CPU stand-in; the GPU test at the end
runs the same two-rank path on the real library.
"""
import ctypes
import hashlib
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

from conftest import ROOT
from masterthesis_gpu_acceleration_b200 import shard


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, data_dir, q):
    sys.path.insert(0, str(ROOT))
    import torch.distributed as dist
    from masterthesis_gpu_acceleration_b200 import shard, synth
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        d = synth.generate("c1", os.path.join(data_dir, f"r{rank}"), seed=0, rule_seed=shard.rule_seed(rank))
        triples = hashlib.sha256((d / "triples.bin").read_bytes()).hexdigest()
        rules = synth.read_rules(d)
        # a per-rank "timed span": the reported value uses the slowest rank
        span = 100.0 + 50.0 * rank
        mx = shard.max_over_ranks(span)
        # strong layout: slice a shared list and gather the slices back
        shared = [f"rule{i}" for i in range(11)]
        mine = shard.shard_rules(shared, rank, world)
        parts = [None] * world
        dist.all_gather_object(parts, [r.upper() for r in mine])
        back = shard.gather_results(parts, len(shared), world)
        # one rule split over the ranks: partial counts through the wrapper,
        # one int64 all-reduce
        whole = shard.evaluate_rule_split(_stub_wrapper().evaluate_rule_shard, "tiny")
        q.put((rank, triples, rules, mx, back, whole))
    finally:
        dist.destroy_process_group()


# A tiny graph and the rule (?a p ?v) ^ (?b p ?v) => (?a q ?b), counted by
# brute force: body pairs of a slice of head subjects, support of a slice of
# head triples.  Stands in for gpu_evaluate_rule_shard on the CPU.
_P = [(a, v) for a in range(12) for v in range(4) if (a * 7 + v * 3) % 5 < 2]
_Q = [(a, b) for a in range(12) for b in range(12) if (a + 2 * b) % 7 == 0]


def _grounded(a, b):
    return a != b and any(v not in (a, b) and (a, v) in _P and (b, v) in _P for v in range(4))


def _tiny_shard_eval(rule, k, n):
    subj = sorted({a for a, _ in _P})
    lo, hi = shard.shard_bounds(len(subj), k, n)
    mine = set(subj[lo:hi])
    body = sum(1 for a in mine for b in range(12) if _grounded(a, b))
    lo, hi = shard.shard_bounds(len(_Q), k, n)
    sup = sum(1 for a, b in _Q[lo:hi] if _grounded(a, b))
    return [sup, len(_Q), len(_Q), body]


class _StubLib:
    """Stands in for libgpu_rules.so: gpu_evaluate_rule_shard as a C
    function pointer with the library's signature, counting _tiny_shard_eval
    into the caller's int64 array."""

    def __init__(self):
        proto = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int, ctypes.c_int,
                                 ctypes.c_void_p)
        self.gpu_evaluate_rule_shard = proto(self._shard)
        self.calls = []

    def _shard(self, ctx, text, k, n, out):
        if not ctx or not out or not 0 <= k < n:
            return -1
        self.calls.append((text.decode(), k, n))
        (ctypes.c_longlong * 4).from_address(out)[:] = _tiny_shard_eval(text.decode(), k, n)
        return 0

    def gpu_last_error(self):
        return b""


def _stub_wrapper():
    import masterthesis_gpu_acceleration_b200 as eng
    lib = object.__new__(eng.GpuRulesLib)   # the wrapper without loading a graph
    lib._lib = _StubLib()
    lib._ctx = ctypes.c_void_p(1)
    return lib


def test_wrapper_marshals_shard_counts():
    lib = _stub_wrapper()
    got = lib.evaluate_rule_shard("tiny", 1, 3)
    assert got.dtype.name == "int64" and got.tolist() == _tiny_shard_eval("tiny", 1, 3)
    assert lib._lib.calls == [("tiny", 1, 3)]
    with pytest.raises(RuntimeError):
        lib.evaluate_rule_shard("tiny", 3, 3)
    lib._ctx = None   # keep __del__ from freeing the stand-in handle


def test_tiny_shard_eval_is_additive():
    whole = _tiny_shard_eval("tiny", 0, 1)
    assert whole[0] > 0 and whole[3] > 0
    for n in (2, 3, 5):
        parts = [_tiny_shard_eval("tiny", k, n) for k in range(n)]
        assert sum(p[0] for p in parts) == whole[0] and sum(p[3] for p in parts) == whole[3]


def test_two_ranks_gloo(tmp_path):
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, str(tmp_path), q)) for r in range(world)]
    for p in procs:
        p.start()
    out = {}
    for _ in range(world):
        rank, triples, rules, mx, back, whole = q.get(timeout=120)
        out[rank] = (triples, rules, mx, back, whole)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert out[0][0] == out[1][0], "ranks must share the graph"
    assert out[0][1] != out[1][1], "ranks must evaluate different rule sets"
    assert out[0][2] == out[1][2] == 150.0
    assert out[0][3] == out[1][3] == [f"RULE{i}" for i in range(11)]
    single = _tiny_shard_eval("tiny", 0, 1)
    for r in range(world):
        w = out[r][4]
        assert (w["support"], w["headSize"], w["bodySize"]) == (single[0], single[1], single[3])
        assert w["confidence"] == (single[0] / single[3] if single[3] else 0.0)
    assert shard.weak_value(10000, 2, 5, 150.0) == pytest.approx(2 * 10000 * 5 / 0.15)


def test_shard_bounds_cover_exactly():
    for n in (0, 1, 7, 10000):
        for world in (1, 2, 3, 8):
            covered = []
            for r in range(world):
                lo, hi = shard.shard_bounds(n, r, world)
                covered.extend(range(lo, hi))
            assert covered == list(range(n))
    with pytest.raises(ValueError):
        shard.shard_bounds(10, 2, 2)


def _gpu_worker(rank, world, port, data_dir, rules, q):
    sys.path.insert(0, str(ROOT))
    import torch.distributed as dist
    import masterthesis_gpu_acceleration_b200 as eng
    from masterthesis_gpu_acceleration_b200 import synth
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        d = synth.generate("c4s", data_dir, seed=0)
        with eng.GpuRulesLib(d / "graph.ttl") as lib:
            out = [shard.evaluate_rule_split(lib.evaluate_rule_shard, r) for r in rules]
        q.put((rank, out))
    finally:
        dist.destroy_process_group()


@pytest.mark.gpu
def test_two_ranks_split_rules_on_the_library(tmp_path):
    """Two processes (gloo on the host, the same GPU) each evaluate their
    slice of the c4s hub rules with gpu_evaluate_rule_shard; the int64
    all-reduce must give the reference's counts.  The ranks' kernels are
    independent (nothing on the device waits on the other rank)."""
    from masterthesis_gpu_acceleration_b200 import synth
    from conftest import load_fixture
    fx = load_fixture("synthetic_c4s.json")
    synth.generate("c4s", tmp_path / "c4s", seed=0)   # once, before the ranks read it
    idx = list(range(10)) + [42]
    rules = [fx["rules"][i] for i in idx]
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_gpu_worker, args=(r, world, port, str(tmp_path / "c4s"), rules, q))
             for r in range(world)]
    for p in procs:
        p.start()
    out = {}
    for _ in range(world):
        rank, res = q.get(timeout=600)
        out[rank] = res
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    for k, i in enumerate(idx):
        e = fx["expected"][i]
        for r in range(world):
            w = out[r][k]
            assert [w[f] for f in ("support", "headSize", "headSupport", "bodySize")] == \
                [e["support"], e["headSize"], e["headSupport"], e["bodySize"]], (i, r)

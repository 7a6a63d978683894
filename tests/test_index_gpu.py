"""The device-side index build (index_gpu.cu) against the host build.

gpu_load_graph builds the index on the device by default (radix sort of
packed (predicate, key, value) keys, rows, ranks, lookup table and row
signatures from prefix sums); GPU_RULES_INDEX_BUILD=host selects the host
build of index.cpp.  Both graphs are written with gpu_save_index and every
array is compared: all must be equal, except that colliding entries of the
lookup table may sit in other slots (the table is compared as a set of
entries; lookups are the same).
"""
import os
import struct

import numpy as np
import pytest

import masterthesis_gpu_acceleration_b200 as eng
from conftest import load_fixture, wide_domain_graph
from masterthesis_gpu_acceleration_b200 import synth

pytestmark = pytest.mark.gpu

# array order and element types of a graph file (index_io.cpp, each_array)
ARRAYS = [(f"{name}{d}", "i4") for d in (0, 1) for name in
          ("val", "valRank", "src", "srcRank", "rowKey", "rowBeg", "predRow", "predEdge")]
ARRAYS += [("hash", "hash"), ("hubOf0", "i4"), ("hubOf1", "i4"), ("hubOff", "i8"), ("hubBits", "u4"),
           ("valSig0", "u8"), ("valSig1", "u8"), ("sufSig0", "u8"), ("sufSig1", "u8")]


def read_graph_file(path):
    b = open(path, "rb").read()
    assert b[:8] == b"GRGRAPH1"
    _, _, n_pred, n_ent, n_tri, hash_mask, _ = struct.unpack_from("<IIiiqII", b, 8)
    pos = 40

    def skip_strings(count_pairs=1):
        nonlocal pos
        (cnt,) = struct.unpack_from("<Q", b, pos)
        pos += 8
        for _ in range(cnt * count_pairs):
            (ln,) = struct.unpack_from("<I", b, pos)
            pos += 4 + ln

    skip_strings()       # entities
    skip_strings()       # predicates
    skip_strings(2)      # rule prefixes
    out = {"n_pred": n_pred, "n_ent": n_ent, "n_triples": n_tri, "hash_mask": hash_mask}
    for name, kind in ARRAYS:
        (cnt,) = struct.unpack_from("<Q", b, pos)
        pos += 8
        width = 16 if kind == "hash" else int(kind[1])
        raw = np.frombuffer(b, dtype=np.uint8, count=cnt * width, offset=pos)
        pos += cnt * width
        out[name] = raw.view(np.uint32).reshape(-1, 4) if kind == "hash" else raw.view("<" + kind)
    return out


def both_builds(ttl, tmp_path):
    files = {}
    for how in ("host", "device"):
        old = os.environ.get("GPU_RULES_INDEX_BUILD")
        os.environ["GPU_RULES_INDEX_BUILD"] = how
        try:
            with eng.GpuRulesLib(ttl) as lib:
                f = tmp_path / f"{how}.grg"
                lib.save_index(f)
                files[how] = read_graph_file(f)
        finally:
            if old is None:
                del os.environ["GPU_RULES_INDEX_BUILD"]
            else:
                os.environ["GPU_RULES_INDEX_BUILD"] = old
    return files["host"], files["device"]


def assert_same_index(h, d):
    for k in ("n_pred", "n_ent", "n_triples", "hash_mask"):
        assert h[k] == d[k], k
    for name, kind in ARRAYS:
        if kind == "hash":
            def entries(t):
                used = t[t[:, 0] != 0xFFFFFFFF]
                return len(used), {tuple(r) for r in used.tolist()}
            (hn, he), (dn, de) = entries(h[name]), entries(d[name])
            assert hn == dn == len(he) and he == de, "lookup table entries differ"
        else:
            assert np.array_equal(h[name], d[name]), name


@pytest.mark.parametrize("name", ["fuzz_0.json", "fuzz_3.json", "edge_cases.json"])
def test_device_index_equals_host_small(tmp_path, name):
    fx = load_fixture(name)
    p = tmp_path / "graph.ttl"
    p.write_text(fx["ttl"])
    assert_same_index(*both_builds(p, tmp_path))


@pytest.mark.parametrize("cfg", ["c3", "c4s"])
def test_device_index_equals_host_synthetic(data_dir, tmp_path, cfg):
    d = synth.generate(cfg, data_dir / cfg, seed=0)
    assert_same_index(*both_builds(d / "graph.ttl", tmp_path))


def test_device_index_equals_host_wide(tmp_path):
    ttl, _, _ = wide_domain_graph(tmp_path / "wide")
    assert_same_index(*both_builds(ttl, tmp_path))

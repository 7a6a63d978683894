"""The graph load path on the CPU: the multi-threaded Turtle read and index
build (tests/native/load_check.cpp, compiled here with g++) agree with one
reader over the whole text, and the index answers every row and triple."""
import subprocess

import pytest

from conftest import ROOT, fuzz_names, load_fixture
from masterthesis_gpu_acceleration_b200 import synth

CSRC = ROOT / "masterthesis_gpu_acceleration_b200" / "csrc"


@pytest.fixture(scope="module")
def checker(tmp_path_factory):
    out = tmp_path_factory.mktemp("native") / "load_check"
    subprocess.run(["g++", "-O2", "-std=c++17", "-pthread", "-o", str(out),
                    str(ROOT / "tests" / "native" / "load_check.cpp"), str(CSRC / "turtle.cpp"),
                    str(CSRC / "index.cpp"), str(CSRC / "index_io.cpp")], check=True)
    return out


def _run(checker, path, min_chunk):
    scratch = str(path) + ".graph"
    r = subprocess.run([str(checker), str(path), str(min_chunk), scratch], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr


ADVERSARIAL = """@prefix ex: <http://ex/> .
# a comment line that ends with a dot.
ex:a ex:p ex:b ;
     ex:q "v1" ,
          "v2" .
ex:b ex:p ex:c . ex:c ex:p ex:a .
<http://ex/d> <http://ex/p> "12.5" .
ex:d ex:q "dot at the end." .
ex:e ex:p ex:f;
     ex:q ex:g.
ex:f ex:p ex:a .
"""


@pytest.mark.parametrize("min_chunk", [16, 64, 4096])
def test_parallel_read_matches_one_reader_fuzz(checker, tmp_path, min_chunk):
    for name in fuzz_names() + ["edge_cases.json"]:
        p = tmp_path / f"{name}.ttl"
        p.write_text(load_fixture(name)["ttl"])
        _run(checker, p, min_chunk)
    p = tmp_path / "adversarial.ttl"
    p.write_text(ADVERSARIAL * 50)
    _run(checker, p, min_chunk)


def test_prefix_after_first_chunk_falls_back(checker, tmp_path):
    p = tmp_path / "late_prefix.ttl"
    body = "".join(f"<http://e/{i}> <http://p/0> <http://e/{i + 1}> .\n" for i in range(400))
    p.write_text(body + "@prefix ex: <http://ex/> .\nex:x <http://p/0> ex:y .\n" + body)
    _run(checker, p, 256)


def test_parallel_read_and_index_synthetic(checker, data_dir):
    d = synth.generate("c2s", data_dir / "c2s_load", seed=3)
    _run(checker, d / "graph.ttl", 1 << 16)


def test_graph_file_reader_of_the_index_comparison(checker, tmp_path):
    """tests/test_index_gpu.py compares host- and device-built indexes by
    reading graph files; its reader is checked here on a file the native
    checker wrote from the host build."""
    from test_index_gpu import ARRAYS, read_graph_file
    p = tmp_path / "fuzz.ttl"
    p.write_text(load_fixture("fuzz_2.json")["ttl"])
    _run(checker, p, 64)
    g = read_graph_file(str(p) + ".graph")
    n = g["n_triples"]
    assert n > 0 and g["hash"].shape == (g["hash_mask"] + 1, 4)
    for d in (0, 1):
        for name in ("val", "valRank", "src", "srcRank", "valSig", "sufSig"):
            assert len(g[f"{name}{d}"]) == n, (name, d)
        assert g[f"rowBeg{d}"][-1] == n and g[f"predEdge{d}"][-1] == n
        assert len(g[f"predRow{d}"]) == len(g[f"predEdge{d}"]) == g["n_pred"] + 1
        assert len(g[f"rowKey{d}"]) + 1 == len(g[f"rowBeg{d}"]) == g[f"predRow{d}"][-1] + 1
    used = (g["hash"][:, 0] != 0xFFFFFFFF).sum()
    assert used == len(g["rowKey0"]) + len(g["rowKey1"])
    assert len(ARRAYS) == 25

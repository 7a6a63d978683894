"""The planner's shared-memory layout on CPU (tests/native/plan_check.cpp,
compiled here with g++): for every device phase of the fuzz, edge-case and
synthetic rule sets, planned for 128-, 256- and 512-thread blocks, the
frontier levels and the widest task's dedup bits fit the block's pool and
every index a plan holds stays inside its arrays."""
import subprocess

import pytest

from conftest import ROOT, fuzz_names, load_fixture
from masterthesis_gpu_acceleration_b200 import synth

CSRC = ROOT / "masterthesis_gpu_acceleration_b200" / "csrc"


@pytest.fixture(scope="module")
def checker(tmp_path_factory):
    out = tmp_path_factory.mktemp("native") / "plan_check"
    subprocess.run(["g++", "-O2", "-std=c++17", "-pthread", "-o", str(out),
                    str(ROOT / "tests" / "native" / "plan_check.cpp")] +
                   [str(CSRC / f) for f in ("turtle.cpp", "index.cpp", "rules.cpp", "planner.cpp", "tasks.cpp")],
                   check=True)
    return out


def _run(checker, ttl, rules):
    r = subprocess.run([str(checker), str(ttl), str(rules)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr


def test_plans_fit_fixtures(checker, tmp_path):
    for name in fuzz_names() + ["edge_cases.json"]:
        fx = load_fixture(name)
        ttl, rules = tmp_path / f"{name}.ttl", tmp_path / f"{name}.txt"
        ttl.write_text(fx["ttl"])
        texts = fx["rules"] if "rules" in fx else [c["rule"] for c in fx["cases"]]
        rules.write_text("\n".join(texts) + "\n")
        _run(checker, ttl, rules)


@pytest.mark.parametrize("cfg", ["c3", "c4s"])
def test_plans_fit_synthetic(checker, data_dir, cfg):
    d = synth.generate(cfg, data_dir / f"{cfg}_plans", seed=0)
    _run(checker, d / "graph.ttl", d / "rules.txt")

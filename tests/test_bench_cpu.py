"""The reference arm of bench.py on CPU: `--impl reference` times the
reference's own CPU_01 code (oracle/_ref) and prints one JSON line with the
contract's keys.  Uses the small c1 configuration so that it takes seconds."""
import json
import subprocess
import sys

import pytest

import oracle
from conftest import ROOT


@pytest.mark.skipif(not oracle.ref_available(), reason="oracle/_ref not built")
def test_reference_arm_prints_contract_line(tmp_path):
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--config", "c1",
                        "--steps", "1", "--warmup", "1", "--data", str(tmp_path)],
                       capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["unit"] == "rules/s" and line["value"] > 0
    for k in ("metric", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "config"):
        assert k in line, k
    cb = line["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] >= 1 and cb["value"] == line["value"] and cb["sample"]
    assert cb["host"]["logical_cores"] >= cb["cores"]
    assert line["e2e"] == {"value": line["value"], "unit": "rules/s", "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}


@pytest.mark.skipif(not oracle.ref_available(), reason="oracle/_ref not built")
def test_engine_arm_cpu_baseline_helper(tmp_path):
    """The engine arm's cpu_baseline (timed by the reference's CPU code on a
    bounded sample) runs without a GPU and states the host."""
    sys.path.insert(0, str(ROOT))
    import bench
    from masterthesis_gpu_acceleration_b200 import synth
    d = synth.generate("c1", tmp_path / "c1", seed=0)
    cb = bench.cpu_baseline(d, synth.read_rules(d), "c1")
    assert cb["kind"] == "reference" and cb["value"] > 0 and cb["cores"] == 1
    assert cb["host"]["logical_cores"] >= 1 and "model" in cb["host"]

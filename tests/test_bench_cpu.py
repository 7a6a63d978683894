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
    assert line["e2e"] == {"value": line["value"], "unit": "rules/s", "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}

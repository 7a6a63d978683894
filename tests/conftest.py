import json
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = Path(__file__).resolve().parent / "golden"
sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def load_fixture(name: str) -> dict:
    return json.loads((GOLDEN / name).read_text())


def fuzz_names():
    return sorted(p.name for p in GOLDEN.glob("fuzz_*.json"))


def terms_to_ir(rule_terms, ) -> np.ndarray:
    """Rule IR (oracle input) from the fixture's term lists; variables get
    ids in first-seen order (body atoms, then the head), as the reference's
    parser assigns them; unknown constants keep their distinct negative ids."""
    out = []
    for atoms in rule_terms:
        body, head = atoms[:-1], atoms[-1]
        ids = {}

        def term(t):
            kind, v = t
            if kind == "v":
                if v not in ids:
                    ids[v] = len(ids)
                return [0, ids[v]]
            return [1, v]

        enc_body = []
        for p, s, o in body:
            enc_body.append([p] + term(s) + term(o))
        hp, hs, ho = head
        enc_head = [hp] + term(hs) + term(ho)
        out.append(len(body))
        out.extend(enc_head)
        for a in enc_body:
            out.extend(a)
    return np.array(out, dtype=np.int32)


@pytest.fixture(scope="session")
def data_dir(tmp_path_factory):
    return tmp_path_factory.mktemp("kg")

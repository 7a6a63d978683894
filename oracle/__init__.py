"""CPU oracle for the rule-counting hot path — TEST INFRASTRUCTURE ONLY.

Only the tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` use this package, and only as the checker.  The engine
(libgpu_rules.so) never calls it.

* ``liborules.so`` (rules_oracle.c): a plain-C restatement of the reference's
  CPU_01_nonparallel counting semantics, evaluated on integer triples and the
  rule IR written by the generator.
* ``_ref/cpu01_harness``: the reference's own CPU_01_nonparallel sources,
  compiled where they lie by build_ref.sh, run on the Turtle graph and rule
  text (used to pin the restatement and as the timed reference baseline).
"""
from __future__ import annotations

import ctypes
import json
import subprocess
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "lib" / "liborules.so"
REF_BIN = HERE / "_ref" / "cpu01_harness"

_lib = None


def build() -> None:
    """Builds liborules.so (and the reference harness where the sources exist)."""
    subprocess.run(["bash", str(HERE / "build_ref.sh")], check=True)


def _load():
    global _lib
    if _lib is None:
        if not LIB.exists() or LIB.stat().st_mtime < (HERE / "rules_oracle.c").stat().st_mtime:
            build()
        lib = ctypes.CDLL(str(LIB))
        lib.oracle_graph_build.restype = ctypes.c_void_p
        lib.oracle_graph_build.argtypes = [ctypes.c_void_p, ctypes.c_longlong, ctypes.c_int]
        lib.oracle_graph_free.restype = None
        lib.oracle_graph_free.argtypes = [ctypes.c_void_p]
        lib.oracle_eval_rules.restype = ctypes.c_int
        lib.oracle_eval_rules.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_longlong, ctypes.c_int,
                                          ctypes.c_void_p, ctypes.c_void_p]
        _lib = lib
    return _lib


class OracleGraph:
    def __init__(self, triples: np.ndarray, n_pred: int):
        self._t = np.ascontiguousarray(triples, dtype=np.int32)
        self.n_pred = int(n_pred)
        self._g = _load().oracle_graph_build(self._t.ctypes.data, len(self._t), self.n_pred)

    def evaluate_ir(self, ir: np.ndarray, n_rules: int):
        """Returns (counts[n,4] = support, headSize, headSupport, bodySize; status[n])."""
        ir = np.ascontiguousarray(ir, dtype=np.int32)
        out = np.zeros((n_rules, 4), dtype=np.int64)
        st = np.zeros(n_rules, dtype=np.int32)
        rc = _load().oracle_eval_rules(self._g, ir.ctypes.data, len(ir), n_rules, out.ctypes.data, st.ctypes.data)
        if rc != 0:
            raise ValueError("malformed rule IR")
        return out, st

    def close(self):
        if self._g:
            _load().oracle_graph_free(self._g)
            self._g = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def split_ir(ir: np.ndarray) -> list[np.ndarray]:
    """Splits an IR stream into one array per rule."""
    out, pos = [], 0
    while pos < len(ir):
        nb = int(ir[pos])
        n = 6 + 5 * nb
        out.append(ir[pos:pos + n])
        pos += n
    return out


def measures(counts: np.ndarray) -> list[dict]:
    """Result fields as FinalRule::setMeasures / setConfidence derive them
    (CPU_01_nonparallel/FinalRule.cpp:19-41)."""
    res = []
    for sup, hsz, hsup, body in counts.tolist():
        res.append({
            "support": sup, "headSize": hsz, "headSupport": hsup, "bodySize": body,
            "headCoverage": sup / hsz if hsz > 0 else 0.0,
            "confidence": sup / body if body > 0 else 0.0,
        })
    return res


def ref_available() -> bool:
    return REF_BIN.exists()


def run_reference(ttl: Path | str, rules: Path | str, threads: int = 1, first: int = -1,
                  repeat: int = 1, quiet: bool = False, timeout: float | None = None):
    """Runs the compiled reference (CPU_01_nonparallel) on a graph and rule file.

    Returns (per-rule dicts, summary dict)."""
    cmd = [str(REF_BIN), str(ttl), str(rules), "--threads", str(threads), "--repeat", str(repeat)]
    if first >= 0:
        cmd += ["--first", str(first)]
    if quiet:
        cmd.append("--quiet")
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout)
    if r.returncode != 0:
        raise RuntimeError(f"reference harness failed: {r.stderr}")
    rows, summary = [], {}
    for line in r.stdout.splitlines():
        d = json.loads(line)
        if d.get("summary"):
            summary = d
        else:
            rows.append(d)
    return rows, summary


def time_oracle(graph: OracleGraph, ir: np.ndarray, n_rules: int) -> float:
    t0 = time.perf_counter()
    graph.evaluate_ir(ir, n_rules)
    return time.perf_counter() - t0

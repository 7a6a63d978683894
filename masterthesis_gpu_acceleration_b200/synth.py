"""Seeded synthetic knowledge graphs and rule sets (libkg_synth.so).

Configurations (sizes of the reference's benchmark shapes):

    c1   10,000 entities, 20 predicates, 100,000 uniform triples; 10 chain
         rules with 1-2 body atoms
    c2   2,000 entities, 10 predicates, 100,000 uniform triples; 10 chain
         rules with 2-3 body atoms
    c2s  as c2 with Zipf(1.3) subjects
    c3   DBpedia-shaped: 100,000 entities, 600 predicates (Zipf(1.1) sizes),
         206,000 triples, Zipf(1.5) subjects / Zipf(1.3) objects; 10,000
         chain rules with 1-4 body atoms (weights .2/.4/.3/.1), predicates
         drawn by frequency
    c4   biomedical-shaped: 300,000 entities, 50 predicates, 6.8M triples,
         Zipf(1.2) objects, two 50,000-in-degree hubs on each of 5 hub
         predicates; 50 chain rules with 2-5 body atoms, 10 through hubs
         (5 of them cross a hub from both sides, (?x p ?v) ^ (?y p ?v))
    c4s  c4 at a tenth of the size (30,000 entities, 680,000 triples,
         5,000-in-degree hubs), small enough for the CPU oracle
"""
from __future__ import annotations

import ctypes
from pathlib import Path

import numpy as np

from .build import build_synth

_lib = None


def _load():
    global _lib
    if _lib is None:
        so = build_synth()
        _lib = ctypes.CDLL(str(so))
        _lib.kg_synth_write.restype = ctypes.c_longlong
        _lib.kg_synth_write.argtypes = [ctypes.c_char_p, ctypes.c_ulonglong, ctypes.c_int, ctypes.c_char_p]
        _lib.kg_synth_write2.restype = ctypes.c_longlong
        _lib.kg_synth_write2.argtypes = [ctypes.c_char_p, ctypes.c_ulonglong, ctypes.c_ulonglong, ctypes.c_int,
                                         ctypes.c_char_p]
        _lib.kg_synth_rule_stream.restype = ctypes.c_int
        _lib.kg_synth_rule_stream.argtypes = [ctypes.POINTER(ctypes.c_longlong), ctypes.c_int, ctypes.c_int,
                                              ctypes.c_double, ctypes.c_int, ctypes.c_ulonglong, ctypes.c_char_p]
    return _lib


GEN_VERSION = "2"   # kGenVersion of kg_synth.cpp


def generate(cfg: str, out_dir: Path | str, seed: int = 0, n_rules: int = -1, rule_seed: int | None = None) -> Path:
    """Writes graph.ttl, triples.bin, rules.txt, rules.ir and meta.txt (cached).

    rule_seed=None continues the graph's random stream (the configuration's
    standard rule set); an integer draws the rules from their own stream."""
    out = Path(out_dir)
    out.mkdir(parents=True, exist_ok=True)
    meta = out / "meta.txt"
    want = f"config={cfg}\nseed={seed}\n"
    if meta.exists() and meta.read_text().startswith(want) and (out / "graph.ttl").exists():
        m = read_meta(out)
        if (n_rules < 0 or m.get("rules") == str(n_rules)) and m.get("rule_seed") == (
                None if rule_seed is None else str(rule_seed)) and m.get("gen") == GEN_VERSION:
            return out
    rs = (1 << 64) - 1 if rule_seed is None else int(rule_seed)
    n = _load().kg_synth_write2(cfg.encode(), seed, rs, n_rules, str(out).encode())
    if n < 0:
        raise RuntimeError(f"generator failed for {cfg}")
    return out


def rule_stream(pred_counts, n: int, out_dir: Path | str, p: float = 0.4, max_len: int = 8, seed: int = 0) -> Path:
    """Serving requests: chain rules with geometric(p) length in 1..max_len."""
    out = Path(out_dir)
    out.mkdir(parents=True, exist_ok=True)
    pc = np.ascontiguousarray(pred_counts, dtype=np.int64)
    arr = pc.ctypes.data_as(ctypes.POINTER(ctypes.c_longlong))
    if _load().kg_synth_rule_stream(arr, len(pc), n, p, max_len, seed, str(out).encode()) != n:
        raise RuntimeError("rule stream generation failed")
    return out


def read_meta(d: Path | str) -> dict:
    return dict(line.split("=", 1) for line in Path(d, "meta.txt").read_text().split())


def read_triples(d: Path | str) -> np.ndarray:
    return np.fromfile(Path(d) / "triples.bin", dtype=np.int32).reshape(-1, 3)


def read_rules(d: Path | str) -> list[str]:
    return [l for l in Path(d, "rules.txt").read_text().splitlines() if l.strip()]


def read_rule_ir(d: Path | str) -> np.ndarray:
    return np.fromfile(Path(d) / "rules.ir", dtype=np.int32)


def pred_counts(triples: np.ndarray, n_pred: int) -> np.ndarray:
    return np.bincount(triples[:, 1], minlength=n_pred).astype(np.int64)

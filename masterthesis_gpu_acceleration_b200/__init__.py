"""B200 rule-evaluation engine: Python host binding of libgpu_rules.so.

This mirrors the reference's JVM binding (GPU_03/GpuRulesLib.scala:23-116):
``GpuRuleResult`` has the same fields in the same order, and ``GpuRulesLib``
checks device memory, loads the graph once, evaluates rules one by one and
frees the graph on ``close()``.  ``evaluate_rules_batch`` is the additive
batched entry point (one persistent device launch for many rules).

Everything below calls the compiled library; there is no Python or CPU
evaluation path.  Importing works without a GPU; loading a graph needs one.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path
from typing import Sequence

PKG_DIR = Path(__file__).resolve().parent
LIB_DIR = PKG_DIR / "lib"
LIB_PATH = LIB_DIR / "libgpu_rules.so"

#: symbols declared in include/gpu_rules_api.h
API_SYMBOLS = (
    "gpu_load_graph",
    "gpu_evaluate_rule",
    "gpu_evaluate_rule_json",
    "gpu_free_graph",
    "gpu_query_vram",
    "gpu_evaluate_rules_batch",
    "gpu_batch_prepare",
    "gpu_batch_run",
    "gpu_batch_info",
    "gpu_batch_kernels",
    "gpu_batch_count_bytes",
    "gpu_batch_free",
    "gpu_evaluate_rule_noalloc",
    "gpu_batch_profile",
    "gpu_batch_autotune",
    "gpu_set_option",
    "gpu_serve_start",
    "gpu_serve_submit",
    "gpu_serve_poll",
    "gpu_serve_stats",
    "gpu_serve_stop",
    "gpu_graph_stats",
    "gpu_graph_predicate",
    "gpu_save_index",
    "gpu_load_index",
    "gpu_batch_counts",
    "gpu_evaluate_rule_shard",
    "gpu_batch_dedup",
    "gpu_last_error",
)


class GpuRuleResult(ctypes.Structure):
    """Same layout as GpuRuleResult in include/gpu_rules_api.h (56 bytes)."""

    _fields_ = [
        ("support", ctypes.c_int),
        ("headSize", ctypes.c_int),
        ("headSupport", ctypes.c_int),
        ("headCoverage", ctypes.c_double),
        ("bodySize", ctypes.c_int),
        ("confidence", ctypes.c_double),
        ("supportMs", ctypes.c_double),
        ("confidenceMs", ctypes.c_double),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}

    def __repr__(self) -> str:  # mirrors GpuRulesLib.scala:39-42
        return (f"support={self.support}, headSize={self.headSize}, headCoverage={self.headCoverage}, "
                f"bodySize={self.bodySize}, confidence={self.confidence}, "
                f"supportMs={self.supportMs} ms, confidenceMs={self.confidenceMs} ms")


class GpuServeResult(ctypes.Structure):
    """Same layout as GpuServeResult in include/gpu_rules_api.h."""

    _fields_ = [
        ("requestId", ctypes.c_longlong),
        ("status", ctypes.c_int),
        ("result", GpuRuleResult),
        ("latencyMs", ctypes.c_double),
    ]


_lib = None


def _c_strings(texts: Sequence[str]):
    """A char*[] over texts: one encoded buffer of NUL-terminated strings and
    its pointer array, built without a Python object per string.  Returns
    (what must stay alive during the call, the pointer array)."""
    import numpy as np
    n = len(texts)
    if n == 0:
        return None, (ctypes.c_char_p * 1)()
    joined = "\0".join(texts) + "\0"
    buf = joined.encode()
    lens = np.fromiter(map(len, texts), dtype=np.int64, count=n)
    if joined.count("\0") != n:
        ends = None
    elif len(buf) == len(joined):   # one byte per character: string ends follow from the lengths
        ends = np.cumsum(lens + 1) - 1
    else:
        ends = np.flatnonzero(np.frombuffer(buf, dtype=np.uint8) == 0)
        if len(ends) != n:
            ends = None
    if ends is None:   # a text holds a NUL: one object per string
        arr = (ctypes.c_char_p * n)(*[t.encode() for t in texts])
        return arr, arr
    cbuf = ctypes.create_string_buffer(buf, len(buf))
    ptrs = np.empty(n, dtype=np.uint64)
    ptrs[0] = 0
    ptrs[1:] = (ends[:-1] + 1).astype(np.uint64)
    ptrs += np.uint64(ctypes.addressof(cbuf))
    return (cbuf, ptrs), ptrs.ctypes.data_as(ctypes.POINTER(ctypes.c_char_p))


def load_library(path: os.PathLike | str | None = None) -> ctypes.CDLL:
    """Loads libgpu_rules.so (built in-tree); raises if it is missing."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path is not None else LIB_PATH
    if not p.exists():
        raise RuntimeError(f"{p} is missing: build it with `python -m masterthesis_gpu_acceleration_b200.build`")
    lib = ctypes.CDLL(str(p))
    lib.gpu_load_graph.restype = ctypes.c_void_p
    lib.gpu_load_graph.argtypes = [ctypes.c_char_p]
    lib.gpu_evaluate_rule.restype = ctypes.c_int
    lib.gpu_evaluate_rule.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.POINTER(GpuRuleResult)]
    lib.gpu_evaluate_rule_json.restype = ctypes.c_int
    lib.gpu_evaluate_rule_json.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.POINTER(GpuRuleResult)]
    lib.gpu_free_graph.restype = None
    lib.gpu_free_graph.argtypes = [ctypes.c_void_p]
    lib.gpu_query_vram.restype = ctypes.c_int
    lib.gpu_query_vram.argtypes = [ctypes.POINTER(ctypes.c_size_t), ctypes.POINTER(ctypes.c_size_t)]
    lib.gpu_evaluate_rules_batch.restype = ctypes.c_int
    lib.gpu_evaluate_rules_batch.argtypes = [
        ctypes.c_void_p, ctypes.POINTER(ctypes.c_char_p), ctypes.c_int, ctypes.c_int,
        ctypes.POINTER(GpuRuleResult), ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double)]
    lib.gpu_batch_prepare.restype = ctypes.c_void_p
    lib.gpu_batch_prepare.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_char_p), ctypes.c_int, ctypes.c_int]
    lib.gpu_batch_run.restype = ctypes.c_int
    lib.gpu_batch_run.argtypes = [ctypes.c_void_p, ctypes.c_longlong, ctypes.POINTER(GpuRuleResult),
                                  ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double)]
    lib.gpu_batch_info.restype = ctypes.c_int
    lib.gpu_batch_info.argtypes = [ctypes.c_void_p] + [ctypes.POINTER(ctypes.c_longlong)] * 4
    lib.gpu_batch_kernels.restype = ctypes.c_int
    lib.gpu_batch_kernels.argtypes = [ctypes.c_void_p]
    lib.gpu_batch_count_bytes.restype = ctypes.c_int
    lib.gpu_batch_count_bytes.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_ulonglong)]
    lib.gpu_batch_free.restype = None
    lib.gpu_batch_free.argtypes = [ctypes.c_void_p]
    lib.gpu_evaluate_rule_noalloc.restype = ctypes.c_int
    lib.gpu_evaluate_rule_noalloc.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.POINTER(GpuRuleResult)]
    lib.gpu_batch_profile.restype = ctypes.c_int
    lib.gpu_batch_profile.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_ulonglong), ctypes.c_void_p,
                                      ctypes.c_void_p, ctypes.c_longlong]
    lib.gpu_batch_counts.restype = ctypes.c_int
    lib.gpu_batch_counts.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    lib.gpu_batch_dedup.restype = ctypes.c_int
    lib.gpu_batch_dedup.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(ctypes.c_longlong)]
    lib.gpu_evaluate_rule_shard.restype = ctypes.c_int
    lib.gpu_evaluate_rule_shard.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int, ctypes.c_int,
                                            ctypes.c_void_p]
    lib.gpu_batch_autotune.restype = ctypes.c_int
    lib.gpu_batch_autotune.argtypes = [ctypes.c_void_p, ctypes.c_int]
    lib.gpu_set_option.restype = ctypes.c_int
    lib.gpu_set_option.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_longlong]
    lib.gpu_serve_start.restype = ctypes.c_void_p
    lib.gpu_serve_start.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_longlong]
    lib.gpu_serve_submit.restype = ctypes.c_int
    lib.gpu_serve_submit.argtypes = [ctypes.c_void_p, ctypes.c_longlong, ctypes.c_char_p]
    lib.gpu_serve_poll.restype = ctypes.c_int
    lib.gpu_serve_poll.argtypes = [ctypes.c_void_p, ctypes.POINTER(GpuServeResult), ctypes.c_int, ctypes.c_int]
    lib.gpu_serve_stats.restype = ctypes.c_int
    lib.gpu_serve_stats.argtypes = [ctypes.c_void_p] + [ctypes.POINTER(ctypes.c_longlong)] * 4 + \
        [ctypes.POINTER(ctypes.c_double)] * 2
    lib.gpu_serve_stop.restype = None
    lib.gpu_serve_stop.argtypes = [ctypes.c_void_p]
    lib.gpu_graph_predicate.restype = ctypes.c_int
    lib.gpu_graph_predicate.argtypes = [ctypes.c_void_p, ctypes.c_longlong, ctypes.c_char_p, ctypes.c_int,
                                        ctypes.POINTER(ctypes.c_longlong)]
    lib.gpu_save_index.restype = ctypes.c_int
    lib.gpu_save_index.argtypes = [ctypes.c_void_p, ctypes.c_char_p]
    lib.gpu_load_index.restype = ctypes.c_void_p
    lib.gpu_load_index.argtypes = [ctypes.c_char_p]
    lib.gpu_graph_stats.restype = ctypes.c_int
    lib.gpu_graph_stats.argtypes = [ctypes.c_void_p] + [ctypes.POINTER(ctypes.c_longlong)] * 3
    lib.gpu_last_error.restype = ctypes.c_char_p
    lib.gpu_last_error.argtypes = []
    if path is None:
        _lib = lib
    return lib


def query_vram() -> tuple[int, int]:
    """(free, total) bytes of the current device; raises without a device."""
    lib = load_library()
    free, total = ctypes.c_size_t(), ctypes.c_size_t()
    if lib.gpu_query_vram(ctypes.byref(free), ctypes.byref(total)) != 0:
        raise RuntimeError("gpu_query_vram failed — no CUDA device?")
    return free.value, total.value


class GpuRulesLib:
    """Graph resident on the GPU between calls (GPU_03/GpuRulesLib.scala:61-116)."""

    def __init__(self, ttl_path: os.PathLike | str | None = None, index_path: os.PathLike | str | None = None):
        """Loads a Turtle file, or (index_path) a graph file written by
        save_index, which skips parsing and indexing."""
        if (ttl_path is None) == (index_path is None):
            raise ValueError("give exactly one of ttl_path and index_path")
        self._lib = load_library()
        query_vram()
        if index_path is not None:
            ctx = self._lib.gpu_load_index(str(index_path).encode())
            what, src = "gpu_load_index", index_path
        else:
            ctx = self._lib.gpu_load_graph(str(ttl_path).encode())
            what, src = "gpu_load_graph", ttl_path
        if not ctx:
            err = self._lib.gpu_last_error().decode(errors="replace")
            raise RuntimeError(f"{what} failed for: {src} ({err})")
        self._ctx = ctypes.c_void_p(ctx)

    # -- reference entry points -------------------------------------------------
    def evaluate_rule(self, rule_text: str) -> GpuRuleResult:
        res = GpuRuleResult()
        rc = self._lib.gpu_evaluate_rule(self._handle(), rule_text.encode(), ctypes.byref(res))
        if rc != 0:
            raise RuntimeError(f"gpu_evaluate_rule error code {rc} for: {rule_text} "
                               f"({self._lib.gpu_last_error().decode(errors='replace')})")
        return res

    def evaluate_rule_json(self, rule_json: str) -> GpuRuleResult:
        res = GpuRuleResult()
        rc = self._lib.gpu_evaluate_rule_json(self._handle(), rule_json.encode(), ctypes.byref(res))
        if rc != 0:
            raise RuntimeError(f"gpu_evaluate_rule_json error code {rc}")
        return res

    # -- additive entry points ---------------------------------------------------
    def evaluate_rules_batch(self, rules: Sequence[str], is_json: bool = False):
        """Returns (results, statuses, device_ms) for all rules in one launch.

        results is a ctypes array of n GpuRuleResult (indexable, iterable,
        sliceable), statuses a list of n ints."""
        n = len(rules)
        keep, arr = _c_strings(rules)
        out = (GpuRuleResult * max(n, 1))()
        st = (ctypes.c_int * max(n, 1))()
        ms = ctypes.c_double()
        rc = self._lib.gpu_evaluate_rules_batch(self._handle(), arr, n, int(is_json), out, st, ctypes.byref(ms))
        del keep
        if rc != 0:
            raise RuntimeError(f"gpu_evaluate_rules_batch failed "
                               f"({self._lib.gpu_last_error().decode(errors='replace')})")
        return (out if n else []), st[:n], ms.value

    def evaluate_rule_noalloc(self, rule_text: str) -> GpuRuleResult:
        """gpu_evaluate_rule without any device allocation (fixed in-library
        scratch; for callers that may not call cudaMalloc per request)."""
        res = GpuRuleResult()
        rc = self._lib.gpu_evaluate_rule_noalloc(self._handle(), rule_text.encode(), ctypes.byref(res))
        if rc != 0:
            raise RuntimeError(f"gpu_evaluate_rule_noalloc error code {rc} for: {rule_text} "
                               f"({self._lib.gpu_last_error().decode(errors='replace')})")
        return res

    def evaluate_rule_shard(self, rule_text: str, shard: int, n_shards: int):
        """Slice `shard` of `n_shards` of one rule (gpu_evaluate_rule_shard):
        int64 array [support part, headSize, headSupport, bodySize part]."""
        import numpy as np
        out = np.zeros(4, dtype=np.int64)
        rc = self._lib.gpu_evaluate_rule_shard(self._handle(), rule_text.encode(), int(shard), int(n_shards),
                                               out.ctypes.data)
        if rc != 0:
            raise RuntimeError(f"gpu_evaluate_rule_shard failed for: {rule_text} "
                               f"({self._lib.gpu_last_error().decode(errors='replace')})")
        return out

    def prepare_batch(self, rules: Sequence[str], is_json: bool = False) -> "PreparedBatch":
        return PreparedBatch(self, rules, is_json)

    def serve(self, slots: int = 3, max_batch: int = 4096, mem_budget: int = 1 << 30) -> "GpuServer":
        return GpuServer(self, slots, max_batch, mem_budget)

    def set_option(self, name: str, value: int) -> None:
        if self._lib.gpu_set_option(self._handle(), name.encode(), int(value)) != 0:
            raise ValueError(f"bad option {name}={value}")

    def save_index(self, path: os.PathLike | str) -> None:
        """Writes the loaded graph to one binary file (load it with
        GpuRulesLib(index_path=...))."""
        if self._lib.gpu_save_index(self._handle(), str(path).encode()) != 0:
            raise RuntimeError(f"gpu_save_index failed: {self._lib.gpu_last_error().decode(errors='replace')}")

    def stats(self) -> dict:
        e, p, t = ctypes.c_longlong(), ctypes.c_longlong(), ctypes.c_longlong()
        self._lib.gpu_graph_stats(self._handle(), ctypes.byref(e), ctypes.byref(p), ctypes.byref(t))
        return {"entities": e.value, "predicates": p.value, "triples": t.value}

    def predicates(self) -> list[tuple[str, int]]:
        """(IRI, distinct triples) of every predicate of the graph, by id."""
        out = []
        n = self.stats()["predicates"]
        buf = ctypes.create_string_buffer(4096)
        t = ctypes.c_longlong()
        for i in range(n):
            k = self._lib.gpu_graph_predicate(self._handle(), i, None, 0, None)
            if k >= len(buf):
                buf = ctypes.create_string_buffer(k + 1)
            self._lib.gpu_graph_predicate(self._handle(), i, buf, len(buf), ctypes.byref(t))
            out.append((buf.value.decode(errors="replace"), t.value))
        return out

    def close(self) -> None:
        if getattr(self, "_ctx", None) is not None and self._ctx.value:
            self._lib.gpu_free_graph(self._ctx)
            self._ctx = None

    def _handle(self):
        if self._ctx is None:
            raise RuntimeError("graph already freed")
        return self._ctx

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class PreparedBatch:
    """Rules parsed, planned and uploaded once; each run() is one CUDA-graph
    launch of the persistent kernel over all of them."""

    def __init__(self, lib: GpuRulesLib, rules: Sequence[str], is_json: bool = False):
        self._owner = lib
        self._lib = lib._lib
        self.n = len(rules)
        arr = (ctypes.c_char_p * max(self.n, 1))(*[r.encode() for r in rules])
        h = self._lib.gpu_batch_prepare(lib._handle(), arr, self.n, int(is_json))
        if not h:
            raise RuntimeError(f"gpu_batch_prepare failed ({self._lib.gpu_last_error().decode(errors='replace')})")
        self._h = ctypes.c_void_p(h)
        self._out = (GpuRuleResult * max(self.n, 1))()
        self._st = (ctypes.c_int * max(self.n, 1))()

    def run(self, flush_bytes: int = 0, fetch: bool = True):
        """Returns (results or None, statuses or None, device_ms)."""
        ms = ctypes.c_double()
        out = self._out if fetch else None
        st = self._st if fetch else None
        if self._lib.gpu_batch_run(self._h, flush_bytes, out, st, ctypes.byref(ms)) != 0:
            raise RuntimeError(f"gpu_batch_run failed ({self._lib.gpu_last_error().decode(errors='replace')})")
        if not fetch:
            return None, None, ms.value
        return list(self._out)[:self.n], list(self._st)[:self.n], ms.value

    def counts(self):
        """The last run's counts in 64 bits: int64 array [n, 4] of support,
        headSize, headSupport, bodySize (gpu_batch_counts)."""
        import numpy as np
        out = np.zeros((max(self.n, 1), 4), dtype=np.int64)
        if self._lib.gpu_batch_counts(self._h, out.ctypes.data, None) != 0:
            raise RuntimeError("gpu_batch_counts failed")
        return out[:self.n]

    def info(self) -> dict:
        v = [ctypes.c_longlong() for _ in range(4)]
        self._lib.gpu_batch_info(self._h, *[ctypes.byref(x) for x in v])
        d = dict(zip(("plans", "tasks", "h2d_bytes", "d2h_bytes"), (x.value for x in v)))
        d["kernels_per_run"] = int(self._lib.gpu_batch_kernels(self._h))
        return d

    def dedup(self):
        """(modes, sort keys): per rule, how its body size deduplicates pairs
        in the current staging (gpu_batch_dedup: -1 none on the device, 0
        shared bitmap, 1 global rows, 2 block rows, 3 sorted keys), and the
        pair keys the last run appended."""
        import numpy as np
        m = np.zeros(max(self.n, 1), dtype=np.int32)
        k = ctypes.c_longlong()
        if self._lib.gpu_batch_dedup(self._h, m.ctypes.data, ctypes.byref(k)) != 0:
            raise RuntimeError("gpu_batch_dedup failed")
        return m[:self.n], k.value

    def autotune(self, rounds: int = 1) -> None:
        """Measure task times and rebalance the batch's tasks (see gpu_batch_autotune)."""
        if self._lib.gpu_batch_autotune(self._h, rounds) != 0:
            raise RuntimeError(f"gpu_batch_autotune failed ({self._lib.gpu_last_error().decode(errors='replace')})")

    def count_bytes(self) -> int:
        b = ctypes.c_ulonglong()
        if self._lib.gpu_batch_count_bytes(self._h, ctypes.byref(b)) != 0:
            raise RuntimeError("gpu_batch_count_bytes failed")
        return b.value

    def profile(self):
        """Instrumented run: (algorithmic bytes, task table) where each task row is
        (rule, phase, root_begin, root_end, start_ns, end_ns)."""
        import numpy as np
        n = self.info()["tasks"]
        ns = np.zeros((max(n, 1), 2), dtype=np.uint64)
        ti = np.zeros((max(n, 1), 3), dtype=np.int32)
        b = ctypes.c_ulonglong()
        if self._lib.gpu_batch_profile(self._h, ctypes.byref(b), ns.ctypes.data, ti.ctypes.data, n) != 0:
            raise RuntimeError("gpu_batch_profile failed")
        tab = np.zeros((n, 6), dtype=np.int64)
        tab[:, 0] = ti[:n, 0] // 2
        tab[:, 1] = ti[:n, 0] % 2
        tab[:, 2:4] = ti[:n, 1:3]
        tab[:, 4:6] = ns[:n].astype(np.int64)
        return b.value, tab

    def close(self):
        if getattr(self, "_h", None) is not None:
            self._lib.gpu_batch_free(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class GpuServer:
    """Continuous-batching request loop on a loaded graph (gpu_serve_*)."""

    def __init__(self, lib: GpuRulesLib, slots: int = 3, max_batch: int = 4096, mem_budget: int = 1 << 30):
        self._owner = lib
        self._lib = lib._lib
        h = self._lib.gpu_serve_start(lib._handle(), slots, max_batch, mem_budget)
        if not h:
            raise RuntimeError(f"gpu_serve_start failed ({self._lib.gpu_last_error().decode(errors='replace')})")
        self._h = ctypes.c_void_p(h)
        self._buf = (GpuServeResult * 4096)()

    def submit(self, request_id: int, rule_text: str) -> None:
        if self._lib.gpu_serve_submit(self._h, request_id, rule_text.encode()) != 0:
            raise RuntimeError("gpu_serve_submit failed")

    def poll(self, wait_ms: int = 0) -> list:
        """Completed requests as (request_id, status, GpuRuleResult, latency_ms)."""
        n = self._lib.gpu_serve_poll(self._h, self._buf, len(self._buf), wait_ms)
        if n < 0:
            raise RuntimeError("gpu_serve_poll failed")
        out = []
        for i in range(n):
            r = self._buf[i]
            res = GpuRuleResult()
            ctypes.pointer(res)[0] = r.result
            out.append((r.requestId, r.status, res, r.latencyMs))
        return out

    def stats(self) -> dict:
        v = [ctypes.c_longlong() for _ in range(4)] + [ctypes.c_double() for _ in range(2)]
        self._lib.gpu_serve_stats(self._h, *[ctypes.byref(x) for x in v])
        return dict(zip(("submitted", "completed", "launches", "mem_in_use", "device_ms", "host_ms"),
                        (x.value for x in v)))

    def stop(self) -> None:
        if getattr(self, "_h", None) is not None:
            self._lib.gpu_serve_stop(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.stop()

    def __del__(self):
        try:
            self.stop()
        except Exception:
            pass

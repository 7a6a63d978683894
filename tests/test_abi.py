"""The C-ABI library: load, exported symbols, struct layout, host-side
error paths (CPU only; nothing here launches device work)."""
import ctypes
import re
import subprocess

import pytest
import torch

import masterthesis_gpu_acceleration_b200 as eng
from conftest import ROOT

HEADERS = sorted((ROOT / "include").glob("*.h"))


def _declared_functions():
    names = []
    for h in HEADERS:
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        names += re.findall(r"^\s*[A-Za-z_][\w\s\*]*?\b(gpu_\w+)\s*\(", text, flags=re.M)
    return sorted(set(names))


def test_library_exists_and_loads():
    assert eng.LIB_PATH.exists(), "build with python -m masterthesis_gpu_acceleration_b200.build"
    eng.load_library()


def test_exports_every_declared_symbol():
    declared = _declared_functions()
    assert {"gpu_load_graph", "gpu_evaluate_rule", "gpu_evaluate_rule_json",
            "gpu_free_graph", "gpu_query_vram"} <= set(declared)
    out = subprocess.run(["nm", "-D", "--defined-only", str(eng.LIB_PATH)], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (gpu_\w+)$", out, flags=re.M))
    assert set(declared) <= exported, set(declared) - exported
    assert set(eng.API_SYMBOLS) == set(declared)


def test_result_struct_layout_matches_reference():
    # GPU_03/gpu_rules_api.h:21-30 with natural alignment on x86-64
    R = eng.GpuRuleResult
    assert ctypes.sizeof(R) == 56
    offs = [getattr(R, f).offset for f, _ in R._fields_]
    assert offs == [0, 4, 8, 16, 24, 32, 40, 48]
    # the C header agrees
    src = ROOT / "include" / "gpu_rules_api.h"
    prog = r'''
#include <stdio.h>
#include <stddef.h>
#include "gpu_rules_api.h"
int main(void){printf("%zu %zu %zu %zu %zu %zu %zu %zu %zu\n", sizeof(GpuRuleResult),
 offsetof(GpuRuleResult,support), offsetof(GpuRuleResult,headSize), offsetof(GpuRuleResult,headSupport),
 offsetof(GpuRuleResult,headCoverage), offsetof(GpuRuleResult,bodySize), offsetof(GpuRuleResult,confidence),
 offsetof(GpuRuleResult,supportMs), offsetof(GpuRuleResult,confidenceMs)); return 0;}
'''
    import tempfile, os
    with tempfile.TemporaryDirectory() as t:
        c = os.path.join(t, "l.c")
        open(c, "w").write(prog)
        subprocess.run(["gcc", "-I", str(src.parent), c, "-o", os.path.join(t, "l")], check=True)
        out = subprocess.run([os.path.join(t, "l")], capture_output=True, text=True).stdout.split()
    assert list(map(int, out)) == [56, 0, 4, 8, 16, 24, 32, 40, 48]


def test_null_arguments_are_errors_not_crashes():
    lib = eng.load_library()
    res = eng.GpuRuleResult()
    assert lib.gpu_evaluate_rule(None, b"(?a <p> ?b) => (?a <q> ?b)", ctypes.byref(res)) == -1
    assert lib.gpu_evaluate_rule_json(None, b"{}", ctypes.byref(res)) == -1
    assert lib.gpu_evaluate_rules_batch(None, None, 0, 0, None, None, None) == -1
    lib.gpu_free_graph(None)
    assert lib.gpu_load_graph(None) is None


@pytest.mark.skipif(torch.cuda.is_available(), reason="checks the no-device path")
def test_no_device_paths_return_errors(tmp_path):
    lib = eng.load_library()
    f, t = ctypes.c_size_t(), ctypes.c_size_t()
    assert lib.gpu_query_vram(ctypes.byref(f), ctypes.byref(t)) == -1
    ttl = tmp_path / "g.ttl"
    ttl.write_text("<http://e/1> <http://p/0> <http://e/2> .\n")
    assert lib.gpu_load_graph(str(ttl).encode()) is None
    assert b"gpu_load_graph" in lib.gpu_last_error()


def test_missing_file_is_an_error(tmp_path):
    lib = eng.load_library()
    assert lib.gpu_load_graph(str(tmp_path / "absent.ttl").encode()) is None

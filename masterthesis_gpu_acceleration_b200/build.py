"""Builds the native libraries in-tree (sm_100a only).

    libgpu_rules.so  the engine and its C ABI (include/gpu_rules_api.h)
    libkg_synth.so   the seeded synthetic graph / rule generator

Objects are compiled in parallel into masterthesis_gpu_acceleration_b200/_build
and linked into masterthesis_gpu_acceleration_b200/lib.  A library is rebuilt
when any of its sources or headers is newer than it.
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "lib"
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

ENGINE_SOURCES = ["turtle.cpp", "rules.cpp", "index.cpp", "index_io.cpp", "planner.cpp", "tasks.cpp", "kernels.cu",
                  "sort.cu", "index_gpu.cu", "context.cu", "serve.cu"]
HEADERS = ["common.hpp", "turtle.hpp", "rules.hpp", "index.hpp", "index_io.hpp", "planner.hpp", "tasks.hpp",
           "engine.hpp", "parallel.hpp"]


def _newer(target: Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(Path(d).stat().st_mtime > t for d in deps)


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed: " + " ".join(map(str, cmd)) + "\n" + r.stdout + r.stderr)
    return r.stdout + r.stderr


def _compile(src: str, verbose: bool) -> Path:
    s = CSRC / src
    obj = BUILD / (src + ".o")
    deps = [s] + [CSRC / h for h in HEADERS] + [ROOT / "include" / "gpu_rules_api.h"]
    if not _newer(obj, deps):
        return obj
    flags = ["-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-I", str(ROOT / "include")]
    if src.endswith(".cu"):
        cmd = [NVCC, *ARCH, "-lineinfo", *flags, "-c", str(s), "-o", str(obj)]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
    else:
        cmd = [NVCC, "-x", "cu", *ARCH, *flags, "-c", str(s), "-o", str(obj)]
    out = _run(cmd)
    if verbose and out:
        print(out, file=sys.stderr)
    return obj


def build_engine(verbose: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    LIB.mkdir(exist_ok=True)
    with ThreadPoolExecutor(max_workers=len(ENGINE_SOURCES)) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), ENGINE_SOURCES))
    so = LIB / "libgpu_rules.so"
    if _newer(so, objs):
        _run([NVCC, *ARCH, "-shared", *map(str, objs), "-o", str(so), "-lcudart"])
    return so


def build_synth() -> Path:
    LIB.mkdir(exist_ok=True)
    src = CSRC / "kg_synth.cpp"
    so = LIB / "libkg_synth.so"
    if _newer(so, [src]):
        _run(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", str(src), "-o", str(so)])
    return so


def build_all(verbose: bool = False) -> None:
    build_synth()
    build_engine(verbose)


if __name__ == "__main__":
    build_all(verbose="-v" in sys.argv)
    print("built", LIB)

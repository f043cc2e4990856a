"""Build the native parts of coincgraph_b200 in-tree.

- ``coincgraph_b200/libcig.so``: the sm_100a engine (``csrc/engine.cu``)
  behind the C ABI of ``include/cig.h``;
- ``coincgraph_b200/libcig_gen.so``: seeded graph/update generator
  (``csrc/graphgen.cpp``, host only, OpenMP);
- ``coincgraph_b200/bin/hybrid_{bfs,sssp,cc,pr}``: the drop-in command-line
  tools (``csrc/cli/hybrid_main.cpp``) linked against ``libcig.so``.

Usage: ``python -m coincgraph_b200.build [--force]``.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

CLI_TOOLS = ("bfs", "sssp", "cc", "pr")


def _run(cmd: list[str]) -> str:
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
        sys.stderr.write(proc.stdout + proc.stderr)
        raise RuntimeError("build step failed: " + " ".join(cmd))
    return proc.stdout + proc.stderr


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _sources(ext: tuple[str, ...]) -> list[str]:
    out = []
    for dirpath, _, files in os.walk(CSRC):
        out += [os.path.join(dirpath, f) for f in files if f.endswith(ext)]
    return out


def build_engine(force: bool = False, verbose_ptxas: bool = False) -> str:
    out = os.path.join(HERE, "libcig.so")
    deps = _sources((".cu", ".cuh")) + [os.path.join(INCLUDE, "cig.h")]
    if force or verbose_ptxas or _stale(out, deps):
        cmd = [NVCC, *ARCH, "-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr",
               "-Xcompiler", "-fPIC", "-shared", "-I" + INCLUDE,
               os.path.join(CSRC, "engine.cu"), os.path.join(CSRC, "noalloc.cu"), "-o", out]
        if verbose_ptxas:
            cmd.insert(1, "-Xptxas=-v")
        log = _run(cmd)
        if verbose_ptxas:
            sys.stdout.write(log)
    return out


def build_engine_bounds_checked(force: bool = False) -> str:
    """``libcig_bc.so``: the engine compiled with -DCIG_BOUNDS_CHECK, which
    checks every arena slot and every vertex id read from a row against its
    bound and reports a violation through the device status word
    (CIG_ERR_LIMIT, "device index out of bounds") instead of touching memory
    outside the arrays.  A test-and-debug build (slower); select it with
    CIG_LIBRARY=<path> in the Python binding or by linking it instead of
    libcig.so."""
    out = os.path.join(HERE, "libcig_bc.so")
    deps = _sources((".cu", ".cuh")) + [os.path.join(INCLUDE, "cig.h")]
    if force or _stale(out, deps):
        _run([NVCC, *ARCH, "-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr", "-DCIG_BOUNDS_CHECK",
              "-Xcompiler", "-fPIC", "-shared", "-I" + INCLUDE,
              os.path.join(CSRC, "engine.cu"), os.path.join(CSRC, "noalloc.cu"), "-o", out])
    return out


def build_generator(force: bool = False) -> str:
    out = os.path.join(HERE, "libcig_gen.so")
    src = os.path.join(CSRC, "graphgen.cpp")
    if force or _stale(out, [src, os.path.join(INCLUDE, "cig_gen.h")]):
        _run(["g++", "-std=c++17", "-O3", "-fopenmp", "-fPIC", "-shared", src, "-o", out])
    return out


def build_cli(force: bool = False) -> list[str]:
    src = os.path.join(CSRC, "cli", "hybrid_main.cpp")
    if not os.path.exists(src):
        return []
    bindir = os.path.join(HERE, "bin")
    os.makedirs(bindir, exist_ok=True)
    deps = [src, os.path.join(INCLUDE, "cig.h"), os.path.join(HERE, "libcig.so")]
    outs = []
    for tool in CLI_TOOLS:
        out = os.path.join(bindir, "hybrid_" + tool)
        if force or _stale(out, deps):
            _run(["g++", "-std=c++17", "-O2", "-I" + INCLUDE, f"-DCIG_TOOL_{tool.upper()}=1", src,
                  "-o", out, "-L" + HERE, "-lcig", "-Wl,-rpath,$ORIGIN/..", "-lpthread"])
        outs.append(out)
    return outs


def build_all(force: bool = False) -> dict:
    return {
        "engine": build_engine(force),
        "engine_bounds_checked": build_engine_bounds_checked(force),
        "generator": build_generator(force),
        "cli": build_cli(force),
    }


if __name__ == "__main__":
    force = "--force" in sys.argv
    if "--ptxas" in sys.argv:
        build_engine(verbose_ptxas=True)
    else:
        print(build_all(force))

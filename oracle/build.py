"""Build recipe for the CPU oracle (test infrastructure only).

- ``oracle/liboracle.so``: the plain-C restatement in ``oracle/oracle.c``.
- ``oracle/_ref/libcigref.so``: ``oracle/ref_shim.cpp`` compiled together with
  the reference's own sources where they lie (its header-only
  ``SourceLocalChunkStore`` and the host checkers
  ``samples/hybrid_cc/hybrid_cc_host.cu`` and
  ``samples/hybrid_pr/hybrid_pr_host.cu``).  Built only when the reference
  tree is present; the built file travels with the repository snapshot.

Nothing in the product imports this module.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
# The reference source tree (read-only; only this recipe reads it).
REFERENCE = os.environ.get("CIG_REFERENCE_DIR", "/root/reference")
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")


def _run(cmd: list[str]) -> None:
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
        sys.stderr.write(proc.stdout + proc.stderr)
        raise RuntimeError("command failed: " + " ".join(cmd))


def _stale(target: str, sources: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources if os.path.exists(s))


def build_oracle(force: bool = False) -> str:
    src = os.path.join(HERE, "oracle.c")
    out = os.path.join(HERE, "liboracle.so")
    if force or _stale(out, [src, os.path.join(HERE, "oracle.h")]):
        _run(["gcc", "-O2", "-std=c11", "-fPIC", "-shared", src, "-o", out, "-lm"])
    return out


def build_ref(force: bool = False) -> str | None:
    """Compile the reference's CPU code; returns None when the tree is absent."""
    out_dir = os.path.join(HERE, "_ref")
    out = os.path.join(out_dir, "libcigref.so")
    if not os.path.isdir(os.path.join(REFERENCE, "include")):
        return out if os.path.exists(out) else None
    cc_host = os.path.join(REFERENCE, "samples", "hybrid_cc", "hybrid_cc_host.cu")
    pr_host = os.path.join(REFERENCE, "samples", "hybrid_pr", "hybrid_pr_host.cu")
    shim = os.path.join(HERE, "ref_shim.cpp")
    if not (force or _stale(out, [shim, cc_host, pr_host])):
        return out
    os.makedirs(out_dir, exist_ok=True)
    _run([
        "g++", "-std=c++17", "-O2", "-fPIC", "-shared",
        "-I" + os.path.join(REFERENCE, "include"),
        "-I" + os.path.join(REFERENCE, "samples", "hybrid_cc"),
        "-I" + os.path.join(REFERENCE, "samples", "hybrid_pr"),
        "-I" + os.path.join(CUDA_HOME, "include"),
        shim, "-x", "c++", cc_host, pr_host, "-x", "none",
        "-o", out,
        "-L" + os.path.join(CUDA_HOME, "lib64"), "-lcudart", "-lpthread",
        "-Wl,-rpath," + os.path.join(CUDA_HOME, "lib64"),
    ])
    return out


if __name__ == "__main__":
    print(build_oracle(force=True))
    print(build_ref(force=True))

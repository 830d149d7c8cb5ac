"""Build libxcal_b200.so in-tree with nvcc for sm_100a.

Flags that matter for the arithmetic contract:
  --fmad=false                  no a*b+c contraction on the device (the Julia
                                reference never fuses)
  -Xcompiler -ffp-contract=off  same for host-side geometry precomputation
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libxcal_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

FLAGS = [
    "-O3", "-std=c++17", "-shared", "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off",
    "--fmad=false", "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo",
    "-Xptxas", "-warn-spills",
]


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def needs_build() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = sources() + glob.glob(os.path.join(CSRC, "*.h*")) + glob.glob(os.path.join(CSRC, "*.cuh"))
    deps.append(os.path.join(HERE, "..", "include", "xcal_b200.h"))
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False, extra=None) -> str:
    """Compile every csrc/*.cu to an object file (in parallel, under
    _build/), then link the shared library."""
    if not force and not needs_build():
        return LIB
    from concurrent.futures import ThreadPoolExecutor
    env = dict(os.environ)
    # nvcc picks the host compiler from PATH; use the system g++
    env.pop("CXX", None)
    env.pop("CC", None)
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    compile_flags = [f for f in FLAGS if f != "-shared"] + (extra or [])

    def compile_one(src):
        obj = os.path.join(objdir, os.path.basename(src)[:-3] + ".o")
        cmd = [NVCC] + compile_flags + ["-c", "-o", obj, src]
        r = subprocess.run(cmd, cwd=CSRC, capture_output=True, text=True, env=env)
        return src, obj, cmd, r

    with ThreadPoolExecutor(max_workers=max(1, min(len(sources()), os.cpu_count() or 1))) as ex:
        results = list(ex.map(compile_one, sources()))
    failed = False
    for src, obj, cmd, r in results:
        if verbose or r.returncode != 0:
            sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        failed |= r.returncode != 0
    if failed:
        raise RuntimeError("nvcc failed building libxcal_b200.so")
    cmd = [NVCC, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", LIB] + [o for _, o, _, _ in results]
    r = subprocess.run(cmd, cwd=CSRC, capture_output=True, text=True, env=env)
    if verbose or r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
    if r.returncode != 0:
        raise RuntimeError("linking libxcal_b200.so failed")
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)

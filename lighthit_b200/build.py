"""Build the sm_100a shared library in-tree: ``python -m lighthit_b200.build``.

One nvcc invocation compiles every ``csrc/*.cu`` into ``liblh_b200.so`` next
to this file (the library travels with the source tree; nothing is installed
elsewhere).
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
LIB = HERE / "liblh_b200.so"
SOURCES = sorted((HERE / "csrc").glob("*.cu"))
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc():
    found = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(found).exists():
        raise RuntimeError("nvcc not found; the CUDA 12.9 toolkit is required to build")
    return found


def needs_build():
    if not LIB.exists():
        return True
    newest = max(p.stat().st_mtime for p in list((HERE / "csrc").glob("*")) +
                 [HERE.parent / "include" / "lighthit_b200.h"])
    return LIB.stat().st_mtime < newest


def build(verbose=False, force=False):
    """Compile if any source is newer than the library; return its path."""
    if not force and not needs_build():
        return LIB
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr",
           "-shared", "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off",
           "-I", str(HERE.parent / "include"),
           "-o", str(tmp), *map(str, SOURCES)]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    env = dict(os.environ)
    res = subprocess.run(cmd, capture_output=True, text=True, env=env)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError("nvcc failed building liblh_b200.so")
    if verbose:
        sys.stderr.write(res.stderr)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(verbose="-v" in sys.argv, force=True)
    print(LIB)

"""Compile the oracle's C restatements with gcc (test infrastructure only).

``python -m oracle.build`` (also run by ``__graft_entry__.build()``) writes
``oracle/liboracle.so`` next to the sources.
"""
from __future__ import annotations

import shutil
import subprocess
from pathlib import Path

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"
SOURCES = sorted(HERE.glob("*.c"))


def build(force=False):
    if not force and LIB.exists() and all(LIB.stat().st_mtime >= s.stat().st_mtime for s in SOURCES):
        return LIB
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        raise RuntimeError("gcc is needed to build the oracle")
    tmp = LIB.with_suffix(".so.tmp")
    # -ffp-contract=off: no fused multiply-adds, as NumPy/Numba evaluate these expressions
    subprocess.run([cc, "-O2", "-fPIC", "-shared", "-ffp-contract=off", "-o", str(tmp),
                    *map(str, SOURCES), "-lm"], check=True)
    tmp.replace(LIB)
    return LIB


if __name__ == "__main__":
    print(build(force=True))

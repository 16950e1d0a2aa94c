"""Builds the CPU oracle (test infrastructure only) into oracle/_build/liboracle.so.

The oracle is a C restatement of the reference's box FGT used by the tests,
by __graft_entry__.smoke() as the checker and by bench.py's CPU-baseline leg.
The product library never links it.

The reference itself is Fortran 77 and no Fortran compiler exists in this
image, so there is no oracle/_ref build of the reference sources.
"""
from __future__ import annotations

import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
SRC = HERE / "bfgt_oracle.c"
OUT = HERE / "_build" / "liboracle.so"


def build(force: bool = False) -> Path:
    if not force and OUT.exists() and OUT.stat().st_mtime >= SRC.stat().st_mtime:
        return OUT
    OUT.parent.mkdir(exist_ok=True)
    cmd = ["gcc", "-O2", "-std=gnu11", "-fPIC", "-shared", "-fopenmp", "-ffp-contract=off", "-fno-fast-math",
           "-march=x86-64-v2", str(SRC), "-o", str(OUT) + ".tmp", "-lm"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("oracle build failed")
    Path(str(OUT) + ".tmp").replace(OUT)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))

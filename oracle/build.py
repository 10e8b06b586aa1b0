"""Build the oracle (test infrastructure): ``oracle/liboracle.so``.

The oracle is a C++ f64 restatement of the crabSAXS reference algorithms
(oracle.cpp).  It is compiled with -ffp-contract=off so no multiply-add is
fused, and with OpenMP so the per-q loops run on every host core the way the
reference's rayon loops do.  The reference itself is Rust and cannot be
compiled in this environment (no cargo/rustc), so there is no oracle/_ref.
"""
from __future__ import annotations

import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
SRC = HERE / "oracle.cpp"
LIB = HERE / "liboracle.so"
# The seeded synthetic-structure generator (input generation, not a reference
# algorithm) is compiled in as orc_synth_protein, so a CPU measurement of the
# reference path can make its input without loading the product library.
SYNTH = HERE.parent / "crabsaxs_b200" / "csrc" / "synth.cpp"
INCLUDE = HERE.parent / "include"


def build() -> Path:
    if LIB.exists() and LIB.stat().st_mtime >= max(SRC.stat().st_mtime, SYNTH.stat().st_mtime):
        return LIB
    cmd = ["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-fopenmp", "-ffp-contract=off", f"-I{INCLUDE}",
           "-Dcrab_synth_protein=orc_synth_protein", "-o", str(LIB), str(SRC), str(SYNTH)]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"oracle build failed:\n{res.stdout}\n{res.stderr}")
    return LIB


if __name__ == "__main__":
    print(build())
    sys.exit(0)

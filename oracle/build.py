"""Builds the oracle (test infrastructure): oracle/libda_oracle.so from da_oracle.c.

Compiled with -ffp-contract=off so that no multiply-add is fused: the restatement keeps
the reference's rounding sequence.  Only tests, smoke() and bench.py's CPU legs load it.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libda_oracle.so")
SRC = os.path.join(HERE, "da_oracle.c")


def build(verbose: bool = False, force: bool = False) -> str:
    deps = [SRC, __file__, os.path.join(ROOT, "include", "discrete_adjoint.h")]
    extra = [os.path.join(HERE, f) for f in os.listdir(HERE) if f.startswith("da_oracle") and f.endswith(".c")]
    deps += extra
    if force or not os.path.exists(LIB) or any(os.path.getmtime(d) > os.path.getmtime(LIB) for d in deps):
        srcs = sorted(set(extra))
        cmd = ["gcc", "-O2", "-std=c11", "-fPIC", "-shared", "-ffp-contract=off", "-fno-fast-math",
               "-I" + os.path.join(ROOT, "include")] + srcs + ["-o", LIB, "-lm"]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    print(build(verbose=True, force="--force" in sys.argv))

"""Build the FP64 CPU oracle (test infrastructure only).

Compiles oracle/pa_oracle.cpp into oracle/_build/libpa_oracle.so with
g++ -O3 -fopenmp.  The product library never links this file.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT_DIR = os.path.join(HERE, "_build")
LIB = os.path.join(OUT_DIR, "libpa_oracle.so")


def build(force=False, verbose=False):
    src = os.path.join(HERE, "pa_oracle.cpp")
    os.makedirs(OUT_DIR, exist_ok=True)
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= os.path.getmtime(src):
        return LIB
    cmd = ["g++", "-O3", "-march=x86-64-v3", "-fopenmp", "-fPIC", "-shared", "-std=c++17",
           "-o", LIB + ".tmp", src]
    if verbose:
        print(" ".join(cmd))
    subprocess.check_call(cmd)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))

"""Build the FP64 CPU oracle (test infrastructure only).

Compiles oracle/pa_oracle.cpp with g++ -O3 -march=native -fopenmp into
oracle/_build/libpa_oracle-<host>.so, where <host> is a short hash of this
machine's CPU model and instruction-set flags: a library built on one host is
never loaded on a host whose CPU may lack its instructions, and the timed CPU
baseline is always compiled for the cores it runs on.  The product library
never links this file.
"""
import hashlib
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT_DIR = os.path.join(HERE, "_build")
FLAGS = ["-O3", "-march=native", "-fopenmp", "-fPIC", "-shared", "-std=c++17"]


def host_tag():
    """Hash of the CPU model name and flags (first processor in /proc/cpuinfo)."""
    model, flags = "", ""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name") and not model:
                    model = line.split(":", 1)[1].strip()
                elif line.startswith("flags") and not flags:
                    flags = line.split(":", 1)[1].strip()
                if model and flags:
                    break
    except OSError:
        pass
    return hashlib.sha1((model + "|" + flags).encode()).hexdigest()[:10]


LIB = os.path.join(OUT_DIR, f"libpa_oracle-{host_tag()}.so")


def build(force=False, verbose=False):
    src = os.path.join(HERE, "pa_oracle.cpp")
    os.makedirs(OUT_DIR, exist_ok=True)
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= os.path.getmtime(src):
        return LIB
    tmp = f"{LIB}.{os.getpid()}.tmp"
    cmd = ["g++"] + FLAGS + ["-o", tmp, src]
    if verbose:
        print(" ".join(cmd))
    subprocess.check_call(cmd)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))

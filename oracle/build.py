"""Builds the CPU oracle library (oracle/_build/liboracle.so) — test infrastructure only.

    python -m oracle.build          # oracle library
    python -m oracle.build --ref    # also the reference CUDA build into oracle/_ref (needs
                                    # the reference tree; see oracle/ref_build.py)
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(BUILD, "liboracle.so")

C_SOURCES = ["collatz.c", "bfs.c", "photon.c", "inputs.c"]
CXX_SOURCES = ["host_exec.cpp"]
SPEC_DIR = os.path.join(HERE, "..", "harmonize_b200", "csrc", "specs")


def _newer(target, sources):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def build(force=False, quiet=True):
    os.makedirs(BUILD, exist_ok=True)
    srcs = [os.path.join(HERE, s) for s in C_SOURCES + CXX_SOURCES]
    deps = srcs + [os.path.join(HERE, "host_api.h"),
                   os.path.join(HERE, "..", "include", "harmonize", "spec_support.h")]
    deps += [os.path.join(SPEC_DIR, f) for f in os.listdir(SPEC_DIR) if f.endswith(".h")]
    if not force and not _newer(LIB, deps):
        return LIB
    objs = []
    for s in srcs:
        o = os.path.join(BUILD, os.path.basename(s) + ".o")
        if s.endswith(".c"):
            cmd = ["gcc", "-O2", "-fPIC", "-fopenmp", "-ffp-contract=off", "-std=c11", "-c", s, "-o", o]
        else:
            cmd = ["g++", "-O2", "-fPIC", "-fopenmp", "-ffp-contract=off", "-std=c++17",
                   "-I", os.path.join(HERE, "..", "include"), "-I", HERE, "-c", s, "-o", o]
        subprocess.run(cmd, check=True, capture_output=quiet)
        objs.append(o)
    tmp = LIB + ".tmp"
    subprocess.run(["g++", "-shared", "-fopenmp", "-o", tmp] + objs + ["-lm"], check=True, capture_output=quiet)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, quiet=False))

"""Builds libhrm.so (the runtime's C ABI and built-in specs) for sm_100a, in-tree.

    python -m harmonize_b200.build [--force]

nvcc cross-compiles without a GPU. The library lands next to this file so that it travels
with the repository snapshot and is the one the tests and the bench load.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libhrm.so")
SOURCES = [os.path.join(HERE, "csrc", "hrm_capi.cu"), os.path.join(HERE, "csrc", "hrm_batch.cu"),
           os.path.join(HERE, "csrc", "inputs.cpp"), os.path.join(HERE, "csrc", "hrm_pyshim.cpp")]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC,-fopenmp", "-shared",
              "-I", os.path.join(ROOT, "include")]


def _deps():
    out = list(SOURCES)
    for d in (os.path.join(ROOT, "include"), os.path.join(HERE, "csrc")):
        for dirpath, _, files in os.walk(d):
            out += [os.path.join(dirpath, f) for f in files if f.endswith((".h", ".cuh", ".cu", ".cpp"))]
    return out


def needs_build():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(p) > t for p in _deps())


def build(force=False, verbose=False, extra=()):
    """Compiles every translation unit to an object in parallel, then links libhrm.so."""
    if not force and not needs_build():
        return LIB
    obj_dir = os.path.join(HERE, "_build")
    os.makedirs(obj_dir, exist_ok=True)
    flags = [f for f in NVCC_FLAGS if f != "-shared"]
    procs = []
    objs = []
    for src in SOURCES:
        obj = os.path.join(obj_dir, os.path.basename(src) + ".o")
        cmd = ["nvcc"] + ARCH + flags + list(extra) + ["-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd))
        procs.append((subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True), src))
        objs.append(obj)
    errors = []
    for p, src in procs:
        out, err = p.communicate()
        if p.returncode != 0:
            errors.append(f"{src}:\n{out}{err}")
    if errors:
        raise RuntimeError("nvcc failed:\n" + "\n".join(errors))
    tmp = LIB + ".tmp"
    cmd = ["nvcc"] + ARCH + ["-shared", "-Xcompiler", "-fopenmp", "-o", tmp] + objs + ["-lgomp"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("link failed:\n" + r.stdout + r.stderr)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))

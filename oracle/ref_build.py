"""Builds the reference CUDA build (TEST / BENCH INFRASTRUCTURE ONLY).

Compiles oracle/ref_glue.cu — the built-in spec sources driven by the ORIGINAL Harmonize
runtime — against the reference's headers where they lie, with the reference's own
recipe (`nvcc -std=c++17 --restrict -x cu -include harmonize/cpp/harmonize.h`,
examples/cpp/collaz/Makefile:28) plus `-arch=sm_100a`, into oracle/_ref/libhrm_ref.so.
Nothing from the reference tree is copied. The output is git-ignored but travels with the
repository snapshot to the GPU machine, where the reference tree is absent.

    python -m oracle.ref_build [--force] [--reference PATH]
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT_DIR = os.path.join(HERE, "_ref")
LIB = os.path.join(OUT_DIR, "libhrm_ref.so")
DEFAULT_REFERENCE = "/root/reference"


def reference_header(reference=DEFAULT_REFERENCE):
    return os.path.join(reference, "harmonize", "cpp", "harmonize.h")


def available():
    return os.path.exists(LIB)


def build(force=False, reference=DEFAULT_REFERENCE, quiet=True):
    hdr = reference_header(reference)
    if not os.path.exists(hdr):
        if os.path.exists(LIB):
            return LIB  # prebuilt copy (GPU machine)
        raise FileNotFoundError(f"reference headers not found at {hdr}")
    src = os.path.join(HERE, "ref_glue.cu")
    specs = os.path.join(HERE, "..", "harmonize_b200", "csrc", "specs")
    deps = [src] + [os.path.join(specs, f) for f in os.listdir(specs)]
    if not force and os.path.exists(LIB) and all(os.path.getmtime(d) <= os.path.getmtime(LIB) for d in deps):
        return LIB
    os.makedirs(OUT_DIR, exist_ok=True)
    tmp = LIB + ".tmp"
    cmd = ["nvcc", "-std=c++17", "--restrict", "-x", "cu", "-O3", "-arch=sm_100a", "-include", hdr,
           "-Xcompiler", "-fPIC", "-shared", "-o", tmp, src]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("reference build failed:\n" + r.stdout[-4000:] + r.stderr[-4000:])
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    ref = DEFAULT_REFERENCE
    if "--reference" in sys.argv:
        ref = sys.argv[sys.argv.index("--reference") + 1]
    print(build(force="--force" in sys.argv, reference=ref, quiet=False))

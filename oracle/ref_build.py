"""Builds the reference CUDA build (TEST / BENCH INFRASTRUCTURE ONLY).

Compiles oracle/ref_glue.cu — the built-in spec sources driven by the ORIGINAL Harmonize
runtime — against the reference's headers where they lie, with the reference's own
recipe (`nvcc -std=c++17 --restrict -x cu -include harmonize/cpp/harmonize.h`,
examples/cpp/collaz/Makefile:28) plus `-arch=sm_100a`, into oracle/_ref/libhrm_ref.so.
Nothing from the reference tree is copied. The output is git-ignored but travels with the
repository snapshot to the GPU machine, where the reference tree is absent.

    python -m oracle.ref_build [--force] [--reference PATH] [--examples]
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT_DIR = os.path.join(HERE, "_ref")
LIB = os.path.join(OUT_DIR, "libhrm_ref.so")
# Where the reference tree lies; HRM_REFERENCE_DIR overrides the default.
DEFAULT_REFERENCE = os.environ.get("HRM_REFERENCE_DIR", "/root/reference")


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


# ---------------------------------------------------------------------------------------------
# The reference's own example programs, unchanged, built against THIS runtime's header
# (include/harmonize.h forced in where the reference's Makefiles force in theirs,
# examples/cpp/collaz/Makefile:28 and examples/cpp/example_neutron/Makefile:36), so that a GPU
# test can run them: the program files are compiled where they lie; the AsyncProgram variant of
# the Collatz example is the one-line `using ProgType` swap of the README, written to a
# temporary file for the compile and deleted after it.
# ---------------------------------------------------------------------------------------------
EXAMPLES_DIR = os.path.join(OUT_DIR, "examples")
EXAMPLES = {
    "clz_hrm_event": ("examples/cpp/collaz/collaz_hrm.cpp", None),
    "clz_hrm_async": ("examples/cpp/collaz/collaz_hrm.cpp",
                      ("using ProgType = EventProgram < MyProgramSpec >;",
                       "using ProgType = AsyncProgram < MyProgramSpec >;")),
    "neut": ("examples/cpp/example_neutron/program.cpp", None),
}


def examples_available():
    return all(os.path.exists(os.path.join(EXAMPLES_DIR, k)) for k in EXAMPLES)


def build_examples(force=False, reference=DEFAULT_REFERENCE):
    import tempfile
    header = os.path.join(HERE, "..", "include", "harmonize.h")
    if not os.path.isdir(reference):
        if examples_available():
            return EXAMPLES_DIR
        raise FileNotFoundError(f"reference tree not found at {reference}")
    os.makedirs(EXAMPLES_DIR, exist_ok=True)
    our_headers = [os.path.join(r, f) for r, _, fs in os.walk(os.path.join(HERE, "..", "include")) for f in fs]
    for name, (rel, swap) in EXAMPLES.items():
        src = os.path.join(reference, rel)
        out = os.path.join(EXAMPLES_DIR, name)
        deps = [src] + our_headers
        if not force and os.path.exists(out) and all(os.path.getmtime(d) <= os.path.getmtime(out) for d in deps):
            continue
        tmpdir = None
        compile_src = src
        if swap is not None:
            text = open(src).read()
            if swap[0] not in text:
                raise RuntimeError(f"{rel}: the program-type line to swap was not found")
            tmpdir = tempfile.mkdtemp(prefix="hrm_example_")
            compile_src = os.path.join(tmpdir, os.path.basename(src))
            with open(compile_src, "w") as f:
                f.write(text.replace(swap[0], swap[1]))
        try:
            cmd = ["nvcc", "-std=c++17", "--restrict", "-x", "cu", "-O3",
                   "-gencode", "arch=compute_100a,code=sm_100a", "-include", os.path.abspath(header),
                   "-I", os.path.dirname(src), "-o", out + ".tmp", compile_src]
            r = subprocess.run(cmd, capture_output=True, text=True, cwd=os.path.dirname(src))
            if r.returncode != 0:
                raise RuntimeError(f"building {rel} failed:\n" + r.stderr[-4000:])
            os.replace(out + ".tmp", out)
        finally:
            if tmpdir is not None:
                import shutil
                shutil.rmtree(tmpdir, ignore_errors=True)
    return EXAMPLES_DIR


if __name__ == "__main__":
    ref = DEFAULT_REFERENCE
    if "--reference" in sys.argv:
        ref = sys.argv[sys.argv.index("--reference") + 1]
    print(build(force="--force" in sys.argv, reference=ref, quiet=False))
    if "--examples" in sys.argv:
        print(build_examples(force="--force" in sys.argv, reference=ref))

"""Source compatibility: unchanged Harmonize programs compile against include/harmonize.h.

The reference's own example programs are compiled where they lie (read-only), with the
reference's Makefile recipe but this runtime's header forced in instead of the original
(`nvcc -std=c++17 --restrict -x cu -include harmonize.h`, examples/cpp/collaz/Makefile:28).
Skipped where the reference tree is absent (e.g. on the GPU machine). The built-in specs are
also compiled against the original headers by oracle/ref_build.py.
"""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.environ.get("HRM_REFERENCE_DIR", "/root/reference")  # overridable reference location
HEADER = os.path.join(ROOT, "include", "harmonize.h")

EXAMPLES = [
    "examples/cpp/collaz/collaz_hrm.cpp",       # EventProgram, Even/Odd, AtomicIter, DevBuf, ArgSet
    "examples/cpp/collaz/collaz_std.cpp",       # plain kernel using the util:: host helpers
    "examples/cpp/example_neutron/program.cpp", # both program types, load_fraction, sync, cli_graph
]


@pytest.mark.skipif(not os.path.isdir(REF), reason="reference tree not present")
@pytest.mark.parametrize("example", EXAMPLES)
def test_reference_example_compiles_unchanged(example, tmp_path):
    src = os.path.join(REF, example)
    cmd = ["nvcc", "-std=c++17", "--restrict", "-x", "cu", "-gencode", "arch=compute_100a,code=sm_100a",
           "-include", HEADER, "-c", src, "-o", str(tmp_path / "out.o")]
    r = subprocess.run(cmd, capture_output=True, text=True, cwd=os.path.dirname(src))
    assert r.returncode == 0, r.stderr[-3000:]


@pytest.mark.skipif(not os.path.isdir(REF), reason="reference tree not present")
def test_collatz_example_switches_program_type_with_one_line(tmp_path):
    # The README's one-line swap (EventProgram -> AsyncProgram) on the unchanged source.
    src = open(os.path.join(REF, "examples/cpp/collaz/collaz_hrm.cpp")).read()
    assert "using ProgType = EventProgram < MyProgramSpec >;" in src
    swapped = tmp_path / "collaz_async.cpp"
    swapped.write_text(src.replace("using ProgType = EventProgram < MyProgramSpec >;",
                                   "using ProgType = AsyncProgram < MyProgramSpec >;"))
    cmd = ["nvcc", "-std=c++17", "--restrict", "-x", "cu", "-gencode", "arch=compute_100a,code=sm_100a",
           "-include", HEADER, "-c", str(swapped), "-o", str(tmp_path / "out.o")]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]

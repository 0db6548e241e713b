"""LazyLoad arguments (promise.h:208-240 of the original, its ASYNC_LOADS form) on the GPU.

tests/cpp/lazy_load.cu is a user's program whose async calls name their next table entries
by reference (LazyLoad<unsigned int>, LazyLoad<Pair>). Under AsyncProgram those arguments are
copied asynchronously into the promises' shared-memory slots (cp.async), and the team waits
for the copies only before it reads its rings; promises that overflow to the arena read the
value at the call (LEAP=4 makes make_work overflow the two-link rings). Under EventProgram
the values are read at the call. The program checks every walk against the same walk on the
host and exits nonzero on a mismatch; the outputs of all builds must also agree."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "lazy_load.cu")


def build(tmp_path, program_type, leap):
    exe = tmp_path / f"lazy_{program_type}_{leap}"
    subprocess.run(["nvcc", "-std=c++17", "-O3", "-gencode", "arch=compute_100a,code=sm_100a",
                    "-I", os.path.join(ROOT, "include"), f"-DPROGRAM_TYPE={program_type}", f"-DLEAP={leap}",
                    SRC, "-o", str(exe)], check=True, capture_output=True, timeout=600)
    return exe


@pytest.mark.gpu
def test_lazy_load_arguments_all_paths(tmp_path):
    count, steps = 200_000, 9
    outs = {}
    for program_type, leap in (("AsyncProgram", 1), ("AsyncProgram", 4), ("EventProgram", 1)):
        exe = build(tmp_path, program_type, leap)
        out = tmp_path / f"out_{program_type}_{leap}.bin"
        r = subprocess.run([str(exe), str(count), str(steps), str(out)], capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, f"{program_type} leap {leap}: {r.stdout} {r.stderr}"
        assert "mismatches 0" in r.stdout
        outs[(program_type, leap)] = np.fromfile(out, dtype=np.uint32)
    ref = outs[("EventProgram", 1)]
    for k, v in outs.items():
        assert np.array_equal(v, ref), k

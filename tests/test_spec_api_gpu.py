"""The two host-side ways into the runtime, driven on the GPU the way a user drives them.

1. The C++ spec API: tests/cpp/collatz_two_fn.cu is a user's program (its own spec, its own
   main with Instance / init<P> / exec<P> / complete) that includes only include/harmonize.h.
   It is compiled here twice, the program type swapped on one line (PROGRAM_TYPE), and both
   builds must give the oracle's stopping times.
2. The C ABI life cycle (hrm_program_create / init / exec / complete / stats / overview /
   clear_flags / destroy, the counterparts of the generated alloc_program_S, init_program_S,
   exec_program_S, complete_S, clear_flags_S and free_program_S of harmonize/python/templates.py),
   with small exec budgets so that a run spans many execs and resumes from the queues it left.
3. Failure detection without a fault: the runtime's bounded waits, made to run out on purpose.
"""
import os
import struct
import subprocess

import numpy as np
import pytest

import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "collatz_two_fn.cu")


@pytest.mark.gpu
@pytest.mark.parametrize("program_type", ["AsyncProgram", "EventProgram"])
def test_user_spec_program_both_program_types(program_type, tmp_path):
    exe = tmp_path / "collatz_two_fn"
    subprocess.run(["nvcc", "-std=c++17", "-O3", "-gencode", "arch=compute_100a,code=sm_100a",
                    "-I", os.path.join(ROOT, "include"), f"-DPROGRAM_TYPE={program_type}", SRC, "-o", str(exe)],
                   check=True, capture_output=True, timeout=600)
    start, count = 3, 50000
    out = tmp_path / "steps.bin"
    r = subprocess.run([str(exe), str(start), str(count), str(out)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    got = np.fromfile(out, dtype=np.uint32)
    assert np.array_equal(got, oracle.collatz_range(start, count))


def _collatz_state(start, count, out, it):
    # hrm_collatz_state: uint32 start, uint32 limit, uint32* output, void* iterator, uint32 leap
    return struct.pack("<IIQQI4x", start, start + count, out.data_ptr(), it.data_ptr(), 1)


@pytest.mark.gpu
@pytest.mark.parametrize("program,groups,n", [("async", 4, 128), ("async", 0, 0), ("event", 0, 1)])
def test_c_abi_life_cycle(hrm, program, groups, n):
    import torch
    start, count = 1, 30000
    out = torch.full((count,), -1, dtype=torch.int32, device="cuda")
    it = torch.tensor([start, start + count], dtype=torch.int32, device="cuda")
    prog = hrm.Program(hrm.SPEC_COLLATZ, program, arena=0, state=_collatz_state(start, count, out, it))
    try:
        prog.init(groups)
        execs = 0
        while True:
            prog.exec(groups, n)
            execs += 1
            if prog.complete():
                break
            assert execs < 200000
        ref = oracle.collatz_range(start, count)
        assert np.array_equal(out.cpu().numpy().view(np.uint32), ref)
        if program == "async" and groups == 4:
            assert execs > 10  # the run resumed from its queues across many execs
        st = prog.stats()
        assert st["evals"] == int(ref.astype(np.uint64).sum()) + count
        ov = prog.overview()
        if program == "async":
            # links handed out == links on the free list; both function queues and rings empty
            assert ov[0] == ov[1] and not any(ov[2:6])
        else:
            assert not any(ov)  # no promise waiting for either function
        if program == "async":
            assert prog.flags() & hrm.FLAG_COMPLETION  # set by the team that saw quiescence
        else:
            assert prog.flags() & 0xFF == 0  # EventProgram completes when no input is left
        prog.clear_flags()
        assert prog.flags() == 0
    finally:
        prog.close()


@pytest.mark.gpu
def test_waits_that_nobody_ends_time_out_with_a_status(tmp_path):
    """tests/cpp/wait_timeouts.cu makes each bounded wait of the runtime run out on purpose (a
    queue entry never published, a full queue nobody drains, a grid barrier one CTA short):
    each raises WAIT_TIMEOUT and returns an error instead of spinning, the context stays
    usable, and a normal publish-and-take round trip raises nothing."""
    exe = tmp_path / "wait_timeouts"
    subprocess.run(["nvcc", "-std=c++17", "-O3", "-gencode", "arch=compute_100a,code=sm_100a",
                    "-I", os.path.join(ROOT, "include"), os.path.join(ROOT, "tests", "cpp", "wait_timeouts.cu"),
                    "-o", str(exe)], check=True, capture_output=True, timeout=600)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.count("timed out as expected") == 3 and "no wait ran out" in r.stdout

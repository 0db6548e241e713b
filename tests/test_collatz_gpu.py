"""Collatz on the GPU runtime against the CPU oracle (bit-exact uint32 stopping times)."""
import numpy as np
import pytest

import oracle


@pytest.mark.gpu
@pytest.mark.parametrize("program", ["async", "event"])
@pytest.mark.parametrize("start,count", [(0, 1), (0, 1000), (1, 1 << 16), (12345, 77777)])
def test_collatz_matches_oracle(hrm, program, start, count):
    out, res = hrm.collatz(start, count, program=program)
    ref = oracle.collatz_range(start, count)
    assert np.array_equal(out, ref), f"first mismatch at {np.nonzero(out != ref)[0][:5]}"
    assert res["evals"] == int(ref.astype(np.uint64).sum()) + count

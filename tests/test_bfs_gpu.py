"""Label-correcting BFS on the GPU runtime against the serial BFS oracle (bit-exact levels)."""
import numpy as np
import pytest

import oracle


@pytest.fixture(scope="module")
def rmat14(hrm):
    return hrm.rmat_csr(14, 16, seed=3)


@pytest.mark.gpu
@pytest.mark.parametrize("program", ["async", "event"])
@pytest.mark.parametrize("root", [0, 1, 777])
def test_bfs_matches_oracle(hrm, rmat14, program, root):
    rp, col = rmat14
    levels, res = hrm.bfs(rp, col, root, program=program)
    ref = oracle.bfs(rp, col, root)
    assert np.array_equal(levels, ref)
    assert res["evals"] > 0


@pytest.mark.gpu
@pytest.mark.parametrize("program", ["async", "event"])
def test_bfs_path_graph(hrm, program):
    # a long chain: 0 -> 1 -> ... -> n-1 (deep, one promise per level)
    n = 5000
    rp = np.arange(n + 1, dtype=np.uint32)
    rp[-1] = n - 1
    col = np.arange(1, n, dtype=np.uint32)
    levels, _ = hrm.bfs(rp, col, 0, program=program)
    assert np.array_equal(levels, np.arange(n, dtype=np.uint32))


@pytest.mark.gpu
def test_bfs_isolated_root(hrm):
    rp = np.zeros(9, dtype=np.uint32)
    col = np.zeros(0, dtype=np.uint32)
    levels, _ = hrm.bfs(rp, col, 3)
    exp = np.full(8, 0xFFFFFFFF, dtype=np.uint32)
    exp[3] = 0
    assert np.array_equal(levels, exp)


@pytest.mark.gpu
def test_arena_exhaustion_is_reported_and_the_next_run_is_sound(hrm, rmat14):
    """One CTA and an arena of 32 links for a frontier of thousands of vertices: the device
    raises ARENA_EXHAUSTED, the run ends with an error status instead of waiting, and the next
    run, on an arena of the default size, is exact."""
    rp, col = rmat14
    with pytest.raises(hrm.HarmonizeError) as err:
        hrm.bfs(rp, col, 0, program="async", groups=1, arena=32)
    assert err.value.code == hrm.HRM_EDEVICE and "ARENA_EXHAUSTED" in str(err.value)
    levels, _ = hrm.bfs(rp, col, 0, program="async")
    assert np.array_equal(levels, oracle.bfs(rp, col, 0))

"""Parity at the workloads' full benchmark configurations, against the CPU oracle.

  * Collatz stopping times of n = 1..2^20 (the reference checker over every index,
    examples/cpp/collaz/collaz_hrm.cpp:236-242), both program types;
  * BFS levels of the R-MAT 2^22 graph, edge factor 16, (a, b, c) = (0.57, 0.19, 0.19), seed 1,
    from vertex 0, both program types, against the serial BFS;
  * the photon walk on the 128^3 bench medium (medium seed 2024, walk seed 0x5EED0123456789),
    10^6 photons, both program types (AsyncProgram in three tuning variants), against the OpenMP
    host executor of the same spec.
Every output is compared bit for bit; call counts are compared where they are a pure function
of the inputs (Collatz, photon walk)."""
import numpy as np
import pytest

import oracle

BENCH_SEED = 0x5EED0123456789


@pytest.mark.gpu
@pytest.mark.parametrize("program", ["async", "event"])
def test_collatz_full_config(hrm, program):
    count = 1 << 20
    out, res = hrm.collatz(1, count, program=program)
    ref = oracle.collatz_range(1, count)
    assert np.array_equal(out, ref), f"first mismatch at {np.nonzero(out != ref)[0][:5]}"
    assert res["evals"] == int(ref.astype(np.uint64).sum()) + count == 139_348_407


@pytest.fixture(scope="module")
def rmat22(hrm):
    rp, col = hrm.rmat_csr(22, 16, 0.57, 0.19, 0.19, 1)
    return rp, col, oracle.bfs(rp, col, 0)


@pytest.mark.gpu
@pytest.mark.parametrize("program", ["async", "event"])
def test_bfs_full_config(hrm, rmat22, program):
    rp, col, ref = rmat22
    levels, res = hrm.bfs(rp, col, 0, program=program)
    assert np.array_equal(levels, ref), f"{int((levels != ref).sum())} levels differ"
    assert res["evals"] >= int((ref != 0xFFFFFFFF).sum())


@pytest.fixture(scope="module")
def photon128(hrm):
    mu, ab, sp = hrm.photon_medium(128, 2024)
    count = 1_000_000
    ref, calls = oracle.exec_photon(mu, ab, sp, 128, BENCH_SEED, 0, count, threads=oracle.max_threads())
    return mu, ab, sp, count, ref, calls


@pytest.mark.gpu
@pytest.mark.parametrize("program,variant", [("async", 0), ("event", 0), ("async", 7), ("async", 9)])
def test_photon_bench_medium(hrm, photon128, program, variant):
    """Variant 7 is the tuned one; variant 9's 3-link rings spill and refill links of moves on
    most steps, so every wrapped ring position of the spill and fill paths is exercised."""
    mu, ab, sp, count, ref, calls = photon128
    tally, res = hrm.photon_walk(mu, ab, sp, 128, BENCH_SEED, 0, count, program=program, variant=variant)
    assert np.array_equal(tally, ref), f"{int((tally != ref).sum())} tally slots differ"
    assert res["evals"] == int(calls.sum())
    for f in range(3):
        assert res[f"fn{f}_evals"] == int(calls[f])

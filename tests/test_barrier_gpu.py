"""RemappingBarrier / UnitBarrier on the GPU runtime against the serial barrier oracle.

The workload is Harmonize's barrier demo (examples/cpp/barrier_demo/demo.cpp:20-86): every
count must match exactly, every follow-up must run after its barrier released (violations
= 0), and the unit barrier must fire once, after every non-dependent step.
"""
import numpy as np
import pytest

from oracle.barrier import barrier_demo as oracle_demo


@pytest.mark.gpu
@pytest.mark.parametrize("variant", [0, 1])
@pytest.mark.parametrize("dep,ndep,bar", [(0, 1, 1), (1, 0, 1), (10, 3, 3), (4096, 1024, 7), (65536, 4096, 64),
                                          (100000, 1, 1), (1 << 20, 1 << 18, 1000)])
def test_barrier_demo_matches_oracle(hrm, variant, dep, ndep, bar):
    # Held follow-ups occupy arena links until their barrier releases: size for all of them.
    counter, released, res = hrm.barrier_demo(dep, ndep, bar, variant=variant, arena=max(1 << 18, 2 * dep))
    if dep + ndep <= 70000:
        exp_counter, exp_released = oracle_demo(dep, ndep, bar)
    else:  # the oracle's counts in closed form (the serial loop is slow in Python)
        exp_counter = [2 * dep + ndep + (1 if ndep else 0), ndep, 1 if ndep else 0, 0]
        exp_released = [dep // bar + (1 if dep % bar > b else 0) for b in range(bar)]
    assert counter.tolist() == exp_counter
    assert released[:bar].tolist() == exp_released
    # make_work runs the first Step of every id in place (prog.sync): the runtime's batches
    # evaluate only the follow-ups and the final Step.
    assert res["evals"] == dep + (1 if ndep else 0)


@pytest.mark.gpu
def test_barrier_demo_repeats_identically(hrm):
    a = hrm.barrier_demo(30000, 500, 17)
    b = hrm.barrier_demo(30000, 500, 17)
    assert a[0].tolist() == b[0].tolist() and a[1].tolist() == b[1].tolist()


@pytest.mark.gpu
def test_barrier_demo_rejects_event_program_and_zero_barriers(hrm):
    with pytest.raises(hrm.HarmonizeError):
        hrm.barrier_demo(10, 1, 2, program="event")
    with pytest.raises(hrm.HarmonizeError):
        hrm.barrier_demo(10, 1, 0)


@pytest.mark.gpu
def test_held_promises_of_different_warps_share_links(hrm):
    """2^20 held follow-ups spread over 1000 barriers: the lanes of one warp all await different
    barriers, so one link per warp group would take 2^20 arena links. Packed into each
    barrier's partial link across warps they need about 2^15 (+ one partial per barrier), so
    an arena of 2^16 links is enough and the run is exact."""
    dep, ndep, bar = 1 << 20, 1 << 10, 1000
    counter, released, _ = hrm.barrier_demo(dep, ndep, bar, arena=1 << 16)
    assert counter.tolist() == [2 * dep + ndep + 1, ndep, 1, 0]
    assert released[:bar].tolist() == [dep // bar + (1 if dep % bar > b else 0) for b in range(bar)]

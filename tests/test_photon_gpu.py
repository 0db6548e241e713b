"""Photon walk on the GPU runtime against the CPU oracle: bit-exact uint64 fixed-point tallies
and identical per-run call counts (every call is a pure function of photon id and step)."""
import numpy as np
import pytest

import oracle
from harmonize_b200 import VARIANTS


@pytest.fixture(scope="module")
def medium16(hrm):
    return hrm.photon_medium(16, 11)


@pytest.mark.gpu
@pytest.mark.parametrize("program", ["async", "event"])
@pytest.mark.parametrize("first,count", [(0, 1), (0, 700), (123456, 3000)])
def test_photon_matches_oracle(hrm, medium16, program, first, count):
    mu, ab, sp = medium16
    tally, res = hrm.photon_walk(mu, ab, sp, 16, 0xC0FFEE, first, count, program=program)
    ref, calls = oracle.photon_walk(mu, ab, sp, 16, 0xC0FFEE, first, count)
    assert np.array_equal(tally, ref)
    assert res["evals"] == int(calls.sum())


@pytest.mark.gpu
def test_photon_async_equals_event_large_grid(hrm):
    mu, ab, sp = hrm.photon_medium(64, 5)
    a, ra = hrm.photon_walk(mu, ab, sp, 64, 17, 0, 20000, program="async")
    e, re = hrm.photon_walk(mu, ab, sp, 64, 17, 0, 20000, program="event")
    ref, calls = oracle.photon_walk(mu, ab, sp, 64, 17, 0, 20000)
    assert np.array_equal(a, ref) and np.array_equal(e, ref)
    assert ra["evals"] == re["evals"] == int(calls.sum())


@pytest.mark.gpu
def test_photon_zero_photons(hrm, medium16):
    mu, ab, sp = medium16
    tally, res = hrm.photon_walk(mu, ab, sp, 16, 1, 0, 0)
    assert not tally.any() and res["evals"] == 0


@pytest.mark.gpu
@pytest.mark.parametrize("variant", sorted(VARIANTS))
def test_every_compiled_variant_matches_oracle(hrm, medium16, variant):
    """Every compiled tuning variant (ring links per function, teams per CTA, register caps;
    3-link rings in variant 9) gives the same tallies and call count for all three specs."""
    mu, ab, sp = medium16
    for program in ("async", "event"):
        tally, res = hrm.photon_walk(mu, ab, sp, 16, 0xC0FFEE, 5, 2000, program=program, variant=variant)
        ref, calls = oracle.photon_walk(mu, ab, sp, 16, 0xC0FFEE, 5, 2000)
        assert np.array_equal(tally, ref) and res["evals"] == int(calls.sum())
        steps, _ = hrm.collatz(1, 5000, program=program, variant=variant)
        assert np.array_equal(steps, oracle.collatz_range(1, 5000))
        rp, col = hrm.rmat_csr(12, 8, seed=5)
        levels, _ = hrm.bfs(rp, col, 0, program=program, variant=variant)
        assert np.array_equal(levels, oracle.bfs(rp, col, 0))


@pytest.mark.gpu
def test_release_cache_while_another_thread_runs(hrm):
    """hrm_release_cache drops the cached instances and staging buffers; a whole run in
    progress on another thread keeps what it uses until it ends, and its result is exact."""
    import threading
    import time

    mu, ab, sp = hrm.photon_medium(64, 5)
    got = {}

    def run():
        got["tally"] = hrm.photon_walk(mu, ab, sp, 64, 17, 0, 200000)[0]

    t = threading.Thread(target=run)
    t.start()
    time.sleep(0.003)
    hrm.check(hrm.lib().hrm_release_cache())
    t.join()
    again = hrm.photon_walk(mu, ab, sp, 64, 17, 0, 200000)[0]
    assert np.array_equal(got["tally"], again)

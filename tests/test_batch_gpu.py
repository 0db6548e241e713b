"""Batched jobs in one persistent launch against one plain launch per job and the CPU oracle:
every job's output must be identical bit for bit (Collatz steps, photon tallies, BFS levels)."""
import numpy as np
import pytest

import oracle


@pytest.fixture(scope="module")
def small_mix(hrm):
    from harmonize_b200 import jobs
    specs = jobs.make_mix_specs(45, seed=7, max_photons=3000, max_scale=13, max_collatz=1 << 14)
    return jobs.Mix(specs, photon_grid=16, media=3, seed=7)


@pytest.mark.gpu
@pytest.mark.parametrize("variant,job_order", [(0, 0), (1, 0), (1, 1), (2, 1), (2, 2)])
def test_batch_equals_plain_equals_oracle(hrm, small_mix, variant, job_order):
    from harmonize_b200 import jobs
    mix = small_mix
    done_b, res = jobs.batch_run(mix, which=0, variant=variant, job_order=job_order)
    done_p, total = jobs.plain_run(mix, which=1, streams=4)
    assert (done_b != np.iinfo(np.uint64).max).all()
    for i, s in enumerate(mix.specs):
        a, b = mix.output(0, i), mix.output(1, i)
        assert np.array_equal(a, b), (i, s)
        if s["kind"] == jobs.JOB_COLLATZ:
            assert np.array_equal(a, oracle.collatz_range(s["first"], s["count"]))
        elif s["kind"] == jobs.JOB_BFS:
            _, _, rp, col = mix.graphs[s["scale"]]
            assert np.array_equal(a, oracle.bfs(rp, col, s["root"]))
    # photon jobs against the oracle for a few jobs
    checked = 0
    for i, s in enumerate(mix.specs):
        if s["kind"] == jobs.JOB_PHOTON and checked < 3:
            mu, ab, sp = (t.cpu().numpy() for t in mix.media[s["medium"]])
            ref, _ = oracle.photon_walk(mu, ab, sp, 16, s["seed"], s["first"], s["count"])
            assert np.array_equal(mix.output(0, i), ref)
            checked += 1


@pytest.mark.gpu
def test_batch_subset_and_repeat(hrm, small_mix):
    from harmonize_b200 import jobs
    idx = [0, 1, 2, 9, 10, 11]
    d1, _ = jobs.batch_run(small_mix, which=0, indices=idx)
    first = [small_mix.output(0, i).copy() for i in idx]
    d2, _ = jobs.batch_run(small_mix, which=0, indices=idx)
    for k, i in enumerate(idx):
        assert np.array_equal(first[k], small_mix.output(0, i))


@pytest.mark.gpu
@pytest.mark.parametrize("lanes", [1, 3])
def test_batch_with_solo_large_jobs_equals_plain(hrm, small_mix, lanes):
    """Large photon jobs run through the single-spec runtime (one after another, or over three
    concurrent lanes that share the GPU), the rest in one launch: every output still equals one
    plain launch per job."""
    from harmonize_b200 import jobs
    counts = sorted(s["count"] for s in small_mix.specs if s["kind"] == jobs.JOB_PHOTON)
    threshold = counts[len(counts) // 2]  # about half of the photon jobs run alone
    done, total_ms, res = jobs.batch_run_solo(small_mix, which=0, solo_photons=threshold, job_order=1, lanes=lanes)
    assert total_ms > 0 and res is not None and (done > 0).all()
    jobs.plain_run(small_mix, which=1, streams=4)
    for i, s in enumerate(small_mix.specs):
        assert np.array_equal(small_mix.output(0, i), small_mix.output(1, i)), (i, s)

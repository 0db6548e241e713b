"""Serving: jobs admitted into the resident runtime while it runs. Each job's result must be the
same alone and inside the mix (bit for bit), and the same as one plain launch per job."""
import time

import numpy as np
import pytest


@pytest.fixture(scope="module")
def mix(hrm):
    from harmonize_b200 import jobs
    specs = jobs.make_mix_specs(36, seed=21, max_photons=2000, max_scale=12, max_collatz=1 << 13)
    return jobs.Mix(specs, photon_grid=16, media=2, seed=21)


@pytest.mark.gpu
def test_server_results_same_alone_and_in_mix(hrm, mix):
    from harmonize_b200 import jobs
    n = len(mix.specs)
    # alone: each job in its own session, one at a time (output set 1)
    for i in range(n):
        srv = jobs.Server(1, arena=1 << 16)
        srv.submit(mix.job_array(1, [i]))
        srv.close()
        del srv
    alone = [mix.output(1, i).copy() for i in range(n)]
    # in the mix: all jobs submitted in small groups while the session runs (output set 0)
    srv = jobs.Server(n, arena=1 << 18)
    for g in range(0, n, 5):
        srv.submit(mix.job_array(0, list(range(g, min(n, g + 5)))))
        time.sleep(0.002)
    srv.close()
    done, completed = srv.poll()
    assert completed == n and (done[:n] > 0).all()
    for i in range(n):
        assert np.array_equal(mix.output(0, i), alone[i]), (i, mix.specs[i])


@pytest.mark.gpu
@pytest.mark.parametrize("mode,job_order", [("resident", 0), ("resident", 2), ("runtime", 0), ("plain", 0)])
def test_replay_completes_every_job(hrm, mix, mode, job_order):
    from harmonize_b200 import jobs
    n = len(mix.specs)
    arrivals = jobs.poisson_arrivals(n, rate_per_s=20000.0, seed=3)
    lat, span = jobs.serve_replay(mix, arrivals, mode=mode, which=0, streams=4, arena=1 << 18, job_order=job_order)
    assert (lat > 0).all() and span > 0
    ref = [mix.output(0, i).copy() for i in range(n)]
    jobs.plain_run(mix, which=1, streams=4)
    for i in range(n):
        assert np.array_equal(ref[i], mix.output(1, i))


@pytest.mark.gpu
def test_replay_with_solo_photon_jobs(hrm, mix):
    """Large photon jobs served through the solo lane beside the resident kernel: every job
    completes and every output equals one plain launch per job."""
    from harmonize_b200 import jobs
    n = len(mix.specs)
    counts = sorted(s["count"] for s in mix.specs if s["kind"] == jobs.JOB_PHOTON)
    arrivals = jobs.poisson_arrivals(n, rate_per_s=5000.0, seed=4)
    lat, span = jobs.serve_replay(mix, arrivals, mode="resident", which=0, arena=1 << 18, job_order=2,
                                  solo_photons=counts[len(counts) // 2])
    assert (lat > 0).all() and span > 0
    jobs.plain_run(mix, which=1, streams=4)
    for i, s in enumerate(mix.specs):
        assert np.array_equal(mix.output(0, i), mix.output(1, i)), (i, s)


@pytest.mark.gpu
def test_server_rejects_empty_jobs(hrm, mix):
    from harmonize_b200 import jobs
    arr = mix.job_array(0, [0])
    arr[0].count = 0
    srv = jobs.Server(2, arena=1 << 16)
    with pytest.raises(hrm.HarmonizeError):
        srv.submit(arr)
    srv.close()


@pytest.mark.gpu
@pytest.mark.parametrize("variant", [1, 2])
def test_jobs_complete_while_a_full_exec_runs(hrm, mix, variant):
    """Jobs submitted while the resident exec holds every SM (variant 1 fills each SM's register
    file) complete during that exec: the session clears outputs and publishes jobs with copies
    only, never with a kernel launch that would wait for the exec to end. The exec's cycle budget
    (2^24 scheduling rounds, seconds of polling) is far longer than the bound checked here."""
    from harmonize_b200 import jobs
    small = [i for i, s in enumerate(mix.specs) if s["kind"] != jobs.JOB_PHOTON][:6]
    srv = jobs.Server(len(small), arena=1 << 16, cycles=1 << 24, variant=variant)
    time.sleep(0.05)  # the first exec is on the GPU
    for k, i in enumerate(small):
        t0 = time.perf_counter()
        srv.submit(mix.job_array(0, [i]))
        while srv.poll()[1] < k + 1:
            assert time.perf_counter() - t0 < 1.0, f"job {i} not done within 1 s of its submission"
            time.sleep(0.0005)
    srv.close()
    for i in small:
        s = mix.specs[i]
        out = mix.output(0, i)
        if s["kind"] == jobs.JOB_COLLATZ:
            import oracle
            assert np.array_equal(out, oracle.collatz_range(s["first"], s["count"]))

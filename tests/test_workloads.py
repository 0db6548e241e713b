"""CPU checks that the seeded synthetic job mix has the shapes and distributions of the batched
and serving workload: 4096 instances in equal thirds; Collatz ranges of lognormal length
(median 2^12, sigma 1.5) clipped to [2^6, 2^20]; photon batches of 10^3..10^6 photons,
log-uniform; BFS on R-MAT graphs of 2^12..2^18 vertices."""
import numpy as np

from harmonize_b200 import jobs


def test_job_mix_shapes_and_distributions():
    specs = jobs.make_mix_specs(4096, seed=1)
    kinds = np.array([s["kind"] for s in specs])
    assert [int((kinds == k).sum()) for k in (jobs.JOB_COLLATZ, jobs.JOB_PHOTON, jobs.JOB_BFS)] == [1366, 1365, 1365]
    lengths = np.array([s["count"] for s in specs if s["kind"] == jobs.JOB_COLLATZ])
    assert lengths.min() >= 64 and lengths.max() <= 1 << 20
    assert abs(np.median(np.log2(lengths)) - 12) < 0.2
    inner = np.log(lengths[(lengths > 64) & (lengths < 1 << 20)])
    assert abs(inner.std() - 1.5) < 0.15  # clipping trims the tails a little
    photons = np.array([s["count"] for s in specs if s["kind"] == jobs.JOB_PHOTON])
    assert photons.min() >= 1000 and photons.max() <= 1_000_000
    exps = np.log10(photons)
    assert abs(np.median(exps) - 4.5) < 0.15 and abs(exps.mean() - 4.5) < 0.1
    scales = np.array([s["scale"] for s in specs if s["kind"] == jobs.JOB_BFS])
    assert scales.min() == 12 and scales.max() == 18
    assert all(0 <= s["root"] < 1 << s["scale"] for s in specs if s["kind"] == jobs.JOB_BFS)


def test_job_mix_is_seeded():
    assert jobs.make_mix_specs(300, seed=5) == jobs.make_mix_specs(300, seed=5)
    assert jobs.make_mix_specs(300, seed=5) != jobs.make_mix_specs(300, seed=6)


def test_rmat_graph_shape():
    """R-MAT (a, b, c) = (0.57, 0.19, 0.19): E = 16 * V directed edges, and the skew of the
    recursion puts a heavy share of them on low vertex ids (vertex 0 expects E * (a+b)^scale)."""
    import harmonize_b200 as hrm
    scale = 14
    rp, col = hrm.rmat_csr(scale, 16, 0.57, 0.19, 0.19, 3)
    deg = np.diff(rp.astype(np.int64))
    assert len(col) == 16 << scale and deg.sum() == len(col)
    assert col.max() < 1 << scale
    expected0 = (16 << scale) * (0.57 + 0.19) ** scale
    assert 0.5 * expected0 < deg[0] < 2.0 * expected0
    assert deg.max() > 100 * deg.mean()  # heavy-tailed: far above the mean degree of 16


def test_poisson_arrivals_have_the_requested_rate():
    """Serving arrivals: a seeded Poisson process, non-decreasing, mean gap 1/rate."""
    a = jobs.poisson_arrivals(20000, rate_per_s=500.0, seed=3)
    gaps = np.diff(np.concatenate([[0], a.astype(np.float64)]))
    assert np.all(gaps >= 0)
    assert abs(gaps.mean() / 1e9 - 1 / 500.0) < 0.03 / 500.0
    assert abs(gaps.std() / gaps.mean() - 1.0) < 0.05  # exponential gaps: std = mean
    assert np.array_equal(a, jobs.poisson_arrivals(20000, rate_per_s=500.0, seed=3))

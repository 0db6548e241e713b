"""CPU tests of the oracle: pinned to the reference runtime's own outputs (tests/golden, made by
tests/golden/make_golden.py on a GPU) and to known answers; restatements against the host
executors that run the very same spec sources as the GPU runtime."""
import os

import numpy as np
import pytest

import oracle

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def test_collatz_matches_reference_runtime_output():
    ref = np.load(os.path.join(GOLDEN, "ref_collatz_0_4096.npy"))
    assert np.array_equal(oracle.collatz_range(0, 4096), ref)


def test_collatz_known_answers():
    # Stopping times (OEIS A006577): 27 -> 111, 97 -> 118, 871 -> 178, 837799 -> 524 (the
    # maximum below 10^6); 0 and 1 take no step, as in the reference checker.
    steps = oracle.collatz_range(0, 1 << 20)
    assert steps[0] == 0 and steps[1] == 0 and steps[2] == 1
    assert steps[27] == 111 and steps[97] == 118 and steps[871] == 178
    assert steps[837799] == 524 and steps.max() == 524
    # evaluations of the Even/Odd program over n = 1..2^20: sum of (steps + 1)
    total = int(steps[1:].astype(np.uint64).sum()) + (1 << 20) - 1 + 20 + 1
    assert total == 139_348_407


def test_collatz_executor_equals_restatement():
    out, calls = oracle.exec_collatz(1000, 50000, threads=3)
    ref = oracle.collatz_range(1000, 50000)
    assert np.array_equal(out, ref)
    assert int(calls.sum()) == int(ref.astype(np.uint64).sum()) + 50000


def test_philox_known_answers():
    # Known-answer vectors of Philox-4x32-10 (Salmon et al., SC'11; Random123 distribution).
    assert [hex(x) for x in oracle.philox([0, 0, 0, 0], [0, 0])] == \
        ["0x6627e8d5", "0xe169c58d", "0xbc57ac4c", "0x9b00dbd8"]
    assert [hex(x) for x in oracle.philox([0xFFFFFFFF] * 4, [0xFFFFFFFF] * 2)] == \
        ["0x408f276d", "0x41c83b0e", "0xa20bc7c6", "0x6d5451fd"]
    assert [hex(x) for x in oracle.philox([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344],
                                          [0xA4093822, 0x299F31D0])] == \
        ["0xd16cfe09", "0x94fdcceb", "0x5001e420", "0x24126ea1"]


def test_log_accuracy():
    rng = np.random.default_rng(3)
    xs = np.concatenate([rng.random(4000).astype(np.float32) + np.float32(2 ** -24),
                         np.float32(2.0) ** rng.integers(-24, 1, 200).astype(np.float32)])
    for x in xs:
        got = oracle.log(float(x))
        exact = float(np.log(np.float64(x)))
        ulp = float(np.spacing(np.float32(abs(exact)))) if exact != 0 else 1e-45
        assert abs(got - exact) <= 4 * ulp + 1e-7 * abs(exact)


def _medium16():
    m = np.load(os.path.join(GOLDEN, "medium_n16_seed11.npz"))
    return m["mu"], m["ab"], m["sp"]


def test_photon_restatement_matches_reference_runtime_output():
    mu, ab, sp = _medium16()
    ref = np.load(os.path.join(GOLDEN, "ref_photon_n16_s99_500.npy"))
    tally, _ = oracle.photon_walk(mu, ab, sp, 16, 99, 0, 500)
    assert np.array_equal(tally, ref)


@pytest.mark.parametrize("threads", [1, 4])
def test_photon_executor_equals_restatement(threads):
    mu, ab, sp = _medium16()
    a, ca = oracle.photon_walk(mu, ab, sp, 16, 0xC0FFEE, 77, 400)
    b, cb = oracle.exec_photon(mu, ab, sp, 16, 0xC0FFEE, 77, 400, threads=threads)
    assert np.array_equal(a, b)
    assert np.array_equal(ca, cb)


def test_photon_weight_conservation():
    mu, ab, sp = _medium16()
    n, count = 16, 1000
    t, _ = oracle.photon_walk(mu, ab, sp, n, 5, 0, count)
    v = n ** 3
    S = oracle.PHOTON_SPREAD
    total = int(t[:v].sum()) + int(t[v:v + S].sum()) + int(t[v + S:v + 2 * S].sum()) - int(t[v + 2 * S:].sum())
    assert abs(total / 2 ** 32 - count) / count < 1e-5


def test_bfs_restatement_matches_reference_runtime_output():
    g = np.load(os.path.join(GOLDEN, "ref_bfs_rmat10.npz"))
    assert np.array_equal(oracle.bfs(g["rowptr"], g["col"], 0), g["levels"])


@pytest.mark.parametrize("threads", [1, 4])
def test_bfs_executor_equals_restatement(threads):
    g = np.load(os.path.join(GOLDEN, "ref_bfs_rmat10.npz"))
    lv, _ = oracle.exec_bfs(g["rowptr"], g["col"], 5, threads=threads)
    assert np.array_equal(lv, oracle.bfs(g["rowptr"], g["col"], 5))


def test_bfs_edge_cases():
    # empty graph, isolated root, self loops and duplicate edges
    rp = np.array([0, 0, 0], dtype=np.uint32)
    assert list(oracle.bfs(rp, np.zeros(0, np.uint32), 1)) == [0xFFFFFFFF, 0]
    rp = np.array([0, 3, 4, 4], dtype=np.uint32)
    col = np.array([0, 1, 1, 2], dtype=np.uint32)
    assert list(oracle.bfs(rp, col, 0)) == [0, 1, 2]
    lv, _ = oracle.exec_bfs(rp, col, 0)
    assert list(lv) == [0, 1, 2]


def test_barrier_oracle_counts():
    from oracle.barrier import barrier_demo
    for dep, ndep, bar in [(0, 1, 1), (10, 3, 3), (1000, 17, 7), (5, 0, 9)]:
        counter, released = barrier_demo(dep, ndep, bar)
        # demo.cpp:216 expects dep*2 + ndep Steps; the unit barrier adds one final Step.
        assert counter == [2 * dep + ndep + (1 if ndep else 0), ndep, 1 if ndep else 0, 0]
        assert released == [dep // bar + (1 if dep % bar > b else 0) for b in range(bar)]
        assert sum(released) == dep


@pytest.mark.parametrize("n,seed", [(16, 11), (32, 7), (128, 2024)])
def test_oracle_medium_equals_product_medium(hrm, n, seed):
    """The oracle's restated medium generator gives the same bytes as the product's
    hrm_photon_medium (the reference arm and the golden script use the oracle's, so that they
    never load the product library)."""
    a = oracle.photon_medium(n, seed)
    b = hrm.photon_medium(n, seed)
    for x, y in zip(a, b):
        assert x.dtype == y.dtype and np.array_equal(x.view(np.uint8), y.view(np.uint8))


def test_golden_medium_fixture_is_the_seeded_medium():
    mu, ab, sp = _medium16()
    gm, ga, gs = oracle.photon_medium(16, 11)
    assert np.array_equal(mu, gm) and np.array_equal(ab, ga) and np.array_equal(sp, gs)


@pytest.mark.parametrize("scale,ef,seed", [(10, 16, 5), (16, 16, 1), (12, 8, 5)])
def test_oracle_rmat_equals_product_rmat(hrm, scale, ef, seed):
    a = oracle.rmat_csr(scale, ef, seed=seed)
    b = hrm.rmat_csr(scale, ef, seed=seed)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


def test_golden_rmat_fixture_is_the_seeded_graph():
    g = np.load(os.path.join(GOLDEN, "ref_bfs_rmat10.npz"))
    rp, col = oracle.rmat_csr(10, 16, seed=5)
    assert np.array_equal(g["rowptr"], rp) and np.array_equal(g["col"], col)


def _sha256(a):
    import hashlib
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def test_collatz_full_range_matches_reference_runtime_digest():
    """n = 1..2^20, the Collatz benchmark range: the reference AsyncProgram's stopping times
    (digest in tests/golden/ref_collatz_1_2p20.json) equal the restated checker's."""
    import json
    g = json.load(open(os.path.join(GOLDEN, "ref_collatz_1_2p20.json")))
    steps = oracle.collatz_range(g["start"], g["count"])
    assert int(steps.astype(np.uint64).sum()) == g["sum"] and int(steps.max()) == g["max"]
    assert _sha256(steps.astype(np.uint32)) == g["sha256"]


def test_photon_bench_medium_matches_reference_runtime_digest():
    """10^4 photons of the bench walk (128^3 medium, seed 2024; walk seed 0x5EED0123456789)
    through the reference EventProgram: the restated walk gives the same tallies, byte for byte."""
    import json
    g = json.load(open(os.path.join(GOLDEN, "ref_photon_n128_1e4.json")))
    mu, ab, sp = oracle.photon_medium(g["n"], g["medium_seed"])
    t, _ = oracle.photon_walk(mu, ab, sp, g["n"], g["seed"], g["first"], g["count"])
    v, s = g["n"] ** 3, oracle.PHOTON_SPREAD
    assert int(np.count_nonzero(t)) == g["nonzero"]
    assert int(t[:v].astype(object).sum()) == g["voxels"]
    assert int(t[v + s:v + 2 * s].astype(object).sum()) == g["killed"]
    assert int(t[v + 2 * s:].astype(object).sum()) == g["gained"]
    assert _sha256(t) == g["sha256"]


def test_bfs_rmat16_matches_reference_runtime_output():
    g = np.load(os.path.join(GOLDEN, "ref_bfs_rmat16_levels.npz"))
    rp, col = oracle.rmat_csr(int(g["scale"]), int(g["edge_factor"]), seed=int(g["seed"]))
    assert np.array_equal(oracle.bfs(rp, col, int(g["root"])), g["levels"])

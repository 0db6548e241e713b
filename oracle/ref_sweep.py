"""Sweeps the launch shape of the ORIGINAL Harmonize EventProgram on the photon walk (BENCH
INFRASTRUCTURE ONLY), so that the reference arm times its best configuration.

Parameters, each over the values below, by coordinate descent from the examples' defaults
(one parameter at a time, the others held at the best so far):
  wg          work groups of one warp per launch (exec<P>(inst, wg, chunk))
  chunk       promises per lane per grab, the third argument of EventProgram::exec (event.h:383)
  io          io_size: promises per function per buffer side (EventProgram::Instance)
  load_limit  the spec's make_work throttle: no new photons while the move buffer's fill
              fraction (load_fraction, event.h:540-544) is above it
Every run walks the same photons on the 128^3 bench medium and is checked bit for bit against
the CPU oracle; time = CUDA events around init + the exec loop (oracle/ref_glue.cu).

    python -m oracle.ref_sweep [--photons N] [--grid G]
Prints one JSON line per run and a final line with the best shape.
"""
import argparse
import json
import time

import numpy as np

BENCH_SEED = 0x5EED0123456789
# Only shapes whose runs ended are swept. Left out: chunk 8 (twice a run of the reference
# EventProgram with chunk 8 on this workload did not end; the sweeps were stopped by their time
# limits after about 15 and 25 minutes) and any io size other than 2^24 (a run with io 2^23 did
# not end within 14 minutes either), while the shapes below end in about a second. The
# load_limit throttle therefore stays at 1/64 of io as well (it scales with io).
SPACE = {
    "wg": [148 * 8, 148 * 12, 148 * 16, 148 * 24, 148 * 32, 148 * 48, 148 * 64],
    "chunk": [1, 2, 4],
    "io": [1 << 24],
    "load_limit": [1.0 / 64],
}
# The examples' shape was the start of the first sweeps (148 * 12 groups, chunk 1, io 2^24,
# 1/64); the best of those (148 * 32 groups, chunk 4) starts this one.
START = {"wg": 148 * 32, "chunk": 4, "io": 1 << 24, "load_limit": 1.0 / 64}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--photons", type=int, default=1_000_000)
    ap.add_argument("--grid", type=int, default=128)
    ap.add_argument("--passes", type=int, default=1)
    ap.add_argument("--max-execs", type=int, default=4000,
                    help="give up on a shape after this many execs (the examples' shape needs about 1,400 on "
                         "10^6 photons; a shape whose buffers overflow never completes)")
    a = ap.parse_args()
    import torch
    import oracle
    n, count = a.grid, a.photons
    mu, ab, sp = oracle.photon_medium(n, 2024)
    t0 = time.perf_counter()
    ref, calls = oracle.exec_photon(mu, ab, sp, n, BENCH_SEED, 0, count, threads=oracle.max_threads())
    print(json.dumps({"oracle_s": round(time.perf_counter() - t0, 2), "calls": int(calls.sum())}), flush=True)
    calls = int(calls.sum())
    d_mu, d_ab, d_sp = (torch.from_numpy(x).cuda() for x in (mu, ab, sp))
    d_t = torch.zeros(n ** 3 + 3 * 1024, dtype=torch.int64, device="cuda")
    seen = {}

    def run(shape):
        key = tuple(sorted(shape.items()))
        if key in seen:
            return seen[key]
        try:
            r = oracle.ref_photon_device(d_mu.data_ptr(), d_ab.data_ptr(), d_sp.data_ptr(), n, BENCH_SEED, 0, count,
                                         d_t.data_ptr(), wg=shape["wg"], nn=shape["chunk"], arena=shape["io"],
                                         load_limit=shape["load_limit"], max_execs=a.max_execs)
            ok = np.array_equal(d_t.cpu().numpy().view(np.uint64), ref)
            ms = r["ms"] if ok else float("inf")
            row = dict(shape, ms=round(r["ms"], 2), execs=r["execs"], calls_per_s=calls / (r["ms"] / 1e3),
                       output="exact" if ok else "differs")
        except RuntimeError as e:
            ms = float("inf")
            row = dict(shape, error=str(e)[:200])
        print(json.dumps(row), flush=True)
        seen[key] = ms
        return ms

    best = dict(START)
    best_ms = run(best)
    for _ in range(a.passes):
        for p, values in SPACE.items():
            for v in values:
                cand = dict(best, **{p: v})
                ms = run(cand)
                if ms < best_ms:
                    best, best_ms = cand, ms
    print(json.dumps({"best": best, "ms": round(best_ms, 2), "calls": calls,
                      "calls_per_s": calls / (best_ms / 1e3), "photons": count, "grid": n}), flush=True)


if __name__ == "__main__":
    main()

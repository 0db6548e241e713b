"""Reference arm of bench.py (`--impl reference`) — bench infrastructure only.

Times the ORIGINAL Harmonize runtime (oracle/_ref/libhrm_ref.so: the reference's headers
compiled with the same spec sources) on the bench's workload, configuration and metric (async
calls/s). Harmonize has no CPU implementation of this path; its implementation is this CUDA
runtime. This process loads only oracle/ libraries (inputs come from the oracle's own
generators), never the product library.

  * photon walk: the full workload of the bench line (10^7 photons on the 128^3 medium by
    default), on the reference EventProgram with the launch shape its sweep found best
    (oracle.REF_PHOTON_SHAPE, profiles/reference_eventprogram_photon_sweep.txt). Its
    AsyncProgram raised an illegal memory access on this spec
    (profiles/reference_asyncprogram_photon_fault.txt) and is not run again. The call count of
    a photon set is a pure function of the photon ids (from the CPU oracle); the tallies of
    the warm-up run are checked bit for bit against the OpenMP host executor, whose run is
    also the CPU baseline of the line;
  * collatz: the reference AsyncProgram on n = 1..2^20 (139,348,407 calls).
Under torchrun only rank 0 runs; other ranks exit without work.
"""
import json
import os
import time

import numpy as np


def _line(args, value, ms_steps, config, cpu, dtype, extra=None):
    line = {
        "impl": "reference", "metric": "async calls/s", "value": round(value, 1), "unit": "calls/s",
        "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(sum(ms_steps) / max(1, len(ms_steps)), 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": dtype, "data": "synthetic",
        "config": config, "cpu_baseline": cpu,
        "e2e": {"value": round(value, 1), "unit": "calls/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    if extra:
        line.update(extra)
    return line


def main(args, config):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import torch
    import oracle
    try:
        oracle.ref_load()
    except Exception as e:
        print(json.dumps({"impl": "reference", "unavailable": f"reference CUDA build missing: {e}"}))
        return
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    threads = oracle.max_threads()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    if args.workload == "photon":
        n, count = args.grid, args.photons
        seed = 0x5EED0123456789
        mu, ab, sp = oracle.photon_medium(n, 2024)
        d_mu, d_ab, d_sp = (torch.from_numpy(x).cuda() for x in (mu, ab, sp))
        d_t = torch.zeros(n ** 3 + 3 * 1024, dtype=torch.int64, device="cuda")
        shape = dict(oracle.REF_PHOTON_SHAPE)

        def step():
            flush.zero_()
            torch.cuda.synchronize()
            return oracle.ref_photon_device(d_mu.data_ptr(), d_ab.data_ptr(), d_sp.data_ptr(), n, seed, 0, count,
                                            d_t.data_ptr(), program="event")["ms"]

        for _ in range(max(args.warmup, 1)):
            step()
        got = d_t.cpu().numpy().view(np.uint64).copy()
        t0 = time.perf_counter()
        ref_t, calls = oracle.exec_photon(mu, ab, sp, n, seed, 0, count, threads=threads)
        cpu_s = time.perf_counter() - t0
        if not np.array_equal(got, ref_t):
            raise SystemExit("reference runtime: tallies differ from the oracle")
        calls = int(calls.sum())
        ms = [step() for _ in range(args.steps)]
        value = calls * len(ms) / (sum(ms) / 1e3)
        cpu = {"value": calls / cpu_s, "unit": "calls/s", "cores": threads, "kind": "port",
               "sample": f"the whole workload ({count} photons), OpenMP host executor of the same spec source "
                         f"({calls} calls in {cpu_s:.1f} s)"}
        extra = {"calls_per_step": calls, "oracle_check": "exact",
                 "reference_program": {"program": "EventProgram (its AsyncProgram faulted on this spec)",
                                       "work_groups": shape["wg"], "chunk": shape["chunk"], "io_size": shape["io"],
                                       "load_limit": shape["load_limit"]}}
        print(json.dumps(_line(args, value, ms, config, cpu, "f32", extra)), flush=True)
    elif args.workload == "collatz":
        count = 1 << 20

        def step():
            flush.zero_()
            torch.cuda.synchronize()
            out, r = oracle.ref_collatz(1, count, program="async")
            return out, r["ms"]

        for _ in range(max(args.warmup, 0)):
            step()
        ref = oracle.collatz_range(1, count)
        calls = int(ref.astype(np.uint64).sum()) + count
        ms = []
        for _ in range(args.steps):
            out, m = step()
            if not np.array_equal(out, ref):
                raise SystemExit("reference runtime: collatz output differs from the oracle")
            ms.append(m)
        value = calls * len(ms) / (sum(ms) / 1e3)
        t0 = time.perf_counter()
        _, c = oracle.exec_collatz(1, count, threads=threads)
        cpu = {"value": float(c.sum()) / (time.perf_counter() - t0), "unit": "calls/s", "cores": threads,
               "kind": "port", "sample": "n = 1..2^20, OpenMP host executor"}
        extra = {"oracle_check": "exact",
                 "reference_program": {"program": "AsyncProgram", "work_groups": oracle.REF_WG,
                                       "cycles": oracle.REF_CYCLES}}
        print(json.dumps(_line(args, value, ms, config, cpu, "u64", extra)), flush=True)
    else:
        print(json.dumps({"impl": "reference", "unavailable":
                          "BFS call counts depend on the schedule and the reference runtime has no call counter; "
                          "its EventProgram time to solution is compared by oracle/compare_runtimes.py"}))

"""Reference arm of bench.py (`--impl reference`) — bench infrastructure only.

Times the ORIGINAL Harmonize runtime (oracle/_ref/libhrm_ref.so: the reference's headers
compiled with the same spec sources) on the bench's workload and metric, async calls/s.
Harmonize has no CPU implementation of this path; its implementation is this CUDA runtime.

  * photon walk: the reference EventProgram (its AsyncProgram raised an illegal memory access
    on this spec — profiles/reference_asyncprogram_photon_fault.txt — and is not run again),
    on a bounded sample of 10^6 photons of the same 128^3 medium per step; the number of
    calls of a photon set is a pure function of the photon ids, taken from the CPU oracle;
  * collatz: the reference AsyncProgram on n = 1..2^20 (139,348,407 calls).
Under torchrun only rank 0 runs; other ranks exit without work. The line also carries the
CPU baseline (OpenMP host executor of the same spec source).
"""
import json
import os
import time

import numpy as np


def _line(args, value, ms_steps, config, cpu, extra=None):
    line = {
        "impl": "reference", "metric": "async calls/s", "value": round(value, 1), "unit": "calls/s",
        "n_gpus": int(os.environ.get("WORLD_SIZE", "1")), "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(sum(ms_steps) / max(1, len(ms_steps)), 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": config.pop("dtype"), "data": "synthetic",
        "config": config, "cpu_baseline": cpu,
        "e2e": {"value": round(value, 1), "unit": "calls/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    if extra:
        line.update(extra)
    return line


def main(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import torch
    import harmonize_b200 as hrm
    import oracle
    try:
        oracle.ref_load()
    except Exception as e:
        print(json.dumps({"impl": "reference", "unavailable": f"reference CUDA build missing: {e}"}))
        return
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    threads = oracle.max_threads()
    if args.workload == "photon":
        n = args.grid
        sample = min(args.photons, 1_000_000)
        seed = 0x5EED0123456789
        mu, ab, sp = hrm.photon_medium(n, 2024)
        d_mu, d_ab, d_sp = (torch.from_numpy(x).cuda() for x in (mu, ab, sp))
        d_t = torch.zeros(n ** 3 + 3 * 1024, dtype=torch.int64, device="cuda")
        t0 = time.perf_counter()
        ref_t, calls = oracle.exec_photon(mu, ab, sp, n, seed, 0, sample, threads=threads)
        cpu_s = time.perf_counter() - t0
        calls = int(calls.sum())

        def step():
            r = oracle.ref_photon_device(d_mu.data_ptr(), d_ab.data_ptr(), d_sp.data_ptr(), n, seed, 0, sample,
                                         d_t.data_ptr(), program="event")
            return r["ms"]

        for _ in range(max(args.warmup, 0)):
            step()
        if not np.array_equal(d_t.cpu().numpy().view(np.uint64), ref_t):
            raise SystemExit("reference runtime: tallies differ from the oracle")
        ms = [step() for _ in range(args.steps)]
        value = calls * len(ms) / (sum(ms) / 1e3)
        cpu = {"value": calls / cpu_s, "unit": "calls/s", "cores": threads, "kind": "port",
               "sample": f"{sample} photons, OpenMP host executor of the same spec source"}
        config = {"workload": f"photon_walk_{args.photons:.0e}_photons_{n}^3",
                  "sample_per_step": f"{sample} photons of the workload",
                  "reference_program": "EventProgram (reference AsyncProgram faults on this spec)",
                  "chunk": 1, "work_groups": oracle.REF_WG, "dtype": "f32"}
        print(json.dumps(_line(args, value, ms, config, cpu, {"calls_per_step": calls})), flush=True)
    elif args.workload == "collatz":
        count = 1 << 20

        def step():
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
        config = {"workload": "collatz_1_to_2^20", "reference_program": "AsyncProgram",
                  "work_groups": oracle.REF_WG, "cycles": oracle.REF_CYCLES, "dtype": "u64"}
        print(json.dumps(_line(args, value, ms, config, cpu)), flush=True)
    else:
        print(json.dumps({"impl": "reference", "unavailable":
                          "reference AsyncProgram faulted on multi-call specs; BFS reference timing is "
                          "reported separately with the reference EventProgram"}))

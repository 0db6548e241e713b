"""Times this runtime against the ORIGINAL Harmonize runtime on the built-in workloads.

    python -m oracle.compare_runtimes [--photons N] [--scale S] [--reps R]
                                      [--only collatz,photon,bfs] [--programs async,event]
                                      [--runtimes b200,reference]

(--only / --programs / --runtimes restrict the run, e.g. to one kernel under a profiler.)

Both runtimes run the same spec sources on the same device-resident inputs; every output is
checked (Collatz steps and photon tallies bit-exact against the CPU oracle; BFS levels against
the serial BFS). Timing: CUDA events around init + the exec loop, best of R runs, inputs
resident. Calls: Collatz and photon call counts are pure functions of the inputs (oracle);
BFS relaxations depend on the schedule, so BFS is compared by time to solution.
The reference AsyncProgram runs only Collatz: it raised an illegal memory access on the
photon spec (profiles/reference_asyncprogram_photon_fault.txt).
Prints one JSON object per measurement and a table.
"""
import argparse
import ctypes
import json

import numpy as np


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--photons", type=int, default=1_000_000)
    ap.add_argument("--scale", type=int, default=22)
    ap.add_argument("--reps", type=int, default=2)
    ap.add_argument("--only", default="collatz,photon,bfs")
    ap.add_argument("--programs", default="async,event")
    ap.add_argument("--runtimes", default="b200,reference")
    a = ap.parse_args()
    only, programs, runtimes = (set(x.split(",")) for x in (a.only, a.programs, a.runtimes))
    import torch
    import harmonize_b200 as hrm
    from harmonize_b200.autotune import tuned_variant
    import oracle

    rows = []

    def record(workload, runtime, program, ms, calls, ok, note=""):
        r = {"workload": workload, "runtime": runtime, "program": program, "ms": round(ms, 3),
             "calls": calls, "calls_per_s": (calls / (ms / 1e3)) if calls else None, "output_ok": bool(ok),
             "note": note}
        rows.append(r)
        print(json.dumps(r), flush=True)

    # ---- Collatz n = 1..2^20 --------------------------------------------------------------
    N = 1 << 20
    ref_steps = oracle.collatz_range(1, N)
    calls = int(ref_steps.astype(np.uint64).sum()) + N
    d_out = torch.empty(N, dtype=torch.int32, device="cuda")
    for prog in ("async", "event"):
        if "collatz" not in only or prog not in programs:
            continue
        if "b200" in runtimes:
            best = 1e30
            for _ in range(a.reps + 1):
                cfg = hrm.make_config(prog, variant=tuned_variant("collatz", prog))
                res = hrm.RunResult()
                hrm.check(hrm.lib().hrm_collatz_run_device(1, N, d_out.data_ptr(), ctypes.byref(cfg),
                                                           ctypes.byref(res)))
                best = min(best, res.device_ms)
            ok = np.array_equal(d_out.cpu().numpy().view(np.uint32), ref_steps)
            record("collatz_2^20", "b200", prog, best, calls, ok)
        if "reference" in runtimes:
            best = 1e30
            for _ in range(a.reps + 1):
                out, r = oracle.ref_collatz(1, N, program=prog)
                best = min(best, r["ms"])
            record("collatz_2^20", "reference", prog, best, calls, np.array_equal(out, ref_steps))

    if "photon" in only:
        run_photon(a, hrm, oracle, torch, tuned_variant, record, programs, runtimes)
    if "bfs" in only:
        run_bfs(a, hrm, oracle, torch, tuned_variant, record, programs, runtimes)

    print("\n| workload | runtime | program | ms | calls/s | output |")
    print("|---|---|---|---|---|---|")
    for r in rows:
        cps = f"{r['calls_per_s']:.3e}" if r["calls_per_s"] else "-"
        print(f"| {r['workload']} | {r['runtime']} | {r['program']} | {r['ms']} | {cps} | "
              f"{'exact' if r['output_ok'] else r['note'] or 'MISMATCH'} |")


def run_photon(a, hrm, oracle, torch, tuned_variant, record, programs, runtimes):
    n, seed, P = 128, 0x5EED0123456789, a.photons
    mu, ab, sp = hrm.photon_medium(n, 2024)
    ref_t, c = oracle.exec_photon(mu, ab, sp, n, seed, 0, P, threads=oracle.max_threads())
    calls = int(c.sum())
    d_mu, d_ab, d_sp = (torch.from_numpy(x).cuda() for x in (mu, ab, sp))
    d_t = torch.zeros(n ** 3 + 3 * 1024, dtype=torch.int64, device="cuda")
    for prog in ("async", "event"):
        if prog not in programs or "b200" not in runtimes:
            continue
        best = 1e30
        for _ in range(a.reps + 1):
            cfg = hrm.make_config(prog, variant=tuned_variant("photon", prog))
            res = hrm.RunResult()
            hrm.check(hrm.lib().hrm_photon_run_device(d_mu.data_ptr(), d_ab.data_ptr(), d_sp.data_ptr(), n, seed, 0,
                                                      P, d_t.data_ptr(), ctypes.byref(cfg), ctypes.byref(res)))
            best = min(best, res.device_ms)
        ok = np.array_equal(d_t.cpu().numpy().view(np.uint64), ref_t)
        record(f"photon_{P}_128^3", "b200", prog, best, calls, ok)
    if "reference" not in runtimes:
        return
    if "event" in programs:
        best = 1e30
        for _ in range(a.reps + 1):
            r = oracle.ref_photon_device(d_mu.data_ptr(), d_ab.data_ptr(), d_sp.data_ptr(), n, seed, 0, P,
                                         d_t.data_ptr(), program="event")
            best = min(best, r["ms"])
        record(f"photon_{P}_128^3", "reference", "event", best, calls,
               np.array_equal(d_t.cpu().numpy().view(np.uint64), ref_t))
    if "async" in programs:
        record(f"photon_{P}_128^3", "reference", "async", 0.0, 0, False,
               "not run: the reference AsyncProgram faulted on this spec")


def run_bfs(a, hrm, oracle, torch, tuned_variant, record, programs, runtimes):
    rp, col = hrm.rmat_csr(a.scale, 16, 0.57, 0.19, 0.19, 1)
    nv = len(rp) - 1
    ref_lv = oracle.bfs(rp, col, 0)
    d_rp = torch.from_numpy(rp.view(np.int32)).cuda()
    d_col = torch.from_numpy(col.view(np.int32)).cuda()
    d_lv = torch.empty(nv, dtype=torch.int32, device="cuda")
    for prog in ("async", "event"):
        if prog not in programs or "b200" not in runtimes:
            continue
        best, ev = 1e30, 0
        for _ in range(a.reps + 1):
            cfg = hrm.make_config(prog, variant=tuned_variant("bfs", prog))
            res = hrm.RunResult()
            hrm.check(hrm.lib().hrm_bfs_run_device(d_rp.data_ptr(), d_col.data_ptr(), nv, 0, d_lv.data_ptr(),
                                                   ctypes.byref(cfg), ctypes.byref(res)))
            if res.device_ms < best:
                best, ev = res.device_ms, int(res.stats[0])
        ok = np.array_equal(d_lv.cpu().numpy().view(np.uint32), ref_lv)
        record(f"rmat_bfs_2^{a.scale}", "b200", prog, best, ev, ok, "calls = this run's relaxations + expansions")
    if "reference" in runtimes and "event" in programs:
        best = 1e30
        for _ in range(a.reps + 1):
            r = oracle.ref_bfs_device(d_rp.data_ptr(), d_col.data_ptr(), nv, 0, d_lv.data_ptr(), program="event")
            best = min(best, r["ms"])
        record(f"rmat_bfs_2^{a.scale}", "reference", "event", best, 0,
               np.array_equal(d_lv.cpu().numpy().view(np.uint32), ref_lv), "time to solution only")


if __name__ == "__main__":
    main()

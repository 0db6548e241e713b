"""Benchmark of the B200-native Harmonize runtime (one JSON line on stdout, rank 0).

Default workload: the Monte Carlo photon walk — 10^7 photons of weight 1 launched at the
centre of a 128^3 grid of unit voxels (seeded synthetic medium), AsyncProgram. One step is
one complete run of that batch through the runtime's C ABI. Metric: async calls/s (one
call = one eval), whole job.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload photon|bfs|collatz] [--program async|event]

value : calls / device time with inputs resident in HBM (hrm_*_run_device), CUDA events on
        the launching (default) stream, L2 flushed before every step (untimed).
e2e   : the same metric through the host-buffer entry point (hrm_*_run): input upload and
        result download inside the timed region, pinned host memory.
--gpus N under torchrun: one independent replica per GPU (the walk has no cross-replica
exchange), photon ids offset per rank (weak scaling); time = max over ranks.
--impl reference: the reference runtime (Harmonize's own runtime built from its headers with
the same spec source into oracle/_ref: its EventProgram for the photon walk, on which its
AsyncProgram faulted, at the launch shape its sweep found best) on the same workload, config
and metric; that process loads only oracle/ libraries.
After the timed steps, rank 0 checks the last run's output against the CPU oracle over the
whole workload ("oracle_check": "exact", or the bench fails); that oracle run (OpenMP host
executor of the same spec source) is the line's cpu_baseline.
--workload batched / serving: the job mix in the persistent runtime against one single-spec
runtime run per job and one plain kernel per job (see run_batched / run_serving).
"""
import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

PEAKS_FALLBACK = {"hbm_gbs": 6650.0}
JOB_ORDERS = {"round-robin": 0, "admission": 1, "small-first": 2}  # HRM_JOB_ORDER_*


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--workload", default="photon", choices=["photon", "bfs", "collatz", "batched", "serving"])
    p.add_argument("--jobs", type=int, default=4096, help="batched: number of job instances")
    p.add_argument("--serve-jobs", type=int, default=512, help="serving: jobs per arrival-rate point")
    p.add_argument("--rates", type=float, nargs="+", default=[0.1, 0.25, 0.5, 0.75, 0.9, 1.0, 1.25],
                   help="serving: arrival rates as fractions of the batched throughput")
    p.add_argument("--program", default="async", choices=["async", "event"])
    p.add_argument("--photons", type=int, default=10_000_000)
    p.add_argument("--grid", type=int, default=128)
    p.add_argument("--scale", type=int, default=22)
    p.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    p.add_argument("--variant", type=int, default=-1, help="compiled tuning variant (-1 = autotuned)")
    p.add_argument("--job-order", default="small-first", choices=list(JOB_ORDERS),
                   help="batched/serving: which job make_work serves (HRM_JOB_ORDER_*)")
    p.add_argument("--solo-photons", type=int, default=1 << 15,
                   help="batched: photon jobs at least this large also run alone (the persistent_solo arm)")
    p.add_argument("--solo-lanes", type=int, default=3,
                   help="batched: concurrent lanes of the persistent_solo arm's large jobs (1..8; 3 from a sweep "
                        "of 1..4 on the 4096-job mix)")
    p.add_argument("--serve-solo-photons", type=int, default=1 << 13,
                   help="serving: photon jobs at least this large run through the solo lane (0 = never); "
                        "2^13 from a sweep of 2^13..2^17 (lowest p50 at every load and p99 at 1.0+)")
    return p.parse_args()


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return {"hbm_gbs": float(d["hbm_gbs"]), "source": "measured"}
    except Exception:
        return {"hbm_gbs": PEAKS_FALLBACK["hbm_gbs"], "source": "fallback"}


class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        self.lines = []
        if self.proc is not None:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except Exception:
                self.proc.kill()
                out = ""
            self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in getattr(self, "lines", []):
            f = [x.strip() for x in l.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup(args):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    import torch
    torch.cuda.set_device(local)
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        pg = dist
    return rank, world, local, pg


def _reduce_device(pg):
    """Device of the reduction tensors: the GPU under NCCL, the CPU under gloo."""
    return "cpu" if pg.get_backend() == "gloo" else "cuda"


def barrier(pg):
    import torch
    if pg is not None:
        pg.barrier()
    if torch.cuda.is_available():
        torch.cuda.synchronize()


def max_over_ranks(pg, value):
    import torch
    if pg is None:
        return value
    t = torch.tensor([value], dtype=torch.float64, device=_reduce_device(pg))
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(pg, value):
    import torch
    if pg is None:
        return value
    t = torch.tensor([float(value)], dtype=torch.float64, device=_reduce_device(pg))
    pg.all_reduce(t, op=pg.ReduceOp.SUM)
    return float(t.item())


def replica_range(rank, count):
    """Replicas only: rank r works on ids [r*count, (r+1)*count) (weak scaling, no exchange)."""
    return rank * count, count


def workload_config(args, world):
    """The workload of the bench line, shared by both arms (the reference arm reports the same
    dict): what is run, not how."""
    l2 = "flushed before every step (256 MiB write)"
    if args.workload == "photon":
        return {"workload": f"photon_walk_{args.photons:.0e}_photons_{args.grid}^3", "photons_per_gpu": args.photons,
                "grid": args.grid, "l2": l2,
                "medium": "seeded synthetic: mu_s~lognormal(0,0.5), absorb~U[0.02,0.2], split p=0.1 (seed 2024)",
                "parallelism": f"replicas x{world}"}
    if args.workload == "bfs":
        return {"workload": f"rmat_bfs_2^{args.scale}_ef16", "vertices": 1 << args.scale,
                "edges": 16 << args.scale, "root": 0, "l2": l2, "parallelism": f"replicas x{world}"}
    return {"workload": "collatz_1_to_2^20", "starts": 1 << 20, "l2": l2, "parallelism": f"replicas x{world}"}


def flush_l2(buf):
    buf.zero_()  # 256 MiB > the 126 MB L2


# ---------------------------------------------------------------------------------------
# Algorithmic bytes per call (roofline accounting). A queued promise is written once and
# read once; each function then touches its compulsory application bytes.
#   photon Move    : 2 x 44 B promise + 4 B mu_s + 1 B split flag          =  93 B
#   photon Collide : 2 x 32 B promise (no direction) + 4 B absorb          =  68 B
#   photon Tally   : 2 x 8 B promise (slot and amount in one word)
#                    + 16 B uint64 read-modify-write                       =  32 B
#   BFS Relax      : 2 x 8 B promise + 8 B level read-modify-write          =  24 B
#   BFS Expand     : 2 x 16 B promise + 8 B rowptr + 4 B level of the expanded vertex      =  44 B
#                    (the 4 B column read per edge is counted on the Relax side)
#   Collatz Even/Odd: 2 x 16 B promise (+ 4 B output once per start, ignored) = 32 B
# ---------------------------------------------------------------------------------------
# Measured DRAM traffic (ncu dram__bytes_read.sum + dram__bytes_write.sum) of one exec launch on a
# small case of the same kernel, with its call count: scaled by calls to the bench's launch
# (profiles/photon_walk_async_exec_kernel_ncu.txt: 10^6 photons, variant 7).
TRAFFIC_PROFILE = {("photon", "async"): (47579904 + 609037056, 1613907450)}

BYTES_PER_CALL = {
    "photon": [93, 68, 32],
    "bfs": [24 + 4, 32 + 8 + 4],
    "collatz": [32, 32],
}


def run_photon(args, hrm, rank, world, pg, torch):
    n = args.grid
    count = args.photons
    first, count = replica_range(rank, count)
    seed = 0x5EED0123456789
    mu, ab, sp = hrm.photon_medium(n, 2024)
    nvox = n ** 3
    slots = nvox + 3 * hrm.PHOTON_SPREAD
    d_mu = torch.from_numpy(mu).cuda()
    d_ab = torch.from_numpy(ab).cuda()
    d_sp = torch.from_numpy(sp).cuda()
    d_tally = torch.zeros(slots, dtype=torch.int64, device="cuda")
    cfg = hrm.make_config(args.program, **pick_config(args))
    L = hrm.lib()

    def step_device():
        res = hrm.RunResult()
        hrm.check(L.hrm_photon_run_device(d_mu.data_ptr(), d_ab.data_ptr(), d_sp.data_ptr(), n, seed, first, count,
                                          d_tally.data_ptr(), ctypes.byref(cfg), ctypes.byref(res)))
        return res.as_dict()

    h_mu = torch.from_numpy(mu).pin_memory()
    h_ab = torch.from_numpy(ab).pin_memory()
    h_sp = torch.from_numpy(sp).pin_memory()
    h_tally = torch.zeros(slots, dtype=torch.int64).pin_memory()

    def step_e2e():
        res = hrm.RunResult()
        hrm.check(L.hrm_photon_run(h_mu.data_ptr(), h_ab.data_ptr(), h_sp.data_ptr(), n, seed, first, count,
                                   h_tally.data_ptr(), ctypes.byref(cfg), ctypes.byref(res)))
        return res.as_dict()

    def checksum():
        t = d_tally.cpu().numpy().view(np.uint64)
        total = (int(t[:nvox].sum()) + int(t[nvox:nvox + 1024].sum()) + int(t[nvox + 1024:nvox + 2048].sum())
                 - int(t[nvox + 2048:].sum()))
        return int(t.sum(dtype=np.uint64)), total / 2.0 ** 32

    def oracle_check():
        """The whole workload on the OpenMP host executor of the same spec source, compared bit
        for bit with the last timed run's tallies; its time is the CPU baseline."""
        import oracle
        threads = oracle.max_threads()
        got = d_tally.cpu().numpy().view(np.uint64)
        t0 = time.perf_counter()
        ref, calls = oracle.exec_photon(mu, ab, sp, n, seed, first, count, threads=threads)
        dt = time.perf_counter() - t0
        cpu = {"value": float(calls.sum()) / dt, "unit": "calls/s", "cores": threads, "kind": "port",
               "sample": f"the whole workload ({count} photons on the {n}^3 medium), OpenMP host executor of the "
                         f"same spec source, {int(calls.sum())} calls in {dt:.1f} s"}
        return np.array_equal(got, ref), cpu

    def plain_arm(flush):
        """The same photons through the plain kernel (one thread per source photon, walking its
        split descendants on a per-thread stack; no runtime), best of three with L2 flushed,
        and whether its tallies equal the timed run's. Outside the timed region."""
        from harmonize_b200 import jobs
        d_plain = torch.zeros(slots, dtype=torch.int64, device="cuda")
        arr = (jobs.Job * 1)()
        arr[0] = jobs.Job(jobs.JOB_PHOTON, first, count, n, seed, d_mu.data_ptr(), d_ab.data_ptr(), d_sp.data_ptr(),
                          d_plain.data_ptr())
        JL = jobs._bind()
        best = None
        for _ in range(3):
            flush_l2(flush)
            torch.cuda.synchronize()
            done = np.zeros(1, dtype=np.uint64)
            total = ctypes.c_float()
            hrm.check(JL.hrm_plain_run(ctypes.byref(arr), 1, 1, done.ctypes.data, ctypes.byref(total)))
            best = total.value if best is None else min(best, total.value)
        return best, {"same_tallies": bool(torch.equal(d_plain, d_tally)),
                      "what": "one thread per source photon walking its split descendants on a per-thread stack, "
                              "one launch, best of 3; equivalent calls = the runtime's call count for these photons"}

    return dict(step_device=step_device, step_e2e=step_e2e, checksum=checksum, oracle_check=oracle_check,
                plain_arm=plain_arm,
                h2d=int(mu.nbytes + ab.nbytes + sp.nbytes), d2h=int(slots * 8), dtype="f32",
                bytes_per_call=BYTES_PER_CALL["photon"], launches_per_step=3 if args.program == "async" else 2)


def run_bfs(args, hrm, rank, world, pg, torch):
    rp, col = hrm.rmat_csr(args.scale, 16, 0.57, 0.19, 0.19, 1)
    nv = len(rp) - 1
    d_rp = torch.from_numpy(rp.view(np.int32)).cuda()
    d_col = torch.from_numpy(col.view(np.int32)).cuda()
    d_lev = torch.empty(nv, dtype=torch.int32, device="cuda")
    cfg = hrm.make_config(args.program, **pick_config(args))
    L = hrm.lib()

    def step_device():
        res = hrm.RunResult()
        hrm.check(L.hrm_bfs_run_device(d_rp.data_ptr(), d_col.data_ptr(), nv, 0, d_lev.data_ptr(), ctypes.byref(cfg),
                                       ctypes.byref(res)))
        return res.as_dict()

    h_rp = torch.from_numpy(rp.view(np.int32)).pin_memory()
    h_col = torch.from_numpy(col.view(np.int32)).pin_memory()
    h_lev = torch.empty(nv, dtype=torch.int32).pin_memory()

    def step_e2e():
        res = hrm.RunResult()
        hrm.check(L.hrm_bfs_run(h_rp.data_ptr(), h_col.data_ptr(), nv, 0, h_lev.data_ptr(), ctypes.byref(cfg),
                                ctypes.byref(res)))
        return res.as_dict()

    def checksum():
        lv = d_lev.cpu().numpy().view(np.uint32)
        return int(lv.astype(np.uint64).sum()), int((lv != 0xFFFFFFFF).sum())

    def oracle_check():
        import oracle
        threads = oracle.max_threads()
        got = d_lev.cpu().numpy().view(np.uint32)
        ok = np.array_equal(got, oracle.bfs(rp, col, 0))
        t0 = time.perf_counter()
        _, calls = oracle.exec_bfs(rp, col, 0, threads=threads)
        dt = time.perf_counter() - t0
        cpu = {"value": float(calls.sum()) / dt, "unit": "calls/s", "cores": threads, "kind": "port",
               "sample": f"full R-MAT 2^{args.scale} BFS, OpenMP host executor of the same spec source"}
        return ok, cpu

    return dict(step_device=step_device, step_e2e=step_e2e, checksum=checksum, oracle_check=oracle_check,
                h2d=int(rp.nbytes + col.nbytes), d2h=int(nv * 4), dtype="u32",
                bytes_per_call=BYTES_PER_CALL["bfs"], launches_per_step=3 if args.program == "async" else 2)


def run_collatz(args, hrm, rank, world, pg, torch):
    first, count = replica_range(rank, 1 << 20)
    start = 1 + first
    d_out = torch.empty(count, dtype=torch.int32, device="cuda")
    cfg = hrm.make_config(args.program, **pick_config(args))
    L = hrm.lib()

    def step_device():
        res = hrm.RunResult()
        hrm.check(L.hrm_collatz_run_device(start, count, d_out.data_ptr(), ctypes.byref(cfg), ctypes.byref(res)))
        return res.as_dict()

    h_out = torch.empty(count, dtype=torch.int32).pin_memory()

    def step_e2e():
        res = hrm.RunResult()
        hrm.check(L.hrm_collatz_run(start, count, h_out.data_ptr(), ctypes.byref(cfg), ctypes.byref(res)))
        return res.as_dict()

    def checksum():
        o = d_out.cpu().numpy().view(np.uint32)
        return int(o.astype(np.uint64).sum()), int(o.max())

    def oracle_check():
        import oracle
        threads = oracle.max_threads()
        got = d_out.cpu().numpy().view(np.uint32)
        ok = np.array_equal(got, oracle.collatz_range(start, count))
        t0 = time.perf_counter()
        _, calls = oracle.exec_collatz(start, count, threads=threads)
        dt = time.perf_counter() - t0
        cpu = {"value": float(calls.sum()) / dt, "unit": "calls/s", "cores": threads, "kind": "port",
               "sample": "n = 1..2^20, OpenMP host executor of the same spec source"}
        return ok, cpu

    def plain_arm(flush):
        """The same start values through the plain kernel of the reference's plain Collatz example
        (examples/cpp/collaz/collaz_std.cpp:5-21: one thread per start value, iterating to 1),
        best of three with L2 flushed, and whether its step counts equal the timed run's.
        Outside the timed region."""
        from harmonize_b200 import jobs
        d_plain = torch.empty(count, dtype=torch.int32, device="cuda")
        arr = (jobs.Job * 1)()
        arr[0] = jobs.Job(jobs.JOB_COLLATZ, start, count, 0, 0, None, None, None, d_plain.data_ptr())
        JL = jobs._bind()
        best = None
        for _ in range(3):
            flush_l2(flush)
            torch.cuda.synchronize()
            done = np.zeros(1, dtype=np.uint64)
            total = ctypes.c_float()
            hrm.check(JL.hrm_plain_run(ctypes.byref(arr), 1, 1, done.ctypes.data, ctypes.byref(total)))
            best = total.value if best is None else min(best, total.value)
        return best, {"same_outputs": bool(torch.equal(d_plain, d_out)),
                      "what": "one thread per start value iterating to 1, one launch, best of 3; equivalent calls = "
                              "the runtime's call count for these start values"}

    return dict(step_device=step_device, step_e2e=step_e2e, checksum=checksum, oracle_check=oracle_check,
                plain_arm=plain_arm,
                h2d=0, d2h=count * 4, dtype="u64",
                bytes_per_call=BYTES_PER_CALL["collatz"], launches_per_step=3 if args.program == "async" else 2)


def percentiles_ms(ns):
    a = np.asarray(ns, dtype=np.float64) / 1e6
    return {"p50": round(float(np.percentile(a, 50)), 3), "p99": round(float(np.percentile(a, 99)), 3),
            "p99.9": round(float(np.percentile(a, 99.9)), 3), "max": round(float(a.max()), 3)}


def run_batched(args):
    """Batched uneven instances: the job mix in ONE persistent launch vs one plain launch per job."""
    import torch
    import harmonize_b200 as hrm
    from harmonize_b200 import jobs
    specs = jobs.make_mix_specs(args.jobs, seed=1)
    mix = jobs.Mix(specs, photon_grid=32, media=8, seed=1, sets=4)
    tc = dict(pick_config(args, "batched", "async"), job_order=JOB_ORDERS[args.job_order])
    variant = tc["variant"]
    warm = list(range(min(48, args.jobs)))
    jobs.batch_run(mix, 0, warm, **tc)
    jobs.plain_run(mix, 1, warm)
    jobs.runtime_run(mix, 2, warm)
    # The solo lanes' program instances are made on first use: warm them up on a few large jobs.
    solo_warm = [i for i, s in enumerate(specs)
                 if s["kind"] == jobs.JOB_PHOTON and s["count"] >= args.solo_photons][:max(1, args.solo_lanes)]
    jobs.batch_run_solo(mix, 3, indices=solo_warm, solo_photons=args.solo_photons, lanes=args.solo_lanes, **tc)
    with ClockSampler(0) as clk:
        done_b, res = jobs.batch_run(mix, 0, **tc)
        torch.cuda.synchronize()
        done_p, plain_ms = jobs.plain_run(mix, 1, streams=16)
        torch.cuda.synchronize()
        done_r, runtime_ms = jobs.runtime_run(mix, 2)
        torch.cuda.synchronize()
        done_s, solo_ms, _ = jobs.batch_run_solo(mix, 3, solo_photons=args.solo_photons, lanes=args.solo_lanes, **tc)
    for other, name in ((1, "plain-kernel"), (2, "per-job runtime"), (3, "persistent with solo large jobs")):
        mism = [i for i in range(len(specs)) if not np.array_equal(mix.output(0, i), mix.output(other, i))]
        if mism:
            raise SystemExit(f"bench: {len(mism)} jobs differ between the persistent and {name} runs")
    span_b = res["device_ms"]
    calls = res["evals"]
    line = {
        "metric": "async calls/s", "value": round(calls / (span_b / 1e3), 1), "unit": "calls/s", "n_gpus": 1,
        "steps": 1, "warmup": 1, "ms_per_step": round(span_b, 3), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32+u64", "data": "synthetic",
        "config": {"workload": f"batched_{args.jobs}_mixed_instances", "jobs": mix.total_work(),
                   "variant": dict(tc, ring_links_teams_per_cta=list(hrm.VARIANTS[variant])),
                   "persistent": "one launch (CUDA graph) of AsyncProgram<MixSpec>",
                   "runtime_per_job": "one whole single-spec AsyncProgram run per job (init, exec until "
                                      "complete, synchronised), tuned variant per kind",
                   "plain": "one hand-written plain kernel launch per job (one thread per item), 16 streams",
                   "persistent_solo": f"photon jobs of >= {args.solo_photons} photons through the single-spec "
                                      f"runtime over {args.solo_lanes} concurrent lanes (hrm_solo_run), all other "
                                      "jobs in one persistent launch"},
        "jobs_per_s": {"persistent": round(args.jobs / (span_b / 1e3), 1),
                       "persistent_solo": round(args.jobs / (solo_ms / 1e3), 1),
                       "runtime_per_job": round(args.jobs / (runtime_ms / 1e3), 1),
                       "plain": round(args.jobs / (plain_ms / 1e3), 1)},
        "speedup_job_throughput": {"vs_runtime_per_job": round(runtime_ms / span_b, 3),
                                   "vs_plain_kernels": round(plain_ms / span_b, 3),
                                   "solo_vs_runtime_per_job": round(runtime_ms / solo_ms, 3),
                                   "solo_vs_plain_kernels": round(plain_ms / solo_ms, 3)},
        "completion_ms": {"persistent": percentiles_ms(done_b), "persistent_solo": percentiles_ms(done_s),
                          "runtime_per_job": percentiles_ms(done_r), "plain": percentiles_ms(done_p)},
        "outputs": "identical per job (all four arms)",
        "full_batch_fraction": round(res["full_batches"] / max(1, res["batches"]), 4),
        "clocks": clk.summary(),
    }
    print(json.dumps(line), flush=True)
    return line


def run_serving(args):
    """Serving: Poisson arrivals of the job mix, rate swept as fractions of the resident runtime's
    batched throughput; the resident runtime against, at the same arrivals, plain execution of
    the runtime (one whole single-spec run per job, one job at a time) and one plain kernel
    launch per job (16 streams)."""
    import harmonize_b200 as hrm
    from harmonize_b200 import jobs
    n = args.serve_jobs
    specs = jobs.make_mix_specs(n, seed=2)
    mix = jobs.Mix(specs, photon_grid=32, media=8, seed=2, sets=3)
    tc = dict(pick_config(args, "batched", "async"), job_order=JOB_ORDERS[args.job_order])
    variant = tc["variant"]
    done_b, res = jobs.batch_run(mix, 0, **tc)
    sat = n / (res["device_ms"] / 1e3)
    rows = []
    for frac in args.rates:
        rate = frac * sat
        arr = jobs.poisson_arrivals(n, rate, seed=5)
        lat_r, span_r = jobs.serve_replay(mix, arr, mode="resident", which=0, solo_photons=args.serve_solo_photons,
                                          **tc)
        lat_p, span_p = jobs.serve_replay(mix, arr, mode="plain", which=1, streams=16)
        lat_u, span_u = jobs.serve_replay(mix, arr, mode="runtime", which=2)
        rows.append({"load": frac, "rate_jobs_per_s": round(rate, 1),
                     "resident": dict(percentiles_ms(lat_r), jobs_per_s=round(n / (span_r / 1e3), 1)),
                     "runtime_per_job": dict(percentiles_ms(lat_u), jobs_per_s=round(n / (span_u / 1e3), 1)),
                     "plain": dict(percentiles_ms(lat_p), jobs_per_s=round(n / (span_p / 1e3), 1))})
        print(json.dumps(rows[-1]), flush=True)
    mism = [i for i in range(n) if not (np.array_equal(mix.output(0, i), mix.output(1, i)) and
                                        np.array_equal(mix.output(0, i), mix.output(2, i)))]
    line = {"metric": "job latency p50/p99/p99.9 (ms) and job throughput", "workload": f"serving_{n}_jobs",
            "saturation_jobs_per_s": round(sat, 1), "solo_photons": args.serve_solo_photons, "rates": rows,
            "outputs": "identical per job" if not mism else f"{len(mism)} jobs differ"}
    print(json.dumps(line), flush=True)
    return line


def pick_config(args, workload=None, program=None):
    """--variant (with default tunables), else the autotuner's choice (variant, patience,
    fill_links) for this workload and program type."""
    if args.variant >= 0:
        return {"variant": args.variant, "patience": 0, "fill_links": 0}
    from harmonize_b200.autotune import tuned_config
    return tuned_config(workload or args.workload, program or args.program)


def pick_variant(args, hrm):
    return pick_config(args)["variant"]


def plain_record(ms, runtime_calls, info):
    """The line's plain_kernel entry: the plain kernel's time, the runtime's call count for the
    same inputs over that time, and the leg's own fields (output comparison, description)."""
    return dict({"ms": round(ms, 3), "equivalent_calls_per_s": round(runtime_calls / (ms / 1e3), 1)}, **info)


def algorithmic_bytes(stats, per_call):
    return sum(stats.get(f"fn{i}_evals", 0) * b for i, b in enumerate(per_call))


def main():
    args = parse()
    if args.impl == "reference":
        from oracle import reference_bench
        return reference_bench.main(args, workload_config(args, int(os.environ.get("WORLD_SIZE", "1"))))
    if args.workload == "batched":
        return run_batched(args)
    if args.workload == "serving":
        return run_serving(args)
    import torch
    import harmonize_b200 as hrm
    rank, world, local, pg = dist_setup(args)
    wl = {"photon": run_photon, "bfs": run_bfs, "collatz": run_collatz}[args.workload](args, hrm, rank, world, pg,
                                                                                       torch)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    for _ in range(max(args.warmup, 0)):
        wl["step_device"]()
    ref_sum = wl["checksum"]()

    # Timed device-resident steps.
    barrier(pg)
    step_ms, stats_all = [], []
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            flush_l2(flush)
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            st = wl["step_device"]()
            e1.record()
            e1.synchronize()
            step_ms.append(e0.elapsed_time(e1))
            stats_all.append(st)
            if wl["checksum"]() != ref_sum:
                raise SystemExit("bench: results differ between steps (determinism violated)")
    barrier(pg)
    my_ms = sum(step_ms)
    total_ms = max_over_ranks(pg, my_ms)
    calls = sum(s["evals"] for s in stats_all)
    all_calls = sum_over_ranks(pg, calls)
    value = all_calls / (total_ms / 1e3)

    # End-to-end through the host-buffer entry point.
    wl["step_e2e"]()
    barrier(pg)
    e2e_ms = []
    e2e_steps = max(1, min(args.steps, 3))
    for _ in range(e2e_steps):
        flush_l2(flush)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        st = wl["step_e2e"]()
        e1.record()
        e1.synchronize()
        e2e_ms.append(e0.elapsed_time(e1))
    barrier(pg)
    e2e_total = max_over_ranks(pg, sum(e2e_ms))
    e2e_calls = sum_over_ranks(pg, st["evals"] * e2e_steps)
    e2e_value = e2e_calls / (e2e_total / 1e3)

    # Rank 0: the plain one-thread-per-item kernel on the same inputs (not a bench arm: the
    # runtime's non-runtime baseline, outside the timed region).
    plain = None
    if rank == 0 and "plain_arm" in wl:
        p_ms, p_info = wl["plain_arm"](flush)
        plain = plain_record(p_ms, stats_all[-1]["evals"], p_info)

    pk = peaks()
    s0 = stats_all[-1]
    alg = algorithmic_bytes(s0, wl["bytes_per_call"])
    achieved_gbs = alg / (step_ms[-1] / 1e3) / 1e9
    prof = TRAFFIC_PROFILE.get((args.workload, args.program))
    traffic = round(prof[0] / prof[1] * s0["evals"]) if prof else None
    roofline = {"bound": "hbm", "achieved": round(achieved_gbs, 1), "peak": pk["hbm_gbs"], "unit": "GB/s",
                "frac": round(achieved_gbs / pk["hbm_gbs"], 4), "traffic": traffic,
                "traffic_source": ("ncu DRAM bytes of a 10^6-photon launch scaled by calls" if prof else None),
                "peak_source": pk["source"],
                "algorithmic_bytes_per_launch": alg,
                "note": "algorithmic bytes = each call's promise written and read once plus its compulsory "
                        "application bytes; the launch duration is the whole run (init + exec kernels)"}
    # Parity of the timed workload: rank 0 checks its last device-resident run against the
    # oracle (outside the timed region); the run of the oracle is also the CPU baseline.
    cpu, oracle_check = None, None
    if rank == 0 and not args.no_cpu:
        ok, cpu = wl["oracle_check"]()
        if not ok:
            raise SystemExit("bench: the timed run's output differs from the oracle")
        oracle_check = "exact"
        if world > 1:
            cpu = None
    if rank == 0:
        full = s0.get("full_batches", 0) / max(1, s0.get("batches", 1))
        line = {
            "metric": "async calls/s", "value": round(value, 1), "unit": "calls/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(total_ms / args.steps, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": wl["dtype"],
            "data": "synthetic",
            "config": workload_config(args, world),
            "implementation": {"program": args.program,
                               "variant": dict(pick_config(args), ring_links_teams_per_cta=list(
                                   hrm.VARIANTS[pick_variant(args, hrm)]))},
            "oracle_check": oracle_check,
            "e2e": {"value": round(e2e_value, 1), "unit": "calls/s", "h2d_bytes_per_step": wl["h2d"],
                    "d2h_bytes_per_step": wl["d2h"]},
            "roofline": roofline, "cpu_baseline": cpu, "clocks": clk.summary(),
            "plain_kernel": plain,
            "gpu_launches": wl["launches_per_step"] * args.steps,
            "runtime_stats": {"calls_per_step": s0["evals"], "full_batch_fraction": round(full, 4),
                              "spill_links": s0.get("spill_links"), "fill_links": s0.get("fill_links"),
                              "execs": s0.get("execs")},
        }
        print(json.dumps(line), flush=True)
    if pg is not None:
        pg.destroy_process_group()


if __name__ == "__main__":
    main()

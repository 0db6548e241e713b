"""Mixed job batches over the C ABI: the batched-instances and serving workloads.

A job is one instance of a built-in spec (hrm_job in include/hrm_capi.h). make_mix builds
the seeded synthetic mix of the batched configuration:
  * Collatz ranges of length lognormal(median 2^12, sigma 1.5) clipped to [2^6, 2^20],
    starting at a uniform value in [1, 2^21];
  * photon-walk batches of 10^3..10^6 photons (log-uniform) on 32^3 grids, media drawn with
    the same distributions (a pool of seeded media shared by the jobs);
  * BFS from a random root on R-MAT graphs of 2^12..2^18 vertices, edge factor 16 (one seeded
    graph per size, shared by the jobs).
Device buffers are torch CUDA tensors kept alive by the Mix object.
"""
import ctypes

import numpy as np

from . import (HarmonizeError, RunResult, check, lib, make_config, photon_medium, rmat_csr)

JOB_COLLATZ, JOB_PHOTON, JOB_BFS = 0, 1, 2
KIND_NAMES = {JOB_COLLATZ: "collatz", JOB_PHOTON: "photon", JOB_BFS: "bfs"}
PHOTON_SPREAD = 1024


class Job(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_uint32), ("first", ctypes.c_uint32), ("count", ctypes.c_uint32),
                ("n", ctypes.c_uint32), ("seed", ctypes.c_uint64), ("a", ctypes.c_void_p),
                ("b", ctypes.c_void_p), ("c", ctypes.c_void_p), ("out", ctypes.c_void_p)]


def _bind():
    L = lib()
    if not getattr(L, "_jobs_bound", False):
        L.hrm_batch_run.restype = ctypes.c_int
        L.hrm_batch_run.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p, ctypes.c_void_p,
                                    ctypes.c_void_p]
        L.hrm_serve_replay_runtime.restype = ctypes.c_int
        L.hrm_serve_replay_runtime.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p, ctypes.c_int,
                                               ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(ctypes.c_float)]
        L.hrm_runtime_run.restype = ctypes.c_int
        L.hrm_runtime_run.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_int, ctypes.c_void_p,
                                      ctypes.c_void_p, ctypes.POINTER(ctypes.c_float)]
        L.hrm_plain_run.restype = ctypes.c_int
        L.hrm_plain_run.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_void_p,
                                    ctypes.POINTER(ctypes.c_float)]
        vp, u32 = ctypes.c_void_p, ctypes.c_uint32
        for name, args in {
            "hrm_server_open": [u32, vp, ctypes.POINTER(vp)],
            "hrm_server_submit": [vp, vp, u32, ctypes.POINTER(u32)],
            "hrm_server_poll": [vp, vp, u32, ctypes.POINTER(u32)],
            "hrm_server_close": [vp, u32],
            "hrm_server_destroy": [vp],
            "hrm_serve_replay": [vp, u32, vp, ctypes.c_int, u32, vp, vp, ctypes.POINTER(ctypes.c_float)],
            "hrm_solo_run": [vp, u32, ctypes.c_int, u32, vp, ctypes.POINTER(ctypes.c_float)],
        }.items():
            f = getattr(L, name)
            f.restype = ctypes.c_int
            f.argtypes = args
        L._jobs_bound = True
    return L


class Server:
    """A resident runtime session: submit jobs while it runs, poll completions, close."""

    def __init__(self, capacity, **cfg_kw):
        L = _bind()
        self.cfg = make_config("async", **cfg_kw)
        h = ctypes.c_void_p()
        check(L.hrm_server_open(capacity, ctypes.byref(self.cfg), ctypes.byref(h)))
        self.h = h
        self.capacity = capacity

    def submit(self, job_array):
        first = ctypes.c_uint32()
        check(_bind().hrm_server_submit(self.h, ctypes.byref(job_array), len(job_array), ctypes.byref(first)))
        return first.value

    def poll(self):
        done = np.zeros(self.capacity, dtype=np.uint64)
        c = ctypes.c_uint32()
        check(_bind().hrm_server_poll(self.h, done.ctypes.data, self.capacity, ctypes.byref(c)))
        return done, c.value

    def close(self, timeout_ms=60000):
        check(_bind().hrm_server_close(self.h, timeout_ms))

    def __del__(self):
        if getattr(self, "h", None):
            _bind().hrm_server_destroy(self.h)
            self.h = None


def serve_replay(mix, arrivals_ns, mode="resident", which=0, indices=None, streams=16, **cfg_kw):
    """Replays arrival times against the resident runtime ("resident"), one plain kernel launch
    per job ("plain"), or one whole single-spec runtime run per job, one job at a time
    ("runtime"). Returns (latency_ns array, makespan ms)."""
    L = _bind()
    arr = mix.job_array(which, indices)
    arrivals = np.ascontiguousarray(arrivals_ns, dtype=np.uint64)
    lat = np.zeros(len(arr), dtype=np.uint64)
    span = ctypes.c_float()
    if mode == "runtime":
        from .autotune import tuned_variant
        v = (ctypes.c_int * 3)(*[tuned_variant(w, "async") for w in ("collatz", "photon", "bfs")])
        check(L.hrm_serve_replay_runtime(ctypes.byref(arr), len(arr), arrivals.ctypes.data, 0, v, lat.ctypes.data,
                                         ctypes.byref(span)))
        return lat, span.value
    cfg = make_config("async", **cfg_kw)
    check(L.hrm_serve_replay(ctypes.byref(arr), len(arr), arrivals.ctypes.data, 0 if mode == "resident" else 1,
                             streams, ctypes.byref(cfg), lat.ctypes.data, ctypes.byref(span)))
    return lat, span.value


def poisson_arrivals(n, rate_per_s, seed=11):
    """Cumulative Poisson-process arrival times (ns) of n jobs at the given rate."""
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / rate_per_s, n)
    return np.cumsum(gaps * 1e9).astype(np.uint64)


class Mix:
    """A list of jobs with their device inputs and `sets` sets of device outputs (so that a
    batched run and baseline runs can be compared)."""

    def __init__(self, specs, photon_grid=32, media=8, seed=1, sets=2):
        import torch
        self.torch = torch
        # list of dicts: kind, first, count / scale, medium / graph index
        self.specs = [dict(s, medium=s["medium"] % media) if "medium" in s else dict(s) for s in specs]
        self.grid = photon_grid
        self.media = []
        for m in range(media):
            mu, ab, sp = photon_medium(photon_grid, seed * 1000 + m)
            self.media.append(tuple(torch.from_numpy(x).cuda() for x in (mu, ab, sp)))
        self.graphs = {}
        for s in specs:
            if s["kind"] == JOB_BFS and s["scale"] not in self.graphs:
                rp, col = rmat_csr(s["scale"], 16, 0.57, 0.19, 0.19, seed * 100 + s["scale"])
                self.graphs[s["scale"]] = (torch.from_numpy(rp.view(np.int32)).cuda(),
                                           torch.from_numpy(col.view(np.int32)).cuda(), rp, col)
        self.outputs = [self._alloc_outputs() for _ in range(sets)]

    def _alloc_outputs(self):
        torch = self.torch
        outs = []
        for s in self.specs:
            if s["kind"] == JOB_COLLATZ:
                outs.append(torch.empty(s["count"], dtype=torch.int32, device="cuda"))
            elif s["kind"] == JOB_PHOTON:
                outs.append(torch.empty(self.grid ** 3 + 3 * PHOTON_SPREAD, dtype=torch.int64, device="cuda"))
            else:
                outs.append(torch.empty(1 << s["scale"], dtype=torch.int32, device="cuda"))
        return outs

    def job_array(self, which=0, indices=None):
        idx = range(len(self.specs)) if indices is None else indices
        arr = (Job * len(idx))()
        for k, i in enumerate(idx):
            s = self.specs[i]
            out = self.outputs[which][i].data_ptr()
            if s["kind"] == JOB_COLLATZ:
                arr[k] = Job(JOB_COLLATZ, s["first"], s["count"], 0, 0, None, None, None, out)
            elif s["kind"] == JOB_PHOTON:
                mu, ab, sp = self.media[s["medium"]]
                arr[k] = Job(JOB_PHOTON, s["first"], s["count"], self.grid, s["seed"], mu.data_ptr(),
                             ab.data_ptr(), sp.data_ptr(), out)
            else:
                d_rp, d_col, _, _ = self.graphs[s["scale"]]
                arr[k] = Job(JOB_BFS, s["root"], 1, 1 << s["scale"], 0, d_rp.data_ptr(), d_col.data_ptr(), None,
                             out)
        return arr

    def output(self, which, i):
        t = self.outputs[which][i].cpu().numpy()
        return t.view(np.uint64) if self.specs[i]["kind"] == JOB_PHOTON else t.view(np.uint32)

    def total_work(self):
        return {KIND_NAMES[k]: sum(1 for s in self.specs if s["kind"] == k) for k in KIND_NAMES}


def make_mix_specs(njobs, seed=1, max_photons=1_000_000, max_scale=18, max_collatz=1 << 20):
    """The seeded job mix (equal thirds of Collatz, photon and BFS jobs, interleaved)."""
    rng = np.random.default_rng(seed)
    specs = []
    for j in range(njobs):
        kind = j % 3
        if kind == JOB_COLLATZ:
            length = int(np.clip(round(4096 * np.exp(1.5 * rng.standard_normal())), 64, max_collatz))
            first = int(rng.integers(1, (1 << 21) + 1))
            specs.append({"kind": JOB_COLLATZ, "first": first, "count": length})
        elif kind == JOB_PHOTON:
            count = int(round(10 ** rng.uniform(3.0, np.log10(max_photons))))
            specs.append({"kind": JOB_PHOTON, "first": int(rng.integers(0, 1 << 30)), "count": count,
                          "seed": int(rng.integers(1, 1 << 62)), "medium": int(rng.integers(0, 8))})
        else:
            scale = int(rng.integers(12, max_scale + 1))
            specs.append({"kind": JOB_BFS, "scale": scale, "root": int(rng.integers(0, 1 << scale))})
    return specs


def batch_run(mix, which=0, indices=None, **cfg_kw):
    """All (or the chosen) jobs in one persistent launch. Returns (done_ns array, result dict)."""
    L = _bind()
    arr = mix.job_array(which, indices)
    done = np.zeros(len(arr), dtype=np.uint64)
    cfg = make_config("async", **cfg_kw)
    res = RunResult()
    check(L.hrm_batch_run(ctypes.byref(arr), len(arr), ctypes.byref(cfg), ctypes.byref(res), done.ctypes.data))
    return done, res.as_dict()


def batch_run_solo(mix, which=0, solo_photons=1 << 15, indices=None, lanes=1, **cfg_kw):
    """The batch with its largest jobs taken out of the persistent launch.

    Photon jobs of at least `solo_photons` photons each fill the GPU on their own, so running
    them among the other jobs gains them nothing and costs them the job indirection of the
    multiplexing kernel (about half its speed on photon work). They run through the
    single-spec runtime after one persistent launch of all the other jobs: one after another
    (lanes=1), or over `lanes` concurrent lanes that share the GPU (hrm_solo_run), so that each
    job's tail of dependent calls overlaps the others' work.
    Returns (done_ns per job from the start of the batch, total ms, result of the persistent
    launch or None)."""
    idx = list(range(len(mix.specs))) if indices is None else list(indices)
    solo = [i for i in idx if mix.specs[i]["kind"] == JOB_PHOTON and mix.specs[i]["count"] >= solo_photons]
    solo_set = set(solo)
    rest = [i for i in idx if i not in solo_set]
    pos = {i: k for k, i in enumerate(idx)}
    done = np.zeros(len(idx), dtype=np.uint64)
    total_ms, res = 0.0, None
    if rest:
        d, res = batch_run(mix, which, indices=rest, **cfg_kw)
        for k, i in enumerate(rest):
            done[pos[i]] = d[k]
        total_ms += res["device_ms"]
    if solo and lanes > 1:
        from .autotune import tuned_variant
        L = _bind()
        arr = mix.job_array(which, solo)
        d = np.zeros(len(arr), dtype=np.uint64)
        total = ctypes.c_float()
        check(L.hrm_solo_run(ctypes.byref(arr), len(arr), tuned_variant("photon", "async"), lanes, d.ctypes.data,
                             ctypes.byref(total)))
        for k, i in enumerate(solo):
            done[pos[i]] = d[k] + np.uint64(total_ms * 1e6)
        total_ms += total.value
    elif solo:
        d, ms = runtime_run(mix, which, indices=solo)
        for k, i in enumerate(solo):
            done[pos[i]] = d[k] + np.uint64(total_ms * 1e6)
        total_ms += ms
    return done, total_ms, res


def runtime_run(mix, which=1, indices=None, program="async", variants=None):
    """One whole single-spec runtime run per job, in order (plain execution of the runtime).
    variants: per job kind (Collatz, photon, BFS), default the autotuner's choice for each.
    Returns (done_ns array, total ms)."""
    L = _bind()
    arr = mix.job_array(which, indices)
    done = np.zeros(len(arr), dtype=np.uint64)
    total = ctypes.c_float()
    if variants is None:
        from .autotune import tuned_variant
        variants = [tuned_variant(w, program) for w in ("collatz", "photon", "bfs")]
    v = (ctypes.c_int * 3)(*variants)
    pt = {"async": 0, "event": 1}[program]
    check(L.hrm_runtime_run(ctypes.byref(arr), len(arr), pt, v, done.ctypes.data, ctypes.byref(total)))
    return done, total.value


def plain_run(mix, which=1, indices=None, streams=16):
    """One plain-kernel launch per job. Returns (done_ns array, total ms)."""
    L = _bind()
    arr = mix.job_array(which, indices)
    done = np.zeros(len(arr), dtype=np.uint64)
    total = ctypes.c_float()
    check(L.hrm_plain_run(ctypes.byref(arr), len(arr), streams, done.ctypes.data, ctypes.byref(total)))
    return done, total.value


def main(argv=None):
    """Runs one batch of jobs from the command line and prints its result as JSON:

        python -m harmonize_b200.jobs [--jobs N] [--seed S] [--kind collatz|photon|bfs]
                                      [--photon-job COUNT] [--variant V] [--arena LINKS]

    --photon-job COUNT runs a single photon job of COUNT photons on a 32^3 medium (the case
    used to profile the batched kernel); otherwise the seeded job mix of N jobs, optionally
    restricted to one kind."""
    import argparse
    import json
    ap = argparse.ArgumentParser()
    ap.add_argument("--jobs", type=int, default=384)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--kind", choices=list(KIND_NAMES.values()), default=None)
    ap.add_argument("--photon-job", type=int, default=0)
    ap.add_argument("--variant", type=int, default=2)
    ap.add_argument("--arena", type=int, default=0)
    ap.add_argument("--arm", choices=["persistent", "runtime", "plain"], default="persistent",
                    help="one persistent launch, one single-spec runtime run per job, or one plain kernel per job")
    a = ap.parse_args(argv)
    if a.photon_job:
        specs = [{"kind": JOB_PHOTON, "first": 0, "count": a.photon_job, "seed": 0x1234567, "medium": 0}]
        mix = Mix(specs, photon_grid=32, media=1, seed=a.seed)
        idx = None
    else:
        mix = Mix(make_mix_specs(a.jobs, seed=a.seed), photon_grid=32, media=8, seed=a.seed)
        kinds = {v: k for k, v in KIND_NAMES.items()}
        idx = None if a.kind is None else [i for i, s in enumerate(mix.specs) if s["kind"] == kinds[a.kind]]
    if a.arm == "persistent":
        batch_run(mix, 0, indices=idx, variant=a.variant, arena=a.arena)  # warm-up (graph capture)
        done, res = batch_run(mix, 0, indices=idx, variant=a.variant, arena=a.arena)
        res["calls_per_s"] = res["evals"] / (res["device_ms"] / 1e3)
    else:
        run = runtime_run if a.arm == "runtime" else plain_run
        run(mix, 1, indices=idx)  # warm-up
        done, ms = run(mix, 1, indices=idx)
        res = {"total_ms": ms}
    res["arm"] = a.arm
    res["jobs"] = len(done)
    print(json.dumps(res))


if __name__ == "__main__":
    main()

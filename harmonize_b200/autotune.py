"""Autotuner: picks, per built-in workload and program type, the compiled variant (queue
width = shared-memory ring links per function, and teams per CTA) and the run-time
tunables of AsyncProgram (coalescing threshold `patience`, promise batch `fill_links` = links
one fill takes from the arena) with the highest throughput on the GPU it runs on.

    python -m harmonize_b200.autotune [--specs photon,bfs,collatz,batched] [--reps 2]

Workloads: 10^6 photons on the 128^3 bench medium, R-MAT 2^22 BFS from vertex 0, Collatz
1..2^20. Single-spec workloads are scored by async calls/s, except BFS, scored by searches per second
(its call count depends on the order of evaluation, so fewer calls can be the faster run);
"batched" (a seeded 384-job mix of all three specs in one persistent launch, the
job-multiplexing spec) by jobs/s.

Writes harmonize_b200/tuned.json: {"<workload>/<program>": {"variant": v, "ring_links": r,
"teams_per_cta": t, "patience": p, "fill_links": f, "score": x, "unit": ..., "sweep": [...]}}.
bench.py and the Python wrappers read it; a missing entry means variant 0 and the defaults.
The arena size is not swept: runs size it for their work (default_arena in the C ABI).
"""
import argparse
import itertools
import json
import os
import time

from . import HERE, VARIANTS, bfs, collatz, photon_medium, photon_walk, rmat_csr

TUNED_PATH = os.path.join(HERE, "tuned.json")
PATIENCE = (8, 16, 64)
FILL_LINKS = (2, 4)
BATCH_VARIANTS = (0, 1, 2, 7, 8)  # the variants the job-multiplexing spec is built for


def load_tuned():
    """The tuned table, or {} when none was written (a damaged file raises)."""
    try:
        with open(TUNED_PATH) as f:
            return json.load(f)
    except FileNotFoundError:
        return {}


def tuned_config(workload, program="async"):
    """{variant, patience, fill_links} chosen for a workload (zeros = defaults)."""
    e = load_tuned().get(f"{workload}/{program}", {})
    return {"variant": int(e.get("variant", 0)), "patience": int(e.get("patience", 0)),
            "fill_links": int(e.get("fill_links", 0))}


def tuned_variant(spec, program):
    return tuned_config(spec, program)["variant"]


def _single_spec_workloads():
    mu, ab, sp = photon_medium(128, 2024)
    # BFS at the benchmark's own scale: the best ring size depends on it (R-MAT 2^18 picked
    # 2-link rings, 3.3 ms on 2^22, where 4-link rings take 2.5 ms).
    rp, col = rmat_csr(22, 16, 0.57, 0.19, 0.19, 1)
    return {
        "photon": lambda prog, **kw: photon_walk(mu, ab, sp, 128, 0x5EED, 0, 1_000_000, program=prog, **kw)[1],
        "bfs": lambda prog, **kw: bfs(rp, col, 0, program=prog, **kw)[1],
        "collatz": lambda prog, **kw: collatz(1, 1 << 20, program=prog, **kw)[1],
    }


def _candidates(prog, variants):
    if prog == "event":  # EventProgram has no rings and no arena fills: teams per CTA only
        return [dict(variant=v) for v in variants if v not in (1, 3, 5, 6, 7, 8, 9)]
    return [dict(variant=v, patience=p, fill_links=f) for v, p, f in itertools.product(variants, PATIENCE, FILL_LINKS)]


def _best(sweep):
    ok = [s for s in sweep if "score" in s]
    return max(ok, key=lambda s: s["score"]) if ok else None


def _record(table, key, best, sweep, unit):
    v = best["variant"]
    table[key] = {"variant": v, "ring_links": VARIANTS[v][0], "teams_per_cta": VARIANTS[v][1],
                  "patience": best.get("patience", 0), "fill_links": best.get("fill_links", 0),
                  "score": best["score"], "unit": unit, "sweep": sweep,
                  "when": time.strftime("%Y-%m-%dT%H:%M:%SZ", time.gmtime())}
    print(key, "->", json.dumps({k: table[key][k] for k in ("variant", "patience", "fill_links", "score")}),
          flush=True)


def tune(specs, reps=2, programs=("async", "event")):
    table = load_tuned()
    work = _single_spec_workloads() if set(specs) - {"batched"} else {}
    for spec in specs:
        if spec == "batched":
            tune_batched(table, reps)
            continue
        for prog in programs:
            sweep = []
            for cand in _candidates(prog, VARIANTS):
                best = 0.0
                try:
                    for _ in range(reps + 1):
                        res = work[spec](prog, **cand)
                        work_done = 1.0 if spec == "bfs" else res["evals"]
                        best = max(best, work_done / (res["device_ms"] / 1e3))
                except Exception as e:  # a configuration that fails is not selectable
                    sweep.append(dict(cand, error=str(e)))
                    continue
                sweep.append(dict(cand, score=best))
            b = _best(sweep)
            if b:
                _record(table, f"{spec}/{prog}", b, sweep, "searches/s" if spec == "bfs" else "calls/s")
    with open(TUNED_PATH, "w") as f:
        json.dump(table, f, indent=1, sort_keys=True)
    return table


def tune_batched(table, reps):
    from . import jobs
    n = 384
    mix = jobs.Mix(jobs.make_mix_specs(n, seed=1), photon_grid=32, media=8, seed=1)
    sweep = []
    for cand in _candidates("async", BATCH_VARIANTS):
        best = 0.0
        try:
            for _ in range(reps + 1):
                _, res = jobs.batch_run(mix, 0, job_order=2, **cand)  # small first, as bench.py
                best = max(best, n / (res["device_ms"] / 1e3))
        except Exception as e:
            sweep.append(dict(cand, error=str(e)))
            continue
        sweep.append(dict(cand, score=best))
    b = _best(sweep)
    if b:
        _record(table, "batched/async", b, sweep, "jobs/s")


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--specs", default="photon,bfs,collatz,batched")
    ap.add_argument("--reps", type=int, default=2)
    a = ap.parse_args()
    tune(a.specs.split(","), a.reps)

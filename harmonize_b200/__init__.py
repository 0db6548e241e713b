"""B200-native Harmonize runtime: Python host bindings over libhrm.so (the C ABI).

The runtime itself is C++/CUDA (``include/harmonize.h``); this module loads the in-tree
``libhrm.so`` and exposes its entry points:

  * ``Program``: the instance life cycle of the original's foreign-call shim
    (alloc_program / init_program / exec_program / complete / clear_flags / free_program,
    harmonize/python/templates.py:3-184) for the built-in specs;
  * whole runs of the built-in specs from host arrays: ``collatz``, ``photon_walk``, ``bfs``,
    ``barrier_demo``; seeded inputs ``photon_medium`` and ``rmat_csr``;
  * ``harmonize_b200.jobs``: many jobs in one persistent launch (``batch_run``,
    ``batch_run_solo``), a resident serving session (``Server``, ``serve_replay``) and the
    per-job baselines (``runtime_run``, ``plain_run``);
  * ``harmonize_b200.autotune``: the tuner behind ``tuned.json``.

There is no CPU fallback: if the library or a GPU is missing, calls raise.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libhrm.so")

HRM_OK, HRM_EINVAL, HRM_ECUDA, HRM_EDEVICE, HRM_EINCOMPLETE, HRM_ENOMEM = range(6)
ASYNC, EVENT = 0, 1
SPEC_COLLATZ, SPEC_PHOTON, SPEC_BFS, SPEC_BARRIER_DEMO = range(4)

FLAG_BAD_FUNC_ID = 0x1
FLAG_STASH_FAIL = 0x2
FLAG_ARENA_EXHAUSTED = 0x4
FLAG_QUEUE_OVERFLOW = 0x8
FLAG_WAIT_TIMEOUT = 0x10
FLAG_EARLY_HALT = 0x40000000
FLAG_COMPLETION = 0x80000000

STAT_NAMES = ["evals", "batches", "full_batches", "spill_links", "fill_links", "make_work",
              "idle_polls", "generations"] + [f"fn{i}_evals" for i in range(16)]


class HarmonizeError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"libhrm status {code}: {msg}")
        self.code = code


class RunConfig(ctypes.Structure):
    _fields_ = [("program_type", ctypes.c_int), ("groups", ctypes.c_size_t), ("cycles", ctypes.c_size_t),
                ("chunk", ctypes.c_size_t), ("arena", ctypes.c_size_t), ("max_execs", ctypes.c_size_t),
                ("stream", ctypes.c_void_p), ("variant", ctypes.c_int), ("patience", ctypes.c_uint32),
                ("fill_links", ctypes.c_uint32), ("job_order", ctypes.c_uint32),
                ("solo_photons", ctypes.c_uint32)]


# Compiled tuning variants: (shared-memory ring links per function, teams per CTA). The lean
# variants (5, 6) give the first function 4 links and the others 2 and are compiled for at
# least 10 / 11 resident CTAs per SM; 7 and 8 are R4/T2 and R4/T4 compiled for at least 11 / 5;
# 9 is R3/T2 (3-link rings) compiled for at least 14.
VARIANTS = {0: (2, 4), 1: (4, 4), 2: (4, 2), 3: (8, 2), 4: (2, 8), 5: (4, 2), 6: (4, 2), 7: (4, 2), 8: (4, 4), 9: (3, 2)}


class RunResult(ctypes.Structure):
    _fields_ = [("flags", ctypes.c_uint32), ("execs", ctypes.c_uint32),
                ("stats", ctypes.c_uint64 * len(STAT_NAMES)), ("device_ms", ctypes.c_float)]

    def as_dict(self):
        d = {"flags": int(self.flags), "execs": int(self.execs), "device_ms": float(self.device_ms)}
        d.update({n: int(v) for n, v in zip(STAT_NAMES, self.stats)})
        return d


_lib = None


def lib():
    """Loads libhrm.so (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise HarmonizeError(-1, f"{LIB_PATH} not built: run `python -m harmonize_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        L.hrm_last_error.restype = ctypes.c_char_p
        vp, sz, u32, i32 = ctypes.c_void_p, ctypes.c_size_t, ctypes.c_uint32, ctypes.c_int
        sigs = {
            "hrm_set_device": [i32],
            "hrm_device_sync": [],
            "hrm_program_create": [i32, i32, sz, vp, sz, ctypes.POINTER(vp)],
            "hrm_program_destroy": [vp],
            "hrm_program_init": [vp, sz, vp],
            "hrm_program_exec": [vp, sz, sz, vp],
            "hrm_program_complete": [vp, ctypes.POINTER(i32)],
            "hrm_program_flags": [vp, ctypes.POINTER(u32)],
            "hrm_program_clear_flags": [vp],
            "hrm_program_stats": [vp, vp, sz],
            "hrm_program_overview": [vp, vp, sz, ctypes.POINTER(sz)],
            "hrm_collatz_run": [u32, u32, vp, ctypes.POINTER(RunConfig), ctypes.POINTER(RunResult)],
            "hrm_collatz_run_device": [u32, u32, vp, ctypes.POINTER(RunConfig), ctypes.POINTER(RunResult)],
            "hrm_photon_run": [vp, vp, vp, u32, ctypes.c_uint64, u32, u32, vp, ctypes.POINTER(RunConfig),
                               ctypes.POINTER(RunResult)],
            "hrm_photon_run_device": [vp, vp, vp, u32, ctypes.c_uint64, u32, u32, vp, ctypes.POINTER(RunConfig),
                                      ctypes.POINTER(RunResult)],
            "hrm_bfs_run": [vp, vp, u32, u32, vp, ctypes.POINTER(RunConfig), ctypes.POINTER(RunResult)],
            "hrm_bfs_run_device": [vp, vp, u32, u32, vp, ctypes.POINTER(RunConfig), ctypes.POINTER(RunResult)],
            "hrm_barrier_demo_run": [u32, u32, u32, vp, vp, ctypes.POINTER(RunConfig), ctypes.POINTER(RunResult)],
            "hrm_rmat_csr": [u32, u32, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_uint64, vp, vp],
            "hrm_photon_medium": [u32, ctypes.c_uint64, vp, vp, vp],
        }
        for name, args in sigs.items():
            f = getattr(L, name)
            f.restype = ctypes.c_int
            f.argtypes = args
        _lib = L
    return _lib


def check(rc):
    if rc != HRM_OK:
        raise HarmonizeError(rc, lib().hrm_last_error().decode(errors="replace"))
    return rc


def exported_symbols():
    """Names of the C entry points declared in include/hrm_capi.h."""
    hdr = os.path.join(os.path.dirname(HERE), "include", "hrm_capi.h")
    import re
    names = []
    for line in open(hdr):
        m = re.match(r"\s*(?:const\s+)?\w+\s*\*?\s*(hrm_\w+)\s*\(", line)
        if m:
            names.append(m.group(1))
    return names


def make_config(program="async", groups=0, cycles=0, chunk=0, arena=0, max_execs=0, stream=None, variant=0,
                patience=0, fill_links=0, job_order=0, solo_photons=0):
    pt = {"async": ASYNC, "event": EVENT}[program] if isinstance(program, str) else int(program)
    return RunConfig(pt, groups, cycles, chunk, arena, max_execs, stream, variant, patience, fill_links, job_order,
                     solo_photons)


def collatz(start, count, program="async", **kw):
    """Collatz stopping times of start .. start+count-1, from a whole GPU run.

    Returns (uint32 array, run-result dict)."""
    out = np.zeros(count, dtype=np.uint32)
    cfg = make_config(program, **kw)
    res = RunResult()
    check(lib().hrm_collatz_run(start, count, out.ctypes.data, ctypes.byref(cfg), ctypes.byref(res)))
    return out, res.as_dict()


PHOTON_SPREAD = 1024


def photon_medium(n, seed):
    """Seeded medium of an n^3 grid: (mu_s float32, absorb float32, split uint8)."""
    nv = n ** 3
    mu = np.empty(nv, dtype=np.float32)
    ab = np.empty(nv, dtype=np.float32)
    sp = np.empty(nv, dtype=np.uint8)
    if lib().hrm_photon_medium(n, seed, mu.ctypes.data, ab.ctypes.data, sp.ctypes.data) != 0:
        raise HarmonizeError(HRM_EINVAL, "bad medium arguments")
    return mu, ab, sp


def rmat_csr(scale, edge_factor=16, a=0.57, b=0.19, c=0.19, seed=1):
    """Seeded R-MAT graph as CSR (rowptr uint32[2^scale+1], col uint32[E])."""
    nv = 1 << scale
    rowptr = np.empty(nv + 1, dtype=np.uint32)
    col = np.empty(edge_factor * nv, dtype=np.uint32)
    if lib().hrm_rmat_csr(scale, edge_factor, a, b, c, seed, rowptr.ctypes.data, col.ctypes.data) != 0:
        raise HarmonizeError(HRM_EINVAL, "bad R-MAT arguments")
    return rowptr, col


def photon_walk(mu_s, absorb, split, n, seed, first, count, program="async", **kw):
    """Photon walk of photons [first, first+count) from host arrays.

    Returns (tally uint64[n^3 + 3*1024], run-result dict)."""
    mu_s = np.ascontiguousarray(mu_s, dtype=np.float32)
    absorb = np.ascontiguousarray(absorb, dtype=np.float32)
    split = np.ascontiguousarray(split, dtype=np.uint8)
    tally = np.zeros(n ** 3 + 3 * PHOTON_SPREAD, dtype=np.uint64)
    cfg = make_config(program, **kw)
    res = RunResult()
    check(lib().hrm_photon_run(mu_s.ctypes.data, absorb.ctypes.data, split.ctypes.data, n, seed, first, count,
                               tally.ctypes.data, ctypes.byref(cfg), ctypes.byref(res)))
    return tally, res.as_dict()


def bfs(rowptr, col, root=0, program="async", **kw):
    """Breadth-first levels from `root` (uint32, unreached 0xFFFFFFFF) from host arrays."""
    rowptr = np.ascontiguousarray(rowptr, dtype=np.uint32)
    col = np.ascontiguousarray(col, dtype=np.uint32)
    nv = len(rowptr) - 1
    levels = np.empty(nv, dtype=np.uint32)
    cfg = make_config(program, **kw)
    res = RunResult()
    check(lib().hrm_bfs_run(rowptr.ctypes.data, col.ctypes.data, nv, root, levels.ctypes.data, ctypes.byref(cfg),
                            ctypes.byref(res)))
    return levels, res.as_dict()


class Program:
    """One program instance of a built-in spec (the alloc/init/exec/complete/free life cycle).

    ``state`` is the spec's device-state struct as bytes (see include/hrm_capi.h); device
    pointers inside it are owned by the caller."""

    def __init__(self, spec, program="async", arena=0, state=b""):
        self.type = {"async": ASYNC, "event": EVENT}[program] if isinstance(program, str) else int(program)
        buf = ctypes.create_string_buffer(bytes(state), len(state))
        h = ctypes.c_void_p()
        check(lib().hrm_program_create(spec, self.type, arena, buf, len(state), ctypes.byref(h)))
        self.handle = h

    def init(self, groups=0, stream=None):
        check(lib().hrm_program_init(self.handle, groups or (1 << 30), stream))

    def exec(self, groups=0, n=0, stream=None):
        if n == 0:
            n = (1 << 24) if self.type == ASYNC else 1
        check(lib().hrm_program_exec(self.handle, groups or (1 << 30), n, stream))

    def complete(self):
        out = ctypes.c_int()
        check(lib().hrm_program_complete(self.handle, ctypes.byref(out)))
        return bool(out.value)

    def flags(self):
        out = ctypes.c_uint32()
        check(lib().hrm_program_flags(self.handle, ctypes.byref(out)))
        return out.value

    def clear_flags(self):
        check(lib().hrm_program_clear_flags(self.handle))

    def stats(self):
        arr = (ctypes.c_uint64 * len(STAT_NAMES))()
        check(lib().hrm_program_stats(self.handle, arr, len(STAT_NAMES)))
        return dict(zip(STAT_NAMES, [int(v) for v in arr]))

    def overview(self):
        arr = (ctypes.c_uint32 * 64)()
        n = ctypes.c_size_t()
        check(lib().hrm_program_overview(self.handle, arr, 64, ctypes.byref(n)))
        return [int(arr[i]) for i in range(min(n.value, 64))]

    def close(self):
        if getattr(self, "handle", None):
            lib().hrm_program_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def barrier_demo(dep_count, non_dep_count, barrier_count, program="async", **kw):
    """The remapping-barrier workload (examples/cpp/barrier_demo/demo.cpp:20-86 of Harmonize).

    Returns (counter uint32[4], released uint32[barrier_count], run-result dict); counter is
    (Steps run, non-dependent Steps, final Steps, violations)."""
    counter = np.zeros(4, dtype=np.uint32)
    released = np.zeros(max(barrier_count, 1), dtype=np.uint32)
    cfg = make_config(program, **kw)
    res = RunResult()
    check(lib().hrm_barrier_demo_run(dep_count, non_dep_count, barrier_count, counter.ctypes.data,
                                     released.ctypes.data, ctypes.byref(cfg), ctypes.byref(res)))
    return counter, released, res.as_dict()

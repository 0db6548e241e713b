"""The original Python front end's per-spec host symbol set (include/hrm_pyshim.h;
harmonize/python/templates.py:3-184, bound by name in harmonize/python/runtime.py:1324-1408).

CPU: every name the header declares is exported by libhrm.so, and the argument checks that
need no device reject bad calls with a message for hrm_last_error. GPU: a spec driven through
these names alone, the way the original's RuntimeSpec drives its generated shim (alloc_state,
store_state / store_pointer_state per field, alloc_program, init_program, exec_program until
complete, load_state), gives the oracle's output under both program kinds."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "hrm_pyshim.h")


def declared():
    out = subprocess.run(["gcc", "-E", "-P", "-x", "c", HEADER], capture_output=True, text=True, check=True).stdout
    return sorted(n for n in set(re.findall(r"\b(\w+)\s*\(", out)) if not n.startswith("__"))


def test_header_declares_the_templates_set():
    names = declared()
    for kind in ("event", "async"):
        for spec, fields in (("collatz", ["start", "limit", "output", "iterator", "leap"]),
                             ("photon", ["mu_s", "tally", "source", "n", "load_limit"]),
                             ("bfs", ["rowptr", "col", "levels", "roots", "root", "nv"])):
            s = f"{spec}_{kind}"
            for fn in ("alloc_state", "free_state", "alloc_program", "free_program", "init_program",
                       "exec_program", "complete", "clear_flags", "set_device"):
                assert f"{fn}_{s}" in names
            for f in fields:
                for fn in ("load_state", "store_state", "store_pointer_state"):
                    assert f"{fn}_{f}_{s}" in names


def test_library_exports_every_shim_symbol(hrm):
    out = subprocess.run(["nm", "-D", "--defined-only", hrm.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (\w+)", out))
    missing = [n for n in declared() if n not in exported]
    assert not missing, missing[:10]


def _fn(L, name, res, args):
    f = getattr(L, name)
    f.restype = res
    f.argtypes = args
    return f


vp, sz = ctypes.c_void_p, ctypes.c_size_t


def test_null_instances_are_reported_not_thrown(hrm):
    L = hrm.lib()
    assert _fn(L, "complete_collatz_async", ctypes.c_int, [vp])(None) == -1
    assert "instance is NULL" in L.hrm_last_error().decode()
    _fn(L, "exec_program_photon_event", None, [vp, sz, sz])(None, 4, 1)
    assert "instance is NULL" in L.hrm_last_error().decode()
    assert _fn(L, "alloc_program_bfs_async", vp, [vp, sz])(None, 1024) is None
    assert "device state is NULL" in L.hrm_last_error().decode()
    _fn(L, "store_pointer_state_leap_collatz_event", None, [vp, vp])(ctypes.c_void_p(0x1000), None)
    assert "not a pointer" in L.hrm_last_error().decode()


class Shim:
    """The handles runtime.py binds for one spec suffix."""

    def __init__(self, L, suffix, fields):
        self.suffix = suffix
        self.alloc_state = _fn(L, f"alloc_state_{suffix}", vp, [])
        self.free_state = _fn(L, f"free_state_{suffix}", None, [vp])
        self.alloc_program = _fn(L, f"alloc_program_{suffix}", vp, [vp, sz])
        self.free_program = _fn(L, f"free_program_{suffix}", None, [vp])
        self.init = _fn(L, f"init_program_{suffix}", None, [vp, sz])
        self.exec = _fn(L, f"exec_program_{suffix}", None, [vp, sz, sz])
        self.complete = _fn(L, f"complete_{suffix}", ctypes.c_int, [vp])
        self.clear_flags = _fn(L, f"clear_flags_{suffix}", None, [vp])
        self.set_device = _fn(L, f"set_device_{suffix}", None, [ctypes.c_int])
        self.store = {f: _fn(L, f"store_state_{f}_{suffix}", None, [vp, vp]) for f in fields}
        self.store_ptr = {f: _fn(L, f"store_pointer_state_{f}_{suffix}", None, [vp, vp]) for f in fields}
        self.load = {f: _fn(L, f"load_state_{f}_{suffix}", None, [vp, vp]) for f in fields}

    def run(self, state, size, grid, cycles, max_execs=100000):
        prog = self.alloc_program(state, size)
        assert prog
        try:
            self.init(prog, grid)
            for _ in range(max_execs):
                self.exec(prog, grid, cycles)
                c = self.complete(prog)
                assert c >= 0
                if c:
                    return
            raise AssertionError("did not complete")
        finally:
            self.free_program(prog)


def _u32(v):
    return ctypes.byref(ctypes.c_uint32(v))


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["async", "event"])
def test_collatz_through_the_shim(hrm, kind):
    import torch
    L = hrm.lib()
    sh = Shim(L, f"collatz_{kind}", ["start", "limit", "output", "iterator", "leap"])
    sh.set_device(0)
    start, count = 1, 1 << 16
    out = torch.zeros(count, dtype=torch.int32, device="cuda")
    it = torch.tensor([start, start + count], dtype=torch.int32, device="cuda")  # AtomicIter {value, limit}
    st = sh.alloc_state()
    assert st
    try:
        sh.store["start"](st, _u32(start))
        sh.store["limit"](st, _u32(start + count))
        sh.store_ptr["output"](st, ctypes.c_void_p(out.data_ptr()))
        sh.store_ptr["iterator"](st, ctypes.c_void_p(it.data_ptr()))
        sh.store["leap"](st, _u32(1))
        got = ctypes.c_uint32()
        sh.load["limit"](ctypes.byref(got), st)
        assert got.value == start + count
        sh.run(st, 1 << 16, 296, (1 << 24) if kind == "async" else 1)
    finally:
        sh.free_state(st)
    torch.cuda.synchronize()
    assert np.array_equal(out.cpu().numpy().view(np.uint32), oracle.collatz_range(start, count))


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["async", "event"])
def test_photon_through_the_shim(hrm, kind):
    import torch
    L = hrm.lib()
    fields = ["mu_s", "absorb", "split", "tally", "source", "n", "seed_lo", "seed_hi", "leap", "load_limit"]
    sh = Shim(L, f"photon_{kind}", fields)
    n, seed, first, count = 16, 0xC0FFEE, 0, 3000
    mu, ab, sp = oracle.photon_medium(n, 11)
    d = [torch.from_numpy(x).cuda() for x in (mu, ab, sp)]
    tally = torch.zeros(n ** 3 + 3 * 1024, dtype=torch.int64, device="cuda")
    it = torch.tensor([first, first + count], dtype=torch.int32, device="cuda")
    st = sh.alloc_state()
    try:
        for f, t in zip(("mu_s", "absorb", "split", "tally", "source"), d + [tally, it]):
            sh.store_ptr[f](st, ctypes.c_void_p(t.data_ptr()))
        sh.store["n"](st, _u32(n))
        sh.store["seed_lo"](st, _u32(seed & 0xFFFFFFFF))
        sh.store["seed_hi"](st, _u32(seed >> 32))
        sh.store["leap"](st, _u32(1))
        sh.store["load_limit"](st, ctypes.byref(ctypes.c_float(0.25)))
        sh.run(st, (1 << 16) if kind == "async" else (1 << 20), 296, (1 << 24) if kind == "async" else 1)
    finally:
        sh.free_state(st)
    ref, _ = oracle.photon_walk(mu, ab, sp, n, seed, first, count)
    assert np.array_equal(tally.cpu().numpy().view(np.uint64), ref)

"""CPU tests of the C ABI boundary: the library loads, exports every entry point declared in
include/hrm_capi.h, and rejects bad arguments with status codes (no GPU needed)."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "hrm_capi.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(hrm_\w+)\s*\(", text)))


def test_header_declares_the_life_cycle():
    names = declared_functions()
    for n in ["hrm_program_create", "hrm_program_init", "hrm_program_exec", "hrm_program_complete",
              "hrm_program_clear_flags", "hrm_program_destroy", "hrm_last_error", "hrm_collatz_run",
              "hrm_photon_run", "hrm_bfs_run", "hrm_collatz_run_device_noalloc"]:
        assert n in names


def test_variant_table_matches_the_header(hrm):
    """Every HRM_VARIANT_* the header defines, and no other, has a (ring links, teams per CTA)
    entry in the package's variant table, and the ring and team counts in each name agree."""
    text = open(HEADER).read()
    defined = dict((n, int(v)) for n, v in re.findall(r"#define HRM_VARIANT_(\w+) (\d+)", text))
    count = defined.pop("COUNT")
    assert sorted(defined.values()) == list(range(count)) == sorted(hrm.VARIANTS)
    for name, v in defined.items():
        m = re.match(r"R(\d+)_T(\d+)", name)
        if m:
            assert hrm.VARIANTS[v] == (int(m.group(1)), int(m.group(2))), name


def test_library_exports_every_declared_symbol(hrm):
    lib = ctypes.CDLL(hrm.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", hrm.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (hrm_\w+)", out))
    assert set(declared_functions()) <= exported


def test_header_compiles_as_c():
    r = subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-fsyntax-only", "-x", "c", HEADER],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_spec_members_are_honoured_at_compile_time(tmp_path):
    """tests/cpp/spec_traits.cu: static checks that optional spec members (ring sizes, teams,
    patience, pop order, ring groups, and their per-function forms) reach the runtime and that
    omitted ones take their defaults. nvcc cross-compiles it here; no kernel runs."""
    src = os.path.join(ROOT, "tests", "cpp", "spec_traits.cu")
    r = subprocess.run(["nvcc", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a",
                        "-I", os.path.join(ROOT, "include"), "-c", src, "-o", str(tmp_path / "traits.o")],
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr


def test_co_residency_arithmetic_at_compile_time(tmp_path):
    """tests/cpp/occupancy.cu: static checks of the CTAs-beside arithmetic that sizes the
    serving session's resident share and solo photon kernel (B200 per-SM limits, registers per
    sub-partition). nvcc cross-compiles it here; no kernel runs."""
    src = os.path.join(ROOT, "tests", "cpp", "occupancy.cu")
    r = subprocess.run(["nvcc", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a",
                        "-I", os.path.join(ROOT, "include"), "-c", src, "-o", str(tmp_path / "occupancy.o")],
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr


def test_bad_arguments_return_einval(hrm):
    L = hrm.lib()
    res = hrm.RunResult()
    cfg = hrm.make_config("async")
    assert L.hrm_photon_run(None, None, None, 16, 1, 0, 10, None, ctypes.byref(cfg), ctypes.byref(res)) == hrm.HRM_EINVAL
    assert L.hrm_bfs_run(None, None, 4, 0, None, ctypes.byref(cfg), ctypes.byref(res)) == hrm.HRM_EINVAL
    assert L.hrm_collatz_run(0, 10, None, ctypes.byref(cfg), ctypes.byref(res)) == hrm.HRM_EINVAL
    h = ctypes.c_void_p()
    state = ctypes.create_string_buffer(8)
    rc = L.hrm_program_create(hrm.SPEC_COLLATZ, hrm.ASYNC, 0, state, 8, ctypes.byref(h))
    assert rc == hrm.HRM_EINVAL and b"state size" in L.hrm_last_error()
    rc = L.hrm_program_create(99, hrm.ASYNC, 0, state, 8, ctypes.byref(h))
    assert rc == hrm.HRM_EINVAL
    assert L.hrm_program_complete(None, None) == hrm.HRM_EINVAL


def test_job_and_input_entry_points_reject_bad_arguments(hrm):
    """The batch, serving and input entry points check their arguments before any CUDA call."""
    L = hrm.lib()
    vp, u32 = ctypes.c_void_p, ctypes.c_uint32
    out = vp()
    assert L.hrm_server_open(u32(0), None, ctypes.byref(out)) == hrm.HRM_EINVAL       # zero capacity
    assert L.hrm_server_open(u32(4), None, None) == hrm.HRM_EINVAL                    # no handle
    first = u32()
    assert L.hrm_server_submit(None, None, u32(0), ctypes.byref(first)) == hrm.HRM_EINVAL
    assert L.hrm_server_poll(None, None, u32(0), None) == hrm.HRM_EINVAL
    assert L.hrm_server_close(None, u32(10)) == hrm.HRM_EINVAL
    assert L.hrm_server_destroy(None) == hrm.HRM_OK                                   # like free(NULL)
    assert L.hrm_batch_run(None, u32(3), None, None, None) == hrm.HRM_EINVAL
    assert L.hrm_plain_run(None, u32(3), u32(4), None, None) == hrm.HRM_EINVAL
    assert L.hrm_runtime_run(None, u32(3), 0, None, None, None) == hrm.HRM_EINVAL
    assert L.hrm_serve_replay(None, u32(3), None, 0, u32(1), None, None, None) == hrm.HRM_EINVAL
    from harmonize_b200 import jobs
    J = jobs._bind()
    assert J.hrm_solo_run(None, u32(3), 7, u32(2), None, None) == hrm.HRM_EINVAL       # no jobs
    one = (jobs.Job * 1)()
    one[0] = jobs.Job(jobs.JOB_COLLATZ, 1, 16, 0, 0, None, None, None, 0x1000)
    assert J.hrm_solo_run(ctypes.byref(one), u32(1), 7, u32(0), None, None) == hrm.HRM_EINVAL   # no lane
    assert J.hrm_solo_run(ctypes.byref(one), u32(1), 7, u32(9), None, None) == hrm.HRM_EINVAL   # too many
    assert J.hrm_solo_run(ctypes.byref(one), u32(1), 7, u32(2), None, None) == hrm.HRM_EINVAL   # not photon
    assert "photon jobs only" in hrm.lib().hrm_last_error().decode()
    rp = np.zeros(5, dtype=np.uint32)
    col = np.zeros(16, dtype=np.uint32)
    assert L.hrm_rmat_csr(2, 4, ctypes.c_double(0.6), ctypes.c_double(0.3), ctypes.c_double(0.3), ctypes.c_uint64(1),
                          rp.ctypes.data, col.ctypes.data) == 1                       # a + b + c > 1
    assert L.hrm_rmat_csr(0, 4, ctypes.c_double(0.5), ctypes.c_double(0.2), ctypes.c_double(0.2), ctypes.c_uint64(1),
                          rp.ctypes.data, col.ctypes.data) == 1                       # scale 0
    mu = np.zeros(8, dtype=np.float32)
    assert L.hrm_photon_medium(0, ctypes.c_uint64(1), mu.ctypes.data, mu.ctypes.data, None) == 1


def test_product_fails_loudly_without_its_library(monkeypatch, tmp_path):
    import harmonize_b200 as h
    monkeypatch.setattr(h, "_lib", None)
    monkeypatch.setattr(h, "LIB_PATH", str(tmp_path / "missing.so"))
    with pytest.raises(h.HarmonizeError):
        h.collatz(0, 10)


def test_inputs_are_deterministic(hrm):
    rp1, c1 = hrm.rmat_csr(12, 8, seed=9)
    rp2, c2 = hrm.rmat_csr(12, 8, seed=9)
    assert np.array_equal(rp1, rp2) and np.array_equal(c1, c2)
    assert rp1[-1] == len(c1) == 8 << 12 and np.all(np.diff(rp1.astype(np.int64)) >= 0)
    m1 = hrm.photon_medium(8, 3)
    m2 = hrm.photon_medium(8, 3)
    assert all(np.array_equal(a, b) for a, b in zip(m1, m2))
    mu, ab, sp = hrm.photon_medium(64, 1)
    assert abs(np.log(mu).mean()) < 0.01 and abs(np.log(mu).std() - 0.5) < 0.01
    assert ab.min() >= 0.02 and ab.max() <= 0.2 and abs(sp.mean() - 0.1) < 0.01


def test_ctypes_structs_match_the_c_layout(hrm, tmp_path):
    """The Python mirrors of hrm_run_config / hrm_run_result / hrm_job have the C layout."""
    from harmonize_b200 import jobs
    src = tmp_path / "layout.c"
    src.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "hrm_capi.h"\n'
                   'int main(void) {\n'
                   '  printf("%zu %zu %zu %zu\\n", sizeof(hrm_run_config), offsetof(hrm_run_config, variant),\n'
                   '         offsetof(hrm_run_config, patience), offsetof(hrm_run_config, fill_links));\n'
                   '  printf("%zu %zu\\n", offsetof(hrm_run_config, job_order), offsetof(hrm_run_config, solo_photons));\n'
                   '  printf("%zu %zu\\n", sizeof(hrm_run_result), offsetof(hrm_run_result, device_ms));\n'
                   '  printf("%zu %zu\\n", sizeof(hrm_job), offsetof(hrm_job, out));\n'
                   '  return 0;\n}\n')
    exe = tmp_path / "layout"
    r = subprocess.run(["gcc", "-std=c99", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    got = [list(map(int, line.split())) for line in subprocess.check_output([str(exe)], text=True).splitlines()]
    C = hrm.RunConfig
    assert got[0] == [ctypes.sizeof(C), C.variant.offset, C.patience.offset, C.fill_links.offset]
    assert got[1] == [C.job_order.offset, C.solo_photons.offset]
    assert got[2] == [ctypes.sizeof(hrm.RunResult), hrm.RunResult.device_ms.offset]
    assert got[3] == [ctypes.sizeof(jobs.Job), jobs.Job.out.offset]


def _noalloc(hrm):
    f = hrm.lib().hrm_collatz_run_device_noalloc
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_void_p, ctypes.POINTER(hrm.RunConfig),
                  ctypes.POINTER(hrm.RunResult)]
    return f


@pytest.mark.parametrize("cfg_kw,message", [
    (dict(program="async", arena=4097), "exceeds the no-allocation maximum"),
    (dict(program="event"), "AsyncProgram only"),
    (dict(program="async", variant=2), "tuning variant 0 only"),
])
def test_noalloc_rejects_bad_configs_before_any_cuda_call(hrm, cfg_kw, message):
    """The no-allocation entry point checks its arguments before it touches the device: an
    arena beyond HRM_NOALLOC_MAX_ARENA_LINKS, EventProgram and other variants are refused with
    HRM_EINVAL. The output pointer is a dummy that is never dereferenced."""
    f = _noalloc(hrm)
    cfg = hrm.make_config(**cfg_kw)
    res = hrm.RunResult()
    rc = f(0, 16, ctypes.c_void_p(0x1000), ctypes.byref(cfg), ctypes.byref(res))
    assert rc == hrm.HRM_EINVAL
    assert message in hrm.lib().hrm_last_error().decode()


def test_noalloc_rejects_null_output_and_overflowing_range(hrm):
    f = _noalloc(hrm)
    cfg = hrm.make_config("async")
    res = hrm.RunResult()
    assert f(0, 16, None, ctypes.byref(cfg), ctypes.byref(res)) == hrm.HRM_EINVAL
    assert f(0xFFFFFFF0, 0x20, ctypes.c_void_p(0x1000), ctypes.byref(cfg), ctypes.byref(res)) == hrm.HRM_EINVAL

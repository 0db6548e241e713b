"""The reference's own example programs, unchanged, running on this runtime on the GPU.

oracle/ref_build.py (build_examples) compiles them where they lie in the reference tree with
this runtime's include/harmonize.h forced in, into oracle/_ref/examples (the binaries travel
with the repository; the reference tree does not):

  * clz_hrm_event: examples/cpp/collaz/collaz_hrm.cpp as it is (EventProgram);
  * clz_hrm_async: the same file with the README's one-line swap to AsyncProgram;
  * neut: examples/cpp/example_neutron/program.cpp, which instantiates both program types and
    picks one with `-async`.
The Collatz program checks its own output against its host `checker` over every index and
prints "Bad output ..." for each mismatch, then "Runtime: <ms>" (collaz_hrm.cpp:236-244).
The neutron program prints its census tallies as CSV (program.cpp:340-372). Each neutron's
history is a pure function of its id (its seed), and with implicit capture off every weight is
1.0, so the float tallies are exact integer counts: both program types must print the same
line, and with scattering alone (no capture, no fission, a medium no neutron leaves before the
census) the tallies must add up to every source neutron.
"""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "oracle", "_ref", "examples")


def run(name, *args, timeout=300):
    path = os.path.join(BIN, name)
    if not os.path.exists(path):
        pytest.skip(f"{path} not built (python -m oracle.ref_build --examples, where the reference tree is)")
    r = subprocess.run([path] + [str(a) for a in args], capture_output=True, text=True, timeout=timeout)
    assert r.returncode == 0, f"{name} exited {r.returncode}: {r.stdout[-2000:]} {r.stderr[-2000:]}"
    return r.stdout


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["clz_hrm_event", "clz_hrm_async"])
@pytest.mark.parametrize("limit", [1000, 1 << 20])
def test_collatz_example_checks_itself(name, limit):
    out = run(name, "-wg_count", 296, "-limit", limit)
    assert "Bad output" not in out, out[:2000]
    assert "Runtime:" in out


def neutron_csv(program, **kw):
    args = {"wg_count": 296, "num": 100000, "time": 1.0, "res": 0.25, "size": 4.0, "pool": 1 << 24,
            "hrzn": 1, "csv": "true", "async": "true" if program == "async" else "false"}
    args.update(kw)
    argv = []
    for k, v in args.items():
        argv += [f"-{k}", v]
    out = run("neut", *argv).strip().splitlines()
    line = [l for l in out if "," in l][-1]
    return line, np.array([float(x) for x in line.split(",")])


@pytest.mark.gpu
@pytest.mark.parametrize("program", ["async", "event"])
def test_neutron_example_conserves_weight_without_absorption(program):
    line, t = neutron_csv(program, sx=1.0, fx=0.0, cx=0.0)
    assert len(t) == 32
    # printed values are count / num / res with 6 decimals
    assert abs(t.sum() * 0.25 - 1.0) < 32 * 1e-6 + 1e-6


@pytest.mark.gpu
def test_neutron_example_same_tallies_under_both_program_types():
    kw = dict(sx=1.0, fx=0.3, cx=0.4, mult=2)
    a, ta = neutron_csv("async", **kw)
    e, te = neutron_csv("event", **kw)
    assert a == e
    assert 0.0 < ta.sum() * 0.25

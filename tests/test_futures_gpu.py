"""Futures (async/future.h of the original) on the GPU: values passed back up a call tree.

tests/cpp/futures.cu sums a complete binary tree: every inner node holds a continuation on its
own Future (a RemappingBarrier with semaphore 2), starts its two children, and each child
stores its value and fulfills its parent's future; the continuation adds the two values once
both are in. The program checks every node's sum against the host and exits nonzero on a
mismatch."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "futures.cu")


@pytest.mark.gpu
@pytest.mark.parametrize("levels", [1, 10, 16])
def test_future_tree_sums(tmp_path, levels):
    exe = tmp_path / "futures"
    subprocess.run(["nvcc", "-std=c++17", "-O3", "-gencode", "arch=compute_100a,code=sm_100a",
                    "-I", os.path.join(ROOT, "include"), SRC, "-o", str(exe)], check=True, capture_output=True,
                   timeout=600)
    out = tmp_path / "sums.bin"
    r = subprocess.run([str(exe), str(levels), str(out)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    sums = np.fromfile(out, dtype=np.uint32)
    leaves = 1 << levels
    vals = ((np.arange(leaves, dtype=np.uint64) * 2654435761) & 0xFFFFFFFF) >> 7
    assert sums.size == 2 * leaves - 1
    assert int(sums[0]) == int(vals.sum()) & 0xFFFFFFFF

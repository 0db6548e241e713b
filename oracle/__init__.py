"""CPU oracle for the B200 Harmonize runtime — TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py``
may import this package. The product (``harmonize_b200``) never imports, links or runs
anything here; its GPU path fails loudly when its CUDA library is missing.

Contents:
  * plain-C restatements of the reference's checkers and of the workloads' algorithms
    (``collatz.c``, ``bfs.c``, ``photon.c``), each citing the reference file it follows;
  * host executors (``host_exec.cpp``) that run the very same spec sources as the GPU
    runtime, serially and with OpenMP — Harmonize itself has no CPU executor;
  * ``build.py``, which compiles the above into ``oracle/_build/liboracle.so`` and, when
    the reference tree is present, the reference CUDA build into ``oracle/_ref``.

Parity pins: the Collatz restatement is checked against known stopping times and against
the reference runtime's own outputs committed under ``tests/golden``.
"""
from .lib import load, collatz_range  # noqa: F401

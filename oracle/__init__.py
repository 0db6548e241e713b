"""CPU oracle for the B200 Harmonize runtime — TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline / reference legs of
``bench.py`` may import this package. The product (``harmonize_b200``) never imports, links
or runs anything here; its GPU path fails loudly when its CUDA library is missing.

Contents:
  * plain-C restatements of the reference's checker and of the workloads' algorithms
    (``collatz.c`` after examples/cpp/collaz/collaz_hrm.cpp:157-168, ``bfs.c``,
    ``photon.c``);
  * host executors (``host_exec.cpp``) that run the very same spec sources as the GPU
    runtime, serially and with OpenMP — Harmonize itself has no CPU executor;
  * ``build.py``, which compiles the above into ``oracle/_build/liboracle.so``;
    ``ref_build.py`` builds the reference CUDA build of the same specs into ``oracle/_ref``.

Parity pins: the Collatz restatement is checked against known stopping times and the
reference runtime's own outputs (``tests/golden``); the photon and BFS restatements agree
bit for bit with the host executors of the spec sources and with the reference runtime.
"""
from .lib import (load, max_threads, collatz_range, exec_collatz, bfs, exec_bfs,  # noqa: F401
                  photon_walk, exec_photon, photon_medium, rmat_csr, philox, log, PHOTON_SPREAD,
                  ref_load, ref_collatz, ref_photon_device, ref_bfs_device, REF_WG, REF_CYCLES,
                  REF_PHOTON_SHAPE, REF_ASYNC_CLOSED_PHOTON, REF_ASYNC_CLOSED_BFS)

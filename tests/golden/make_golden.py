"""Generates the golden fixtures in tests/golden from the ORIGINAL Harmonize runtime.

Runs the built-in spec sources on the reference CUDA build (oracle/_ref/libhrm_ref.so, built
from the reference's own headers by oracle/ref_build.py) on a GPU, and stores its outputs:

  * ref_collatz_0_4096.npy       stopping times of 0..4095 (AsyncProgram; EventProgram agrees)
  * ref_photon_n16_s99_500.npy   uint64 tallies of 500 photons on a 16^3 medium (seed 11),
                                 EventProgram (the reference AsyncProgram faulted on this spec)
  * ref_bfs_rmat10.npz           R-MAT 2^10 graph (seed 5) and its BFS levels from vertex 0,
                                 EventProgram

    python tests/golden/make_golden.py OUTDIR
The CPU tests compare the oracle's restatements with these files.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))


def main(outdir):
    import torch
    import harmonize_b200 as hrm
    import oracle
    os.makedirs(outdir, exist_ok=True)
    steps, _ = oracle.ref_collatz(0, 4096, program="async")
    np.save(os.path.join(outdir, "ref_collatz_0_4096.npy"), steps)
    steps_e, _ = oracle.ref_collatz(0, 4096, program="event")
    assert np.array_equal(steps, steps_e), "reference AsyncProgram and EventProgram disagree"

    mu, ab, sp = hrm.photon_medium(16, 11)
    d_mu, d_ab, d_sp = (torch.from_numpy(x).cuda() for x in (mu, ab, sp))
    d_t = torch.zeros(16 ** 3 + 3 * 1024, dtype=torch.int64, device="cuda")
    oracle.ref_photon_device(d_mu.data_ptr(), d_ab.data_ptr(), d_sp.data_ptr(), 16, 99, 0, 500, d_t.data_ptr())
    tally = d_t.cpu().numpy().view(np.uint64).copy()
    np.save(os.path.join(outdir, "ref_photon_n16_s99_500.npy"), tally)
    np.savez_compressed(os.path.join(outdir, "medium_n16_seed11.npz"), mu=mu, ab=ab, sp=sp)

    rp, col = hrm.rmat_csr(10, 16, 0.57, 0.19, 0.19, 5)
    d_rp = torch.from_numpy(rp.view(np.int32)).cuda()
    d_col = torch.from_numpy(col.view(np.int32)).cuda()
    d_lev = torch.empty(len(rp) - 1, dtype=torch.int32, device="cuda")
    oracle.ref_bfs_device(d_rp.data_ptr(), d_col.data_ptr(), len(rp) - 1, 0, d_lev.data_ptr())
    levels = d_lev.cpu().numpy().view(np.uint32).copy()
    np.savez_compressed(os.path.join(outdir, "ref_bfs_rmat10.npz"), rowptr=rp, col=col, levels=levels)
    print("golden fixtures written to", outdir)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else HERE)

"""Regenerate the golden fixtures from the FP64 oracle.

The reference (Julia) cannot run in this environment; the oracle that writes
these fixtures is itself pinned against the reference's known-answer tests
(tests/test_oracle.py).  The fixtures freeze the cluster tree (sklearn
KMeans), the block partition and the FP64 results of the README case so that
GPU runs compare against the same numbers everywhere.

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from oracle import hm_oracle as O  # noqa: E402


def main():
    out = {}
    rng = np.random.default_rng(0)
    y = rng.random(2000)
    out["y"] = y
    for mr in (5, 25):
        prm = O.Params(Geom=np.linspace(0, 10, 2000), Kernel=O.kernel_cauchy(), MaxBlock=500,
                       MinBlock=64, MaxRank=mr, ConsMethod="svd")
        c, H = O.NewHmat(prm)
        ca = O.cluster_arrays(c)
        out["perm"] = ca["perm"]
        out["cl_s"], out["cl_e"], out["cl_left"], out["cl_right"] = ca["s"], ca["e"], ca["left"], ca["right"]
        out["blocks%d" % mr] = np.asarray(O.block_list(H), np.int64)
        out["Hy%d" % mr] = O.matvec(H, y)
        out["HTy%d" % mr] = O.vec_mat(y, H)[0]
        Hs = O.add_identity(H, 10.0)
        L = O.lu(Hs, prm)
        out["P_shift%d" % mr] = L.P
        out["x_shift%d" % mr] = O.solve(L, y)
        if mr == 25:
            L0 = O.lu(H, prm)
            out["P_noshift25"] = L0.P
    np.savez_compressed(os.path.join(os.path.dirname(os.path.abspath(__file__)), "readme_case.npz"), **out)


if __name__ == "__main__":
    main()

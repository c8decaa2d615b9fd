"""Writes the golden fixtures of this directory from the HPCG 3.1 reference itself.

The reference is built from its own sources into oracle/_ref/libhpcg_ref.so
(`make -C oracle ref`); this script drives its routines through
oracle/ref_bridge.cpp and stores their outputs:

  golden_16.npz   16^3: b, xexact, a seeded x, ComputeSPMV_ref(x), ComputeSYMGS_ref(b, x),
                  ComputeMG_ref(x), CG_ref scaled residual after k = 1..20 iterations, the
                  CG_ref solution after 10 iterations; and the same CG_ref history on the
                  colour-permuted hierarchy (the library's row order), with that order.
  golden_32.json  32^3 known answers: initial residual, scaled residuals after
                  1/10/20/23/50 iterations, TestCG iteration counts, nonzeros per level,
                  and the HPCG flop count of one 50-iteration set.

Run from the repository root:  python tests/golden/make_golden.py
"""
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from hpcg_b200 import binding as B  # noqa: E402
from hpcg_b200 import metrics  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))
SEED = 0x48504347


def history(R, kmax, x0=None):
    out = []
    for k in range(1, kmax + 1):
        _, ni, nr, nr0 = R.cg(k, 0.0, True, x0)
        assert ni == k
        out.append(nr / nr0)
    return np.array(out)


def main():
    assert O.have_reference(), "build oracle/_ref first: make -C oracle ref"
    n = 16
    R = O.Reference(n)
    b, x0, xe = R.vectors()
    xs = np.random.default_rng(SEED).random(n ** 3)
    spmv = R.spmv(xs)
    symgs = R.symgs(b, xs)
    mg = R.mg(xs)
    _, _, nr, nr0 = R.cg(1, 0.0)
    normr0 = nr0
    hist = history(R, 20)
    x10, _, _, _ = R.cg(10, 0.0)
    # colour-permuted hierarchy
    perms = [B.colour_permutation(n >> l, n >> l, n >> l)[0] for l in range(4)]
    Rp = O.Reference(n)
    Rp.permute(perms)
    hist_perm = history(Rp, 20)
    np.savez_compressed(os.path.join(OUT, "golden_16.npz"), b=b, xexact=xe, x_seed=xs, spmv=spmv, symgs=symgs,
                        mg=mg, normr0=normr0, cg_hist=hist, cg_x10=x10, perm0=perms[0], cg_hist_perm=hist_perm)

    n = 32
    R = O.Reference(n)
    _, _, nr, nr0 = R.cg(50, 0.0)
    res = {"n": n, "normr0": nr0, "scaled_residual": {}}
    for k in (1, 10, 20, 23, 50):
        _, _, nr, nr0 = R.cg(k, 0.0)
        res["scaled_residual"][str(k)] = nr / nr0
    res["testcg"] = R.test_cg()
    res["nnz_per_level"] = [int(R.l.ref_level_nnz(R.h, l)) for l in range(4)]
    res["flops_50"] = metrics.hpcg_flops(n, n, n, 50)
    with open(os.path.join(OUT, "golden_32.json"), "w") as f:
        json.dump(res, f, indent=1)
    print("wrote golden_16.npz and golden_32.json")


if __name__ == "__main__":
    main()

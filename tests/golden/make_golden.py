"""Writes tests/golden/golden.npz: outputs of the FP64 oracle (oracle/) on small
seeded inputs, so that later changes to the oracle or to the GPU kernels are
checked against fixed numbers rather than only against each other.

    python tests/golden/make_golden.py

The inputs are not stored: they are regenerated from the seeds below with
grid-mg-bench_b200/inputs.py (numpy PCG64), by this script and by the tests
alike.  Index tables are compared bit for bit, floating-point outputs to
relative squared deviation 1e-26.

The reference itself cannot be built here (it needs Grid) and ships no golden
vectors, so these fixtures pin the restatement against regressions; its
agreement with the reference rests on the identities of tests/test_oracle*.py.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
for p in (os.path.join(ROOT, "grid-mg-bench_b200"), os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)

import inputs  # noqa: E402
import oracle as orc  # noqa: E402

FD, CD = (4, 4, 4, 4), (2, 2, 2, 2)
COARSE_DIMS = (2, 2, 2, 2)
NB_DIMS = (4, 2, 2, 2)
N_COARSE, R_COARSE = 8, 2
MASS, CSW = -0.1, 1.0


def case_inputs():
    """The seeded inputs of every fixture (the tests call this too)."""
    links = inputs.random_links(COARSE_DIMS, N_COARSE, inputs.rng(stream=901))
    x = inputs.gaussian_field((inputs.vol(COARSE_DIMS), R_COARSE, N_COARSE), inputs.rng(stream=902))
    U = inputs.hot_gauge(FD, inputs.rng(stream=903))
    psi = inputs.gaussian_field((inputs.vol(FD), 2, 12), inputs.rng(stream=904))
    h = inputs.gaussian_field((2, inputs.vol(FD), 12), inputs.rng(stream=905))
    B = orc.block_orthonormalise(FD, CD, orc.chiral_double(h, 0.5), passes=1)
    f = inputs.gaussian_field((inputs.vol(FD), 3, 12), inputs.rng(stream=906))
    return dict(links=links, x=x, U=U, psi=psi, B=B, f=f)


def compute(inp):
    cl = orc.clover_build(FD, inp["U"], CSW)
    lut, sizes, rev = orc.lut(FD, CD)
    return {
        "nbr_4x2x2x2": orc.coarse_neighbors(NB_DIMS),
        "lut_4x4x4x4_2x2x2x2": lut,
        "lut_rev_4x4x4x4_2x2x2x2": rev,
        "coarse_m": orc.coarse_apply(COARSE_DIMS, inp["links"], inp["x"], op=orc.OP_M),
        "coarse_mdag": orc.coarse_apply(COARSE_DIMS, inp["links"], inp["x"], op=orc.OP_MDAG),
        "wilson_m": orc.wilson_clover(FD, inp["U"], cl, MASS, 1, inp["psi"]),
        "project": orc.block_project(FD, CD, inp["B"], inp["f"]),
        "coarsen_links": orc.coarsen_wilson(FD, CD, inp["B"], inp["U"], cl, MASS, 1, 0, variant=1),
    }


if __name__ == "__main__":
    out = compute(case_inputs())
    np.savez_compressed(os.path.join(HERE, "golden.npz"), **out)
    print({k: v.shape for k, v in out.items()})

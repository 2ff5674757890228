"""The committed golden fixtures (tests/golden/golden.npz, written by
tests/golden/make_golden.py from the FP64 oracle on seeded inputs).

CPU: the oracle still reproduces them, and the library's host-side lookup
table (CoarseningLookupTable::populate, CoarseningLookupTableRework.h:114-179)
matches bit for bit.  GPU: the FP64 kernels (coarse M / Mdag, Wilson-clover M,
block projection, CoarsenOperator) reproduce them on the same inputs."""
import os
import sys

import numpy as np
import pytest

import gmg
import oracle as orc

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import make_golden as mg  # noqa: E402

GOLD = np.load(os.path.join(HERE, "golden", "golden.npz"))


@pytest.fixture(scope="module")
def case():
    return mg.case_inputs()


def test_oracle_reproduces_golden(case):
    got = mg.compute(case)
    assert set(got) == set(GOLD.files)
    for k, v in got.items():
        if np.issubdtype(v.dtype, np.integer):
            assert np.array_equal(v, GOLD[k]), k
        else:
            assert orc.rel_dev_sq(GOLD[k], v) < 1e-26, k


def test_library_lut_matches_golden():
    l, _, r = gmg.lut_build(mg.FD, mg.CD)
    assert np.array_equal(l, GOLD["lut_4x4x4x4_2x2x2x2"])
    assert np.array_equal(r, GOLD["lut_rev_4x4x4x4_2x2x2x2"])


@pytest.mark.gpu
def test_gpu_kernels_match_golden(case):
    import torch

    dev = "cuda:0"
    tol = 1e-24

    def t(a):
        return torch.from_numpy(np.ascontiguousarray(a)).to(dev)

    cm = gmg.CoarsenedMatrix(mg.COARSE_DIMS, mg.N_COARSE)
    cm.set_links(case["links"])
    for op, key in (("M", "coarse_m"), ("Mdag", "coarse_mdag")):
        y = torch.zeros((16, mg.R_COARSE, mg.N_COARSE), dtype=torch.complex128, device=dev)
        getattr(cm, op)(t(case["x"]), y)
        assert orc.rel_dev_sq(GOLD[key], y.cpu().numpy()) < tol, key

    w = gmg.WilsonClover(mg.FD, mg.MASS, mg.CSW, antiperiodic=1)
    w.set_gauge(case["U"])
    y = torch.zeros((256, 2, 12), dtype=torch.complex128, device=dev)
    w.M(t(case["psi"]), y)
    assert orc.rel_dev_sq(GOLD["wilson_m"], y.cpu().numpy()) < tol

    ag = gmg.Aggregation(mg.FD, mg.CD, 12, 4)
    ag.set_basis(case["B"])
    c = torch.zeros((16, 3, 4), dtype=torch.complex128, device=dev)
    ag.ProjectToSubspace(t(case["f"]), c)
    assert orc.rel_dev_sq(GOLD["project"], c.cpu().numpy()) < tol

    cc = gmg.CoarsenedMatrix(mg.CD, 4)
    cc.CoarsenOperator(ag, w)
    got = cc.get_links()
    for p in range(9):
        assert orc.rel_dev_sq(GOLD["coarsen_links"][p], got[p]) < tol, p

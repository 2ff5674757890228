"""Red-black coarse operator on the GPU against the FP64 oracle
(Rework::CoarsenedMatrix, include/CoarsenedMatrixRework.h:178-245, 288-394, 617-679).

Tolerances (relative squared deviation |ref-res|^2/|ref|^2): FP64 1e-24 (same
arithmetic, different summation order), FP32 1e-10, BF16 tensor-core hops
2e-5 (BF16 operands, FP32 accumulation).  Checkerboard gathers are bit-exact.
"""
import numpy as np
import pytest
import torch

import gmg
import inputs
import oracle as orc

pytestmark = pytest.mark.gpu

DIMS, N, R = (4, 4, 4, 8), 16, 6


@pytest.fixture(scope="module")
def links():
    # gamma5-hermitian Gaussian links with a shifted (invertible) self link
    return inputs.random_links(DIMS, N, inputs.rng(stream=901), diag_shift=2.0)


@pytest.fixture(scope="module")
def cm(links):
    m = gmg.CoarsenedMatrix(DIMS, N)
    m.set_links(links)
    m.prepare("f32")
    m.prepare("bf16")
    m.InvertSelfStencilPoint()
    return m


def dev(x, dt=torch.complex128):
    return torch.from_numpy(np.ascontiguousarray(x)).cuda().to(dt)


def host(t):
    return t.cpu().numpy().astype(np.complex128)


def test_checkerboard_round_trip_bit_exact():
    x = inputs.gaussian_field((512, R, N), inputs.rng(stream=902))
    xd = dev(x)
    for cb in (0, 1):
        h = torch.zeros((256, R, N), dtype=torch.complex128, device="cuda")
        gmg.pick_checkerboard(DIMS, cb, xd, h)
        assert np.array_equal(host(h), orc.pick_checkerboard(DIMS, cb, x))
    e = torch.zeros((256, R, N), dtype=torch.complex128, device="cuda")
    o = torch.zeros_like(e)
    gmg.pick_checkerboard(DIMS, 0, xd, e)
    gmg.pick_checkerboard(DIMS, 1, xd, o)
    back = torch.zeros_like(xd)
    gmg.set_checkerboard(DIMS, 0, e, back)
    gmg.set_checkerboard(DIMS, 1, o, back)
    assert torch.equal(back, xd)


def test_invert_self_matches_oracle(cm, links):
    ref = orc.invert_self_links(links)
    x = inputs.gaussian_field((512, R, N), inputs.rng(stream=903))
    y = torch.zeros((512, R, N), dtype=torch.complex128, device="cuda")
    cm.MooeeInv(dev(x), y)
    assert orc.rel_dev_sq(orc.coarse_mooee(DIMS, links, x, orc.RB_MOOEE_INV, ref), host(y)) < 1e-24


@pytest.mark.parametrize("prec,tol", [("f64", 1e-24), ("f32", 1e-10)])
@pytest.mark.parametrize("op", [orc.RB_MEOOE, orc.RB_MEOOE_DAG, orc.RB_MOOEE, orc.RB_MOOEE_DAG, orc.RB_MOOEE_INV,
                                orc.RB_MOOEE_INV_DAG])
@pytest.mark.parametrize("cb", [0, 1])
def test_rb_ops_match_oracle(cm, links, prec, tol, op, cb):
    inv = orc.invert_self_links(links)
    r = inputs.rng(stream=910 + op * 2 + cb)
    xh = inputs.gaussian_field((256, R, N), r)
    ref = orc.coarse_rb_apply(DIMS, links, xh, op, cb, inv)
    dt = torch.complex128 if prec == "f64" else torch.complex64
    x = dev(xh, dt)
    y = torch.zeros_like(x)
    cm._rb(op, cb, x, y, None)
    assert orc.rel_dev_sq(ref, host(y)) < tol


@pytest.mark.parametrize("nrhs", [1, 6])
def test_rb_single_and_multi_rhs_f64(cm, links, nrhs):
    xh = inputs.gaussian_field((256, nrhs, N), inputs.rng(stream=930 + nrhs))
    y = torch.zeros((256, nrhs, N), dtype=torch.complex128, device="cuda")
    cm.Meooe(dev(xh), y, 1)
    assert orc.rel_dev_sq(orc.coarse_rb_apply(DIMS, links, xh, orc.RB_MEOOE, 1), host(y)) < 1e-24


@pytest.mark.parametrize("dag", [0, 1])
def test_meooe_tensor_cores(cm, links, dag):
    xh = inputs.gaussian_field((256, 16, N), inputs.rng(stream=940 + dag))
    x = dev(xh, torch.complex64)
    y = torch.zeros_like(x)
    (cm.MeooeDag if dag else cm.Meooe)(x, y, 0, compute="bf16")
    op = orc.RB_MEOOE_DAG if dag else orc.RB_MEOOE
    assert orc.rel_dev_sq(orc.coarse_rb_apply(DIMS, links, xh, op, 0), host(y)) < 2e-5


@pytest.mark.parametrize("dag", [0, 1])
def test_dhop_full_grid(cm, links, dag):
    x = inputs.gaussian_field((512, R, N), inputs.rng(stream=950 + dag))
    for prec, tol, dt in (("f64", 1e-24, torch.complex128), ("bf16", 2e-5, torch.complex64)):
        y = torch.zeros((512, R, N), dtype=dt, device="cuda")
        cm.Dhop(dev(x, dt), y, dag=dag, compute=prec)
        assert orc.rel_dev_sq(orc.coarse_dhop(DIMS, links, x, dag), host(y)) < tol


def test_blocks_sum_to_m(cm, links):
    # Meo + Moe + Moo + Mee = M  (src/Test_coarse_red_black.cc:433-482)
    x = inputs.gaussian_field((512, R, N), inputs.rng(stream=960))
    xd = dev(x)
    e = torch.zeros((256, R, N), dtype=torch.complex128, device="cuda")
    o = torch.zeros_like(e)
    gmg.pick_checkerboard(DIMS, 0, xd, e)
    gmg.pick_checkerboard(DIMS, 1, xd, o)
    moe, meo, mee, moo = (torch.zeros_like(e) for _ in range(4))
    cm.Meooe(e, moe, 0)
    cm.Meooe(o, meo, 1)
    cm.Mooee(e, mee, 0)
    cm.Mooee(o, moo, 1)
    full = torch.zeros_like(xd)
    gmg.set_checkerboard(DIMS, 0, mee + meo, full)
    gmg.set_checkerboard(DIMS, 1, moo + moe, full)
    m = torch.zeros_like(xd)
    cm.M(xd, m)
    assert orc.rel_dev_sq(host(m), host(full)) < 1e-24


def test_inverse_dropped_when_links_change(links):
    m = gmg.CoarsenedMatrix(DIMS, N)
    m.set_links(links)
    m.InvertSelfStencilPoint()
    m.set_links(links)
    x = torch.zeros((512, 1, N), dtype=torch.complex128, device="cuda")
    with pytest.raises(gmg.GmgError):
        m.MooeeInv(x, torch.zeros_like(x))


def test_singular_self_link_reported(links):
    bad = links.copy()
    bad[8, 3] = 0.0
    m = gmg.CoarsenedMatrix(DIMS, N)
    m.set_links(bad)
    with pytest.raises(gmg.GmgError):
        m.InvertSelfStencilPoint()

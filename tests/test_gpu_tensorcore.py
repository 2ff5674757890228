"""Tensor-core (tcgen05) multi-RHS coarse stencil against the FP64 oracle.

BF16 / FP16 operands with FP32 accumulation: the links and the vectors are
rounded to 8 (BF16) or 11 (FP16) significant bits, so the stated bound on the
reference's relative squared deviation |ref-res|^2/|ref|^2 is 2e-5 for BF16
(about 4.5e-3 in norm) and 1e-6 for FP16 (1e-3 in norm).
"""
import numpy as np
import pytest
import torch

import gmg
import inputs
import oracle as orc

pytestmark = pytest.mark.gpu

TOL = {"bf16": 2e-5, "f16": 1e-6}


def run(cm, x, op, kind, point=8, active=None):
    inp = torch.from_numpy(x).to("cuda").to(torch.complex64)
    out = torch.zeros_like(inp)
    cm.apply(op, inp, out, point=point, compute=kind, active=active)
    code = np.zeros(1, dtype=np.int32)
    torch.cuda.synchronize()
    assert gmg.lib().gmg_coarse_device_error(cm._h, code.ctypes.data_as(__import__("ctypes").c_void_p)) == 0
    return out.cpu().numpy().astype(np.complex128)


@pytest.mark.parametrize("kind", ["bf16", "f16"])
@pytest.mark.parametrize("N,R", [(32, 32), (32, 5), (24, 16), (40, 8), (16, 48), (12, 24), (20, 8)])
def test_tc_m_and_mdag(kind, N, R):
    dims = (4, 4, 4, 4)
    r = inputs.rng(stream=200 + N + R)
    A = inputs.random_links(dims, N, r)
    x = inputs.gaussian_field((256, R, N), r)
    cm = gmg.CoarsenedMatrix(dims, N)
    cm.set_links(A)
    cm.prepare(kind)
    for op in (orc.OP_M, orc.OP_MDAG):
        ref = orc.coarse_apply(dims, A, x, op)
        got = run(cm, x, op, kind)
        assert orc.rel_dev_sq(ref, got) < TOL[kind], (op, orc.rel_dev_sq(ref, got))


@pytest.mark.parametrize("kind", ["bf16"])
def test_tc_single_points_and_active(kind):
    dims, N, R = (4, 2, 4, 4), 32, 12
    r = inputs.rng(stream=231)
    A = inputs.random_links(dims, N, r)
    x = inputs.gaussian_field((128, R, N), r)
    cm = gmg.CoarsenedMatrix(dims, N)
    cm.set_links(A)
    cm.prepare(kind)
    for p in (0, 3, 5, 8):
        ref = orc.coarse_apply(dims, A, x, orc.OP_MDIR, point=p)
        assert orc.rel_dev_sq(ref, run(cm, x, orc.OP_MDIR, kind, point=p)) < TOL[kind]
    active = [11, 0, 7, 3, 9]
    inp = torch.from_numpy(x).to("cuda").to(torch.complex64)
    out = torch.full_like(inp, 5.0)
    cm.M(inp, out, compute=kind, active=active)
    got = out.cpu().numpy().astype(np.complex128)
    ref = orc.coarse_apply(dims, A, x, orc.OP_M)
    for rr in range(R):
        if rr in active:
            assert orc.rel_dev_sq(ref[:, rr], got[:, rr]) < TOL[kind]
        else:
            assert np.all(got[:, rr] == 5.0)


def test_tc_links_refresh_on_set():
    dims, N = (2, 2, 2, 4), 32
    r = inputs.rng(stream=241)
    A1 = inputs.random_links(dims, N, r)
    A2 = inputs.random_links(dims, N, r)
    x = inputs.gaussian_field((32, 16, N), r)
    cm = gmg.CoarsenedMatrix(dims, N)
    cm.set_links(A1)
    cm.prepare("bf16")
    cm.set_links(A2)  # the prepared BF16 copy must follow
    assert orc.rel_dev_sq(orc.coarse_apply(dims, A2, x), run(cm, x, orc.OP_M, "bf16")) < TOL["bf16"]


def test_tc_full_c2_size_against_fp64_gpu():
    # 8^4 coarse lattice, nbasis 32, 32 RHS: the multi-RHS stencil configuration.
    # Size-independent checks: BF16 vs the (oracle-pinned) FP64 GPU path, and
    # linearity M(a x + b y) = a M x + b M y within the BF16 bound.
    dims, N, R = (8, 8, 8, 8), 32, 32
    r = inputs.rng(stream=251)
    A = inputs.random_links(dims, N, r)
    x = inputs.gaussian_field((4096, R, N), r)
    y = inputs.gaussian_field((4096, R, N), r)
    cm = gmg.CoarsenedMatrix(dims, N)
    cm.set_links(A)
    cm.prepare("bf16")
    xd = torch.from_numpy(x).cuda()
    o64 = torch.zeros_like(xd)
    cm.M(xd, o64)
    ref = o64.cpu().numpy()
    got = run(cm, x, orc.OP_M, "bf16")
    assert orc.rel_dev_sq(ref, got) < TOL["bf16"]
    a, b = 0.7 - 0.2j, -1.3 + 0.5j
    lin = run(cm, a * x + b * y, orc.OP_M, "bf16")
    assert orc.rel_dev_sq(a * got + b * run(cm, y, orc.OP_M, "bf16"), lin) < 4 * TOL["bf16"]


@pytest.mark.parametrize("shape", [(1, 1), (1, 3), (2, 1), (2, 3), (2, 4), (1, 2)])
def test_tc_every_launch_shape(shape):
    # every (CTAs per SM, points per stage) shape the autotuner may pick gives
    # the oracle's result; a shape that does not divide the point count (4 or 2
    # for the 9 points of M) falls back to the tuned one
    dims, N, R = (4, 4, 4, 4), 32, 24
    r = inputs.rng(stream=240 + 3 * shape[0] + shape[1])
    A = inputs.random_links(dims, N, r)
    x = inputs.gaussian_field((256, R, N), r)
    cm = gmg.CoarsenedMatrix(dims, N)
    cm.set_links(A)
    cm.prepare("bf16")
    assert gmg.lib().gmg_coarse_set_shape(cm._h, shape[0], shape[1]) == 0
    ref = orc.coarse_apply(dims, A, x, orc.OP_M)
    assert orc.rel_dev_sq(ref, run(cm, x, orc.OP_M, "bf16")) < TOL["bf16"]
    assert gmg.lib().gmg_coarse_set_shape(cm._h, 0, 0) == 0


def test_tc_autotuner_records_a_shape():
    import ctypes
    dims, N, R = (4, 4, 4, 4), 32, 32
    r = inputs.rng(stream=251)
    A = inputs.random_links(dims, N, r)
    x = inputs.gaussian_field((256, R, N), r)
    cm = gmg.CoarsenedMatrix(dims, N)
    cm.set_links(A)
    cm.prepare("bf16")
    ref = orc.coarse_apply(dims, A, x, orc.OP_M)
    assert orc.rel_dev_sq(ref, run(cm, x, orc.OP_M, "bf16")) < TOL["bf16"]
    ctas, pps = ctypes.c_int(), ctypes.c_int()
    assert gmg.lib().gmg_coarse_tuned_shape(cm._h, R, 9, gmg.BF16, ctypes.byref(ctas), ctypes.byref(pps)) == 0
    assert ctas.value in (1, 2) and pps.value in (1, 3), (ctas.value, pps.value)
    # a second call reuses the kept shape and gives the same result
    assert orc.rel_dev_sq(ref, run(cm, x, orc.OP_M, "bf16")) < TOL["bf16"]

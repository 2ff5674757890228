"""Multigrid-preconditioned solve (the MG apply chain) on small lattices.

Drives the K-cycle / FGMRES chain of MultiGridPreconditioner::operator()
(include/MultigridPreconditioner.h:253-309) through the C ABI and checks the
result independently: the true residual |b - D x| / |b| of every right-hand
side, recomputed with the FP64 fine operator after the solve, must meet the
1e-10 target of the multi-RHS solve configuration, for the plain FP64, the
FP32-preconditioner and the tensor-core (BF16 coarse stencil) forms.  The
Galerkin identity R D P = D_c (:398-421) is checked on the operators the
setup built.
"""
import ctypes

import numpy as np
import pytest
import torch

import gmg
import inputs

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def fine():
    dims = (8, 8, 8, 8)
    U = inputs.smooth_gauge(dims, inputs.rng(stream=301), 0.3)
    w = gmg.WilsonClover(dims, -0.05, 1.0, antiperiodic=True)
    w.set_gauge(U)
    return dims, w


def true_relres(w, b, x):
    r = torch.zeros_like(b)
    w.M(x, r)
    r = b - r
    return (torch.linalg.vector_norm(r, dim=(0, 2)) / torch.linalg.vector_norm(b, dim=(0, 2))).max().item()


@pytest.mark.parametrize("prec,levels", [("f64", 2), ("f32", 2), ("f32", 3), ("bf16", 3)])
def test_mg_solve_reaches_1e10(fine, prec, levels):
    dims, w = fine
    nrhs = 4
    kw = dict(nlevels=levels, nvec=(6, 6), setup_iters=30, prec=prec, coarsest_iters=30, wrapper_iters=6)
    if levels == 2:
        kw["block"] = ((4, 4, 4, 4), (2, 2, 2, 2))
    else:
        kw["block"] = ((2, 2, 2, 2), (2, 2, 2, 2))
    mg = gmg.MultiGrid(w, nrhs, **kw)
    mg.setup()
    # every test vector of every level made it into an orthonormal block basis
    # (a zero test vector shows up as a unit error here)
    for l in range(levels - 1):
        _, ag = mg.level(l)
        e = ctypes.c_double()
        assert gmg.lib().gmg_agg_check_orthogonal(ag, ctypes.byref(e), gmg._stream()) == 0
        assert e.value < 1e-12, (l, e.value)
    b = torch.from_numpy(inputs.gaussian_field((4096, nrhs, 12), inputs.rng(stream=302))).cuda()
    x = torch.zeros_like(b)
    it, rr = mg.solve(b, x, tol=1e-10, maxiter=300)
    assert rr <= 1e-10
    assert true_relres(w, b, x) <= 2e-10, (it, rr)


@pytest.mark.parametrize("prec,levels", [("f32", 2), ("f32", 3), ("bf16", 3)])
def test_mg_graph_captured_cycle(fine, prec, levels):
    # the K-cycle replayed as a CUDA graph (coarse-level Givens on the device,
    # conditional nodes for the early exits) reaches the same tolerance in the
    # same number of outer iterations as the host-driven cycle
    dims, w = fine
    nrhs = 4
    kw = dict(nlevels=levels, nvec=(6, 6), setup_iters=30, prec=prec, coarsest_iters=30, wrapper_iters=6)
    kw["block"] = ((4, 4, 4, 4), (2, 2, 2, 2)) if levels == 2 else ((2, 2, 2, 2), (2, 2, 2, 2))
    b = torch.from_numpy(inputs.gaussian_field((4096, nrhs, 12), inputs.rng(stream=304))).cuda()
    its = {}
    for graph in (0, 1):
        mg = gmg.MultiGrid(w, nrhs, graph=graph, **kw)
        mg.setup()
        x = torch.zeros_like(b)
        it, rr = mg.solve(b, x, tol=1e-10, maxiter=300)
        assert rr <= 1e-10
        assert true_relres(w, b, x) <= 2e-10, (graph, it, rr)
        its[graph] = it
        if graph:
            n, fell_back = mg.graphs()
            assert n >= 1 and fell_back == 0, (n, fell_back)
    assert abs(its[1] - its[0]) <= 1, its


def test_mg_graph_after_compaction(fine):
    # RHS that converge early drop out at the first outer restart; the smaller
    # batch gets its own captured cycle, and every RHS still reaches 1e-10
    dims, w = fine
    nrhs = 4
    mg = gmg.MultiGrid(w, nrhs, nlevels=3, block=((2, 2, 2, 2), (2, 2, 2, 2)), nvec=(6, 6), setup_iters=30,
                       prec="f32", coarsest_iters=30, wrapper_iters=6, outer_restart=4)
    mg.setup()
    b = torch.from_numpy(inputs.gaussian_field((4096, nrhs, 12), inputs.rng(stream=305))).cuda()
    x = torch.zeros_like(b)
    mg.solve(b, x, tol=1e-10, maxiter=300)
    assert mg.graphs() == (1, 0)
    x[:, 2:] = 0  # RHS 0 and 1 start converged
    it, rr = mg.solve(b, x, tol=1e-10, maxiter=300)
    assert rr <= 1e-10
    assert true_relres(w, b, x) <= 2e-10, it
    n, fell_back = mg.graphs()
    assert n == 2 and fell_back == 0, (n, fell_back)


def test_mg_galerkin_identity_on_setup_operators(fine):
    dims, w = fine
    mg = gmg.MultiGrid(w, 2, nlevels=2, block=((4, 4, 4, 4), (2, 2, 2, 2)), nvec=(6, 6), prec="f64")
    mg.setup()
    op1, _ = mg.level(1)
    _, ag0 = mg.level(0)
    N = 12
    # wrap the raw handles for the checks
    cm = gmg.CoarsenedMatrix.__new__(gmg.CoarsenedMatrix)
    cm._h, cm.dims, cm.N, cm.V, cm.hermitian = op1, (2, 2, 2, 2), N, 16, 0
    ag = gmg.Aggregation.__new__(gmg.Aggregation)
    ag._h, ag.fdims, ag.cdims, ag.dof, ag.N, ag.Vf, ag.Vc = ag0, dims, (2, 2, 2, 2), 12, N, 4096, 16
    vc = torch.from_numpy(inputs.gaussian_field((16, 2, N), inputs.rng(stream=303))).cuda()
    f = torch.zeros((4096, 2, 12), dtype=torch.complex128, device="cuda")
    ag.PromoteFromSubspace(vc, f)
    df = torch.zeros_like(f)
    w.M(f, df)
    rdp = torch.zeros_like(vc)
    ag.ProjectToSubspace(df, rdp)
    dc = torch.zeros_like(vc)
    cm.M(vc, dc)
    dev = (torch.linalg.vector_norm(rdp - dc) / torch.linalg.vector_norm(rdp)).item()
    # the handles belong to mg: do not let the wrappers free them
    cm._h = None
    ag._h = None
    assert dev < 1e-12
    assert mg.level(0)[1] is not None

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
    # (restart-time drops only: the in-cycle drop has its own test below)
    dims, w = fine
    nrhs = 4
    mg = gmg.MultiGrid(w, nrhs, nlevels=3, block=((2, 2, 2, 2), (2, 2, 2, 2)), nvec=(6, 6), setup_iters=30,
                       prec="f32", coarsest_iters=30, wrapper_iters=6, outer_restart=4, drop_in_cycle=0)
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


def _links(op, V, N):
    a = np.zeros((9, V, N, N), dtype=np.complex128)
    assert gmg.lib().gmg_coarse_get_links(op, a.ctypes.data_as(ctypes.c_void_p), 0, gmg._stream()) == 0
    return a


def _galerkin_dev(fine_apply, ag, op, Vf, dof, Vc, N, stream):
    # |R D P v_c - D_c v_c| / |R D P v_c| with FP64 transfers and operators
    L = gmg.lib()
    vc = torch.from_numpy(inputs.gaussian_field((Vc, 2, N), inputs.rng(stream=stream))).cuda()
    f = torch.zeros((Vf, 2, dof), dtype=torch.complex128, device="cuda")
    assert L.gmg_agg_promote(ag, gmg.F64, gmg.F64, 2, gmg._ptr(vc), gmg._ptr(f), gmg._stream()) == 0
    df = torch.zeros_like(f)
    fine_apply(f, df)
    rdp = torch.zeros_like(vc)
    assert L.gmg_agg_project(ag, gmg.F64, gmg.F64, 2, gmg._ptr(df), gmg._ptr(rdp), gmg._stream()) == 0
    dc = torch.zeros_like(vc)
    assert L.gmg_coarse_apply(op, gmg.OP_M, 8, gmg.F64, gmg.F64, 2, gmg._ptr(vc), gmg._ptr(dc), None, 0,
                              gmg._stream()) == 0
    return (torch.linalg.vector_norm(rdp - dc) / torch.linalg.vector_norm(rdp)).item()


@pytest.mark.parametrize("prec,levels", [("f64", 2), ("f32", 3), ("bf16", 3)])
def test_mg_refinement_setup(fine, prec, levels):
    # refinementSetup (MultigridPreconditioner.h:213-251): each level's test
    # vectors replaced by its own preconditioner applied to them, the next
    # level's vectors by the coarse solutions (recursive updates), every
    # operator rebuilt in place.  The rebuilt hierarchy is orthonormal, obeys
    # the Galerkin identity on every transition, and the solve still reaches
    # 1e-10 in no more outer iterations than after the initial setup alone.
    dims, w = fine
    nrhs = 4
    kw = dict(nlevels=levels, nvec=(6, 6), setup_iters=30, setup_null=0, prec=prec, coarsest_iters=30,
              wrapper_iters=6, refine_iters=(2, 1))
    kw["block"] = ((4, 4, 4, 4), (2, 2, 2, 2)) if levels == 2 else ((2, 2, 2, 2), (2, 2, 2, 2))
    cdims = [tuple(d // b for d, b in zip(dims, kw["block"][0]))]
    cdims.append(tuple(d // b for d, b in zip(cdims[0], kw["block"][1])))
    Vc = [int(np.prod(c)) for c in cdims]
    b = torch.from_numpy(inputs.gaussian_field((4096, nrhs, 12), inputs.rng(stream=306))).cuda()
    mg = gmg.MultiGrid(w, nrhs, **kw)
    mg.setup()
    x = torch.zeros_like(b)
    it0, rr0 = mg.solve(b, x, tol=1e-10, maxiter=300)
    assert rr0 <= 1e-10
    handles = [mg.level(l) for l in range(levels)]
    before = _links(handles[1][0], Vc[0], 12)
    mg.refine()
    assert [tuple(h.value for h in mg.level(l)) for l in range(levels)] == \
        [tuple(h.value for h in hs) for hs in handles]
    after = _links(handles[1][0], Vc[0], 12)
    assert np.abs(after - before).max() > 1e-3 * np.abs(before).max()
    for l in range(levels - 1):
        e = ctypes.c_double()
        assert gmg.lib().gmg_agg_check_orthogonal(handles[l][1], ctypes.byref(e), gmg._stream()) == 0
        assert e.value < 1e-12, (l, e.value)
    dev = _galerkin_dev(w.M, handles[0][1], handles[1][0], 4096, 12, Vc[0], 12, 307)
    assert dev < 1e-12, dev
    if levels == 3:
        op1 = handles[1][0]

        def coarse_m(inp, out):
            assert gmg.lib().gmg_coarse_apply(op1, gmg.OP_M, 8, gmg.F64, gmg.F64, inp.shape[1], gmg._ptr(inp),
                                              gmg._ptr(out), None, 0, gmg._stream()) == 0

        dev = _galerkin_dev(coarse_m, handles[1][1], handles[2][0], Vc[0], 12, Vc[1], 12, 308)
        assert dev < 1e-12, dev
    x = torch.zeros_like(b)
    it1, rr1 = mg.solve(b, x, tol=1e-10, maxiter=300)
    assert rr1 <= 1e-10
    assert true_relres(w, b, x) <= 2e-10, (it1, rr1)
    print(f"outer iterations: {it0} after the initial setup, {it1} after the refinement")
    assert it1 <= it0 + 1, (it0, it1)


def test_mg_refinement_stops_at_a_level_without_iterations(fine):
    # as in the reference (the recursion sits inside the level's own
    # `setupRefinementIter > 0` branch), no iterations on the first transition
    # leave the whole hierarchy untouched, whatever the second one asks for
    dims, w = fine
    mg = gmg.MultiGrid(w, 2, nlevels=3, block=((2, 2, 2, 2), (2, 2, 2, 2)), nvec=(6, 6), setup_iters=30,
                       prec="f32", coarsest_iters=30, wrapper_iters=6, refine_iters=(0, 3))
    mg.setup()
    op1, op2 = mg.level(1)[0], mg.level(2)[0]
    l1, l2 = _links(op1, 256, 12), _links(op2, 16, 12)
    mg.refine()
    assert np.array_equal(_links(op1, 256, 12), l1)
    assert np.array_equal(_links(op2, 16, 12), l2)


@pytest.mark.parametrize("prec,graph", [("f32", 1), ("bf16", 1), ("f64", 0)])
def test_mg_converged_rhs_leave_within_a_cycle(fine, prec, graph):
    # Right-hand sides whose initial guesses sit at different distances from
    # the solution converge at different Arnoldi steps of one outer cycle.  With
    # drop_in_cycle each leaves the batch at its step: the preconditioner and
    # the operator of the later steps run on fewer RHS (the recorded batch sizes
    # fall), every RHS keeps the iteration count it has without the drop (up to
    # one step: the inner K-cycle solves stop on the slowest RHS of their
    # batch), and every RHS meets the 1e-10 true residual.
    dims, w = fine
    nrhs = 4
    # (FP64 Arnoldi: an FP32 cycle stops at 1e-6 of its starting residual, so
    # the RHS started 1e-1 from the solution would need a second cycle)
    kw = dict(nlevels=3, nvec=(6, 6), setup_iters=30, prec=prec, coarsest_iters=30, wrapper_iters=6, graph=graph,
              block=((2, 2, 2, 2), (2, 2, 2, 2)), outer_restart=24, arnoldi_f32=0)
    b = torch.from_numpy(inputs.gaussian_field((4096, nrhs, 12), inputs.rng(stream=311))).cuda()
    mg = gmg.MultiGrid(w, nrhs, drop_in_cycle=0, **kw)
    mg.setup()
    xs = torch.zeros_like(b)
    mg.solve(b, xs, tol=1e-12, maxiter=400)
    noise = torch.from_numpy(inputs.gaussian_field((4096, nrhs, 12), inputs.rng(stream=312))).cuda()
    scale = torch.tensor([10.0 ** -(2 * r + 1) for r in range(nrhs)], dtype=torch.float64, device="cuda")
    scale = scale * torch.linalg.vector_norm(xs, dim=(0, 2)) / torch.linalg.vector_norm(noise, dim=(0, 2))
    x0 = xs + noise * scale.view(1, nrhs, 1)
    res = {}
    for drop in (0, 1):
        m = gmg.MultiGrid(w, nrhs, drop_in_cycle=drop, **kw)
        m.setup()
        x = x0.clone()
        it, rr = m.solve(b, x, tol=1e-10, maxiter=300)
        assert rr <= 1e-10
        assert true_relres(w, b, x) <= 2e-10, (drop, it, rr)
        its, _ = m.solve_stats(nrhs)
        res[drop] = (its, m.solve_batches())
    its0, b0 = res[0]
    its1, b1 = res[1]
    assert len(set(its1.tolist())) >= 3, its1  # the RHS converge at different steps
    assert np.abs(its1 - its0).max() <= 1, (its0, its1)
    assert b0.min() == nrhs  # without the drop every step of the cycle runs the full batch
    assert b1[0] == nrhs and b1.min() < nrhs and np.all(np.diff(b1) <= 0), b1
    # each drop happened at the step its RHS met the tolerance: the batch of
    # step k counts the RHS that had not converged before it
    for k, sz in enumerate(b1):
        assert sz == int((its1 > k).sum()), (k, b1, its1)


@pytest.mark.parametrize("prec", ["f32", "bf16"])
def test_mg_bf16_smoother_reaches_1e10(fine, prec):
    # the fine smoother with BF16 residual fields (FP32 arithmetic and solution):
    # the outer FP64 FGMRES still reaches the 1e-10 true residual, within two
    # outer iterations of the FP32 smoother
    dims, w = fine
    nrhs = 4
    kw = dict(nlevels=3, nvec=(6, 6), setup_iters=30, prec=prec, coarsest_iters=30, wrapper_iters=6,
              block=((2, 2, 2, 2), (2, 2, 2, 2)))
    b = torch.from_numpy(inputs.gaussian_field((4096, nrhs, 12), inputs.rng(stream=321))).cuda()
    its = {}
    for bf in (0, 1):
        mg = gmg.MultiGrid(w, nrhs, smoother_bf16=bf, **kw)
        mg.setup()
        x = torch.zeros_like(b)
        it, rr = mg.solve(b, x, tol=1e-10, maxiter=300)
        assert rr <= 1e-10
        assert true_relres(w, b, x) <= 2e-10, (bf, it, rr)
        its[bf] = it
    assert its[1] <= its[0] + 2, its


@pytest.mark.gpu
def test_mg_apply_bf16_smoother_matches_fp32_smoother(fine):
    # one K-cycle (MultiGridPreconditioner::operator()) with the BF16 smoother
    # (site-blocked BF16 residual fields, the operator's fused first residual,
    # one solution update per sweep) against the same cycle with the FP32
    # smoother: equal up to BF16 rounding of the smoother's residuals, and a
    # real preconditioner (|D M^-1 b - b| well below |b|)
    dims, w = fine
    nrhs = 5  # not a multiple of the tile's threads per site
    kw = dict(nlevels=3, nvec=(6, 6), setup_iters=30, prec="bf16", coarsest_iters=30, wrapper_iters=6,
              block=((2, 2, 2, 2), (2, 2, 2, 2)), graph=0)
    b = torch.from_numpy(inputs.gaussian_field((4096, nrhs, 12), inputs.rng(stream=341))).cuda()
    outs = {}
    for bf in (0, 1):
        mg = gmg.MultiGrid(w, nrhs, smoother_bf16=bf, **kw)
        mg.setup()
        out = torch.zeros_like(b)
        mg.apply(b, out)
        outs[bf] = out
    rel = (torch.linalg.vector_norm(outs[1] - outs[0], dim=(0, 2)) /
           torch.linalg.vector_norm(outs[0], dim=(0, 2))).max().item()
    assert rel < 2e-2, rel
    Db = torch.zeros_like(b)
    w.M(outs[1], Db)
    red = (torch.linalg.vector_norm(Db - b, dim=(0, 2)) / torch.linalg.vector_norm(b, dim=(0, 2))).max().item()
    assert red < 0.5, red


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["f32", "bf16"])
def test_mg_fp32_arnoldi_reaches_1e10(fine, prec):
    # restart cycles whose Arnoldi process runs in FP32 on the FP64 residual
    # (iterative refinement): the same 1e-10 FP64 true residual, within two
    # outer iterations of the FP64 Arnoldi process, with and without the
    # in-cycle drop
    dims, w = fine
    nrhs = 4
    kw = dict(nlevels=3, nvec=(6, 6), setup_iters=30, prec=prec, coarsest_iters=30, wrapper_iters=6,
              block=((2, 2, 2, 2), (2, 2, 2, 2)), outer_restart=8)
    b = torch.from_numpy(inputs.gaussian_field((4096, nrhs, 12), inputs.rng(stream=331))).cuda()
    for drop in (0, 1):
        its = {}
        for a in (0, 1):
            mg = gmg.MultiGrid(w, nrhs, arnoldi_f32=a, drop_in_cycle=drop, **kw)
            mg.setup()
            x = torch.zeros_like(b)
            it, rr = mg.solve(b, x, tol=1e-10, maxiter=300)
            assert rr <= 1e-10
            assert true_relres(w, b, x) <= 2e-10, (a, drop, it, rr)
            its[a] = it
        assert its[1] <= its[0] + 2, (drop, its)

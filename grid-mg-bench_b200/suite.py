"""Per-row measurements of the hot path (run by `bench.py --suite`).

One JSON line per row, each with achieved rates against the measured
roofline (MEASURED_PEAKS.json) and the kernel time taken from CUDA events on
the launching stream.  Inputs are seeded synthetic fields with the
configurations' shapes (coarse links with the gamma5-hermitian structure,
unit-Gaussian vectors, smooth gauge U = exp(i eps H)).

  C1  coarse M, single RHS, FP64: coarse 4^4, nbasis 24
  C3  block project / promote (FP64, FP32) and orthonormalise (FP64):
      fine 32^4, nbasis 32, 32 RHS, 4^4 blocks
  C4  CoarsenOperator 32^4 -> 8^4 (nbasis 40, Wilson-clover m=-0.3, csw 1,
      eps 0.3), then coarse-of-coarse 8^4 -> 4^4 (2^4 blocks, nbasis 40)
  W   fine Wilson-clover M on 32^4, 1, 12 and 24 RHS, FP64 and FP32
"""
import ctypes
import json
import os
import time

import numpy as np
import torch

import gmg
import inputs

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
L2_FLUSH = 256 << 20


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class Timer:
    """Per-call CUDA-event timing on the current stream with an L2 flush before each call."""

    def __init__(self):
        self.flush = torch.empty(L2_FLUSH // 4, dtype=torch.float32, device="cuda")

    def run(self, fn, reps=5, warm=2, flush=True):
        for _ in range(warm):
            fn()
        s = torch.cuda.current_stream()
        tot = 0.0
        for k in range(reps):
            if flush:
                self.flush.fill_(float(k))
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(s)
            fn()
            b.record(s)
            b.synchronize()
            tot += a.elapsed_time(b)
        return tot / reps * 1e-3  # seconds per call


def kernel_avg(name):
    ms, n = ctypes.c_double(), ctypes.c_int64()
    gmg.lib().gmg_profile_read(name.encode(), ctypes.byref(ms), ctypes.byref(n))
    return (ms.value / n.value * 1e-3) if n.value else None, n.value


def line(row, **kw):
    d = {"row": row}
    d.update(kw)
    print(json.dumps(d), flush=True)


def c1(T, hbm):
    dims, N = (4, 4, 4, 4), 24
    A = inputs.random_links(dims, N, inputs.rng(stream=501))
    x = torch.from_numpy(inputs.gaussian_field((256, 1, N), inputs.rng(stream=502))).cuda()
    cm = gmg.CoarsenedMatrix(dims, N)
    cm.set_links(A)
    out = torch.zeros_like(x)
    flops = 256 * 9 * 8 * N * N
    byts = (9 * N * N + 2 * N) * 16 * 256
    t_cold = T.run(lambda: cm.M(x, out), reps=50)
    t_warm = T.run(lambda: cm.M(x, out), reps=200, flush=False)
    line("C1 coarse M single RHS FP64 (4^4, nbasis 24)", us_l2_flushed=t_cold * 1e6, us_l2_warm=t_warm * 1e6,
         gflops_flushed=flops / t_cold / 1e9, gbs_flushed=byts / t_cold / 1e9,
         frac_hbm_flushed=byts / t_cold / 1e9 / hbm, algorithmic_bytes=byts, algorithmic_flops=flops,
         note="launch-latency bound: 21 MB of links, 10.6 MFLOP")


def c3(T, hbm):
    fd, cd, N, R = (32, 32, 32, 32), (8, 8, 8, 8), 32, 32
    Vf, Vc = 32 ** 4, 8 ** 4
    half = inputs.torch_gaussian((N // 2, Vf, 12), 601)
    B = torch.zeros((N, Vf, 12), dtype=torch.complex128, device="cuda")
    B[: N // 2, :, :6] = half[:, :, :6]  # chiral doubling: upper / lower spin halves
    B[N // 2:, :, 6:] = half[:, :, 6:]
    del half
    ag = gmg.Aggregation(fd, cd, 12, N)
    ag.set_basis(B)
    del B
    torch.cuda.empty_cache()
    t_ortho = T.run(lambda: ag.Orthogonalise(passes=1), reps=2, warm=1)
    err = ag.CheckOrthogonal()
    # per-kernel times of one more pass (events on the stream; the two extra rounds are near-empty)
    gmg.lib().gmg_profile_enable(1)
    ag.Orthogonalise(passes=1)
    torch.cuda.synchronize()
    gmg.lib().gmg_profile_enable(0)
    ortho_kernels = {}
    for kname in ("ortho_gram", "ortho_factor", "ortho_solve"):
        ms_, n_ = kernel_avg(kname)
        ortho_kernels[kname] = {"ms_total": (ms_ or 0.0) * n_ * 1e3, "launches": n_}
    f64 = inputs.torch_gaussian((Vf, R, 12), 602)
    c64 = torch.zeros((Vc, R, N), dtype=torch.complex128, device="cuda")
    flops = 8.0 * Vf * 12 * N * R
    b64 = (N * Vf * 12 + Vf * R * 12 + Vc * R * N) * 16
    res = {}
    gmg.lib().gmg_profile_enable(1)
    t = T.run(lambda: ag.ProjectToSubspace(f64, c64), reps=3, warm=1)
    res["project_f64"] = (t, kernel_avg("project")[0], b64)
    t = T.run(lambda: ag.PromoteFromSubspace(c64, f64), reps=3, warm=1)
    res["promote_f64"] = (t, kernel_avg("promote")[0], b64)
    f32 = f64.to(torch.complex64)
    del f64
    c32 = c64.to(torch.complex64)
    b32 = b64 // 2
    t = T.run(lambda: ag.ProjectToSubspace(f32, c32), reps=3, warm=1)
    res["project_f32"] = (t, kernel_avg("project")[0], b32)
    t = T.run(lambda: ag.PromoteFromSubspace(c32, f32), reps=3, warm=1)
    res["promote_f32"] = (t, kernel_avg("promote")[0], b32)
    # tensor-core forms: BF16 hi + lo basis (8 B per complex, as FP32), FP32 vectors
    t = T.run(lambda: ag.ProjectToSubspace(f32, c32, compute="bf16"), reps=3, warm=1)
    res["project_bf16x2_tc"] = (t, kernel_avg("project_tc")[0], b32)
    t = T.run(lambda: ag.PromoteFromSubspace(c32, f32, compute="bf16"), reps=3, warm=1)
    res["promote_bf16x2_tc"] = (t, kernel_avg("promote_tc")[0], b32)
    gmg.lib().gmg_profile_enable(0)
    # accuracy of the tensor-core forms against the FP64 kernels on the same inputs
    errs = {}
    fx = f32.to(torch.complex128)
    cref = torch.zeros((Vc, R, N), dtype=torch.complex128, device="cuda")
    ag.ProjectToSubspace(fx, cref)
    ag.ProjectToSubspace(f32, c32, compute="bf16")
    errs["project_bf16x2_tc"] = ((c32.to(torch.complex128) - cref).norm() / cref.norm()).item()
    ag.PromoteFromSubspace(c32.to(torch.complex128), fx)
    ag.PromoteFromSubspace(c32, f32, compute="bf16")
    errs["promote_bf16x2_tc"] = ((f32.to(torch.complex128) - fx).norm() / fx.norm()).item()
    del fx
    out = {k: {"ms": v[0] * 1e3, "tflops": flops / v[0] / 1e12, "gbs": v[2] / v[0] / 1e9,
               "frac_hbm": v[2] / v[0] / 1e9 / hbm} for k, v in res.items()}
    for k, e in errs.items():
        out[k]["rel_err_vs_fp64"] = e
    # orthonormalisation: algorithmic bytes = basis read + written once (FP64),
    # flops = 8 K N^2 Vc (the Gram-Schmidt inner products and updates)
    ob = 2 * N * Vf * 12 * 16
    of = 8.0 * 3072 * N * N * Vc
    ortho = {"ms": t_ortho * 1e3, "max_err": err, "algorithmic_bytes": ob, "gbs": ob / t_ortho / 1e9,
             "frac_hbm": ob / t_ortho / 1e9 / hbm, "algorithmic_flops": of, "tflops_fp64": of / t_ortho / 1e12,
             "traffic_model_bytes": 3 * N * Vf * 12 * 16, "kernels": ortho_kernels,
             "note": "one pass: Gram + Cholesky kernel (basis read), forward-substitution kernel (read + write)"}
    line("C3 block project / promote (32^4, nbasis 32, 32 RHS, 4^4 blocks)", results=out,
         orthonormalise=ortho, algorithmic_flops=flops, algorithmic_bytes_f64=b64)


def wilson_and_c4(T, hbm):
    fd = (32, 32, 32, 32)
    V = 32 ** 4
    U = inputs.torch_smooth_gauge(fd, 701, 0.3)
    w = gmg.WilsonClover(fd, -0.3, 1.0, antiperiodic=True)
    w.set_gauge(U)
    del U
    res = {}
    for R in (1, 12, 24):
        for dt, cb in ((torch.complex128, 16), (torch.complex64, 8)):
            x = inputs.torch_gaussian((V, R, 12), 702, dtype=dt)
            y = torch.zeros_like(x)
            byts = V * (2 * 12 * R + 36 + 72) * cb  # in + out per RHS, gauge + clover once
            prec = "f64" if cb == 16 else "f32"
            per = {}
            for variant in (("site", "tile", "quad") if R < 4 else ("tile", "quad", "staged")):
                w.set_kernel(variant)
                per[variant] = round(T.run(lambda: w.M(x, y), reps=5) * 1e3, 3)
            w.set_kernel("auto")
            t = T.run(lambda: w.M(x, y), reps=5)
            res[f"R{R}_{prec}"] = {
                "ms": t * 1e3, "gflops": 1824.0 * V * R / t / 1e9, "gbs": byts / t / 1e9,
                "frac_hbm": byts / t / 1e9 / hbm, "tuned": w.tuned_kernel(prec, R), "ms_per_variant": per}
            del x, y
    line("W fine Wilson-clover M (32^4)", results=res,
         note="flops: 1824 per site per RHS (reference model); bytes: spinor in+out per RHS, gauge 36 + clover 72 complex per site; 'tuned' is the autotuner's pick")
    # C4: CoarsenOperator 32^4 -> 8^4, nbasis 40, then 8^4 -> 4^4
    N = 40
    half = inputs.torch_gaussian((N // 2, V, 12), 703)
    B = torch.zeros((N, V, 12), dtype=torch.complex128, device="cuda")
    B[: N // 2, :, :6] = half[:, :, :6]
    B[N // 2:, :, 6:] = half[:, :, 6:]
    del half
    ag = gmg.Aggregation(fd, (8, 8, 8, 8), 12, N)
    ag.set_basis(B)
    del B
    torch.cuda.empty_cache()
    ag.Orthogonalise(passes=1)
    # the first call also tunes the fine-operator kernels for its batch size
    t_first = None
    for _ in range(2):
        cm = gmg.CoarsenedMatrix((8, 8, 8, 8), N)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        cm.CoarsenOperator(ag, w)
        torch.cuda.synchronize()
        t_c4 = time.perf_counter() - t0
        if t_first is None:
            t_first = t_c4
    h2 = inputs.torch_gaussian((N // 2, 4096, N), 704)
    B2 = torch.zeros((N, 4096, N), dtype=torch.complex128, device="cuda")
    B2[: N // 2, :, : N // 2] = h2[:, :, : N // 2]
    B2[N // 2:, :, N // 2:] = h2[:, :, N // 2:]
    ag2 = gmg.Aggregation((8, 8, 8, 8), (4, 4, 4, 4), N, N)
    ag2.set_basis(B2)
    ag2.Orthogonalise(passes=1)
    cc = gmg.CoarsenedMatrix((4, 4, 4, 4), N)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    cc.CoarsenOperator(ag2, cm)
    torch.cuda.synchronize()
    t_cc = time.perf_counter() - t0
    proj_flops = 2 * 8.0 * 3072 * N * N * 4096
    fine_flops = N * V * (4 * 144 + 2 * 1824) * 1.0
    line("C4 CoarsenOperator 32^4 -> 8^4 (nbasis 40) and 8^4 -> 4^4", seconds=t_c4, first_call_seconds=t_first,
         coarse_of_coarse_seconds=t_cc,
         algorithmic_flops=proj_flops + fine_flops, achieved_tflops=(proj_flops + fine_flops) / t_c4 / 1e12,
         note="FP64; backward Mdir + face-site projections per batch of basis vectors; seconds: second call")


def c5_measure(nrhs=24, plain_rhs=24,
               forms=("mixed_bf16_mrhs", "mixed_bf16_mrhs_graph", "mixed_f32_mrhs", "plain_f64_single_rhs"), L=32):
    """3-level K-cycle MG-preconditioned FGMRES on 32^4 Wilson-clover (m=-0.35, csw 1, eps 0.3,
    antiperiodic t): nbasis 24 on 4^4 blocks, nbasis 32 on 2^4 blocks, MR(8) smoothing;
    `nrhs` Gaussian RHS to a true relative residual of 1e-10.  The plain FP64 single-RHS
    form is timed on `plain_rhs` RHS, one at a time (scaled to `nrhs` when fewer).
    `outer_iterations_per_rhs` lists, per RHS, the outer FGMRES iteration at which its
    residual estimate met the tolerance.  The graph form
    replays the K-cycle as a captured CUDA graph; its first solve also captures the graph
    (after one host-driven cycle per batch size) and is reported separately, the timed one
    is the second solve on the same handle."""
    fd = (L, L, L, L)
    V = L ** 4
    U = inputs.torch_smooth_gauge(fd, 801, 0.3)
    w = gmg.WilsonClover(fd, -0.35, 1.0, antiperiodic=True)
    w.set_gauge(U)
    del U
    b_all = inputs.torch_gaussian((V, nrhs, 12), 802)
    common = dict(nlevels=3, block=((4, 4, 4, 4), (2, 2, 2, 2)), nvec=(12, 16), smoother_iters=8)
    table = {"mixed_bf16_mrhs": ("bf16", nrhs, 0), "mixed_bf16_mrhs_graph": ("bf16", nrhs, 1),
             "mixed_f32_mrhs": ("f32", nrhs, 0), "plain_f64_single_rhs": ("f64", 1, 0)}
    out = {}
    for form in forms:
        prec, R, graph = table[form]
        mg = gmg.MultiGrid(w, R, prec=prec, graph=graph, **common)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        mg.setup()
        torch.cuda.synchronize()
        t_setup = time.perf_counter() - t0
        n_solve = nrhs if R == nrhs else plain_rhs
        t_first = None
        if graph:
            b = b_all.contiguous()
            x = torch.zeros_like(b)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            mg.solve(b, x, tol=1e-10, maxiter=400)
            torch.cuda.synchronize()
            t_first = time.perf_counter() - t0
            del b, x
        iters, worst, t_solve = [], 0.0, 0.0
        for k0 in range(0, n_solve, R):
            b = b_all[:, k0:k0 + R].contiguous()
            x = torch.zeros_like(b)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            it, rr = mg.solve(b, x, tol=1e-10, maxiter=400)
            torch.cuda.synchronize()
            t_solve += time.perf_counter() - t0
            r = torch.zeros_like(b)
            w.M(x, r)
            true = (torch.linalg.vector_norm(b - r, dim=(0, 2)) / torch.linalg.vector_norm(b, dim=(0, 2))).max().item()
            worst = max(worst, true)
            iters.extend(int(v) for v in mg.solve_stats(b.shape[1])[0])
            del b, x, r
        per_rhs = t_solve / n_solve
        out[form] = {"setup_s": t_setup, "solve_s_measured": t_solve, "rhs_measured": n_solve,
                     "solve_s_for_all_rhs": per_rhs * nrhs, "outer_iterations_per_rhs": iters,
                     "max_true_relres": worst}
        if graph:
            out[form]["first_solve_s"] = t_first
            out[form]["graphs"] = mg.graphs()
        del mg
        torch.cuda.empty_cache()
    if "plain_f64_single_rhs" in out:
        base = out["plain_f64_single_rhs"]["solve_s_for_all_rhs"]
        for k in out:
            out[k]["speedup_vs_plain_f64"] = base / out[k]["solve_s_for_all_rhs"]
    return out


def c5(nrhs=24, plain_rhs=24):
    out = c5_measure(nrhs, plain_rhs)
    line("C5 3-level K-cycle MG solve, 32^4 Wilson-clover, 24 RHS to 1e-10", results=out,
         note=f"plain FP64 single-RHS form timed on {plain_rhs} RHS one at a time; "
              "setup (null vectors, orthonormalisation, CoarsenOperator) not included in solve_s")


def c5_small(nrhs=24):
    """The C5 solver on a 16^4 lattice (coarse levels of 256 and 16 sites), where
    the coarse solves are latency-bound: host-driven vs graph-replayed K-cycle."""
    out = c5_measure(nrhs, 1, forms=("mixed_bf16_mrhs", "mixed_bf16_mrhs_graph"), L=16)
    line("C5s same 3-level MG on 16^4 Wilson-clover, 24 RHS to 1e-10: host-driven vs graph-replayed K-cycle",
         results=out, note="graph form: second solve on the handle (the first also captures)")


def profile_rows(rows):
    """Small cases of the C3 transfers, the fine operator, the MG solve and the C4
    construction for ncu captures: 16^4 fine lattice (nbasis 32 on 4^4 blocks,
    32 RHS; Wilson-clover with 24 RHS; one restart cycle of the C5 solve's
    kernels with 24 RHS; CoarsenOperator with nbasis 40)."""
    fd, cd, N, R = (16, 16, 16, 16), (4, 4, 4, 4), 32, 32
    Vf, Vc = 16 ** 4, 4 ** 4
    if "p_c3" in rows:
        B = inputs.torch_gaussian((N, Vf, 12), 611)
        ag = gmg.Aggregation(fd, cd, 12, N)
        ag.set_basis(B)
        ag.Orthogonalise(passes=1)
        f = inputs.torch_gaussian((Vf, R, 12), 612).to(torch.complex64)
        c = torch.zeros((Vc, R, N), dtype=torch.complex64, device="cuda")
        for _ in range(2):
            ag.ProjectToSubspace(f, c, compute="bf16")
            ag.PromoteFromSubspace(c, f, compute="bf16")
        torch.cuda.synchronize()
        line("p_c3 tensor-core project / promote 16^4, nbasis 32, 32 RHS", ok=True)
    if "p_ortho" in rows:
        # block orthonormalisation 16^4, nbasis 32 on 4^4 blocks (basis 403 MB):
        # one pass of the Gram + Cholesky kernel and the forward substitution
        B = inputs.torch_gaussian((N, Vf, 12), 617)
        ag = gmg.Aggregation(fd, cd, 12, N)
        ag.set_basis(B)
        del B
        ag.Orthogonalise(passes=1)
        ag.Orthogonalise(passes=1)
        torch.cuda.synchronize()
        line("p_ortho orthonormalise 16^4, nbasis 32, 4^4 blocks", ok=True, max_err=ag.CheckOrthogonal())
    if "p_w" in rows:
        # the fine-operator forms of the C5 solve at 24 RHS: M in FP32, M with the
        # fused MR products in FP32 (smoother) and M in FP64 (outer FGMRES).  The
        # first call of each tunes the kernel variant; the calls inside the NVTX
        # range "p_w" run the tuned kernels once each, those inside "p_w_staged"
        # the pipelined staged kernel (forced) in FP32 and FP64
        U = inputs.torch_smooth_gauge(fd, 613, 0.3)
        w = gmg.WilsonClover(fd, -0.35, 1.0, antiperiodic=True)
        w.set_gauge(U)
        del U
        x = inputs.torch_gaussian((Vf, 24, 12), 614)
        y = torch.zeros_like(x)
        x32, y32 = x.to(torch.complex64), y.to(torch.complex64)
        for _ in range(2):
            w.M(x32, y32)
            w.M_mr(x32, y32)
            w.M(x, y)
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_push("p_w")
        w.M(x32, y32)
        w.M_mr(x32, y32)
        w.M(x, y)
        torch.cuda.nvtx.range_pop()
        torch.cuda.synchronize()
        w.set_kernel("staged")
        w.M(x32, y32)
        w.M(x, y)
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_push("p_w_staged")
        w.M(x32, y32)
        w.M(x, y)
        torch.cuda.nvtx.range_pop()
        torch.cuda.synchronize()
        w.set_kernel("auto")
        line("p_w Wilson-clover 16^4, 24 RHS: FP32 M, FP32 M with MR products, FP64 M; staged FP32 / FP64 M",
             ok=True, tuned={"f32": w.tuned_kernel("f32", 24), "f32_mr": w.tuned_kernel("f32", 24, fused_mr=True),
                             "f64": w.tuned_kernel("f64", 24)})
    for row5, graph5 in (("p_c5", 1), ("p_c5h", 0)):
        if row5 not in rows:
            continue
        # the C5 mixed BF16 solve (32^4, 24 RHS; p_c5: graph-captured K-cycle, p_c5h:
        # host-driven, every kernel a plain launch): setup and one solve (which
        # captures), then the second solve inside the NVTX range named after the row
        fd5 = (32, 32, 32, 32)
        U = inputs.torch_smooth_gauge(fd5, 801, 0.3)
        w5 = gmg.WilsonClover(fd5, -0.35, 1.0, antiperiodic=True)
        w5.set_gauge(U)
        del U
        b = inputs.torch_gaussian((32 ** 4, 24, 12), 802)
        mg = gmg.MultiGrid(w5, 24, prec="bf16", graph=graph5, nlevels=3, block=((4, 4, 4, 4), (2, 2, 2, 2)),
                           nvec=(12, 16), smoother_iters=8)
        mg.setup()
        x = torch.zeros_like(b)
        mg.solve(b, x, tol=1e-10, maxiter=400)
        x.zero_()
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_push(row5)
        t0 = time.perf_counter()
        it, rr = mg.solve(b, x, tol=1e-10, maxiter=400)
        torch.cuda.synchronize()
        t = time.perf_counter() - t0
        torch.cuda.nvtx.range_pop()
        line(f"{row5} MG solve 32^4, 24 RHS, mixed BF16, " + ("graph-captured" if graph5 else "host-driven") +
             " K-cycle", ok=True, seconds=t, iters=it, relres=rr)
        del mg, x, b, w5
        torch.cuda.empty_cache()
    if "p_mg16" in rows:
        # the C5 solve's kernels on a 16^4 lattice (24 RHS, mixed BF16, host-driven
        # K-cycle): setup, then 8 outer iterations (one restart cycle, every
        # Gram-Schmidt sweep of it) inside the NVTX range "p_mg16"; the solve stops
        # at its iteration limit, well above the tolerance
        U = inputs.torch_smooth_gauge(fd, 801, 0.3)
        w = gmg.WilsonClover(fd, -0.35, 1.0, antiperiodic=True)
        w.set_gauge(U)
        del U
        b = inputs.torch_gaussian((Vf, 24, 12), 802)
        mg = gmg.MultiGrid(w, 24, prec="bf16", graph=0, nlevels=3, block=((4, 4, 4, 4), (2, 2, 2, 2)),
                           nvec=(12, 16), smoother_iters=8, setup_iters=30)
        mg.setup()
        x = torch.zeros_like(b)
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_push("p_mg16")
        try:
            mg.solve(b, x, tol=1e-10, maxiter=8)
        except gmg.GmgError:
            pass
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_pop()
        line("p_mg16 MG solve kernels 16^4, 24 RHS, mixed BF16, 8 outer iterations", ok=True)
    if "p_c4" in rows:
        # CoarsenOperator 16^4 -> 4^4, nbasis 40 (the C4 construction on a
        # sixteenth of its volume): two calls, each with 4 face hops, one
        # self-term operator pass and 5 FP64 projections of 40 RHS
        N4 = 40
        U = inputs.torch_smooth_gauge(fd, 615, 0.3)
        w = gmg.WilsonClover(fd, -0.3, 1.0, antiperiodic=True)
        w.set_gauge(U)
        half = inputs.torch_gaussian((N4 // 2, Vf, 12), 616)
        B = torch.zeros((N4, Vf, 12), dtype=torch.complex128, device="cuda")
        B[: N4 // 2, :, :6] = half[:, :, :6]
        B[N4 // 2:, :, 6:] = half[:, :, 6:]
        ag = gmg.Aggregation(fd, cd, 12, N4)
        ag.set_basis(B)
        ag.Orthogonalise(passes=1)
        cm = gmg.CoarsenedMatrix(cd, N4)
        for _ in range(2):
            cm.CoarsenOperator(ag, w)
        torch.cuda.synchronize()
        line("p_c4 CoarsenOperator 16^4 -> 4^4, nbasis 40", ok=True)


def run(rows=("c1", "c3", "w_c4", "c5")):
    torch.cuda.set_device(0)
    hbm, src = peaks()
    T = Timer()
    if "c1" in rows:
        c1(T, hbm)
    if "c3" in rows:
        c3(T, hbm)
        torch.cuda.empty_cache()
    if "w_c4" in rows:
        wilson_and_c4(T, hbm)
        torch.cuda.empty_cache()
    if "c5" in rows:
        c5()
    if "c5s" in rows:
        c5_small()
    if any(r.startswith("p_") for r in rows):
        profile_rows(rows)
        return
    line("peaks", hbm_gbs=hbm, source=src)

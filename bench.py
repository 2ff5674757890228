#!/usr/bin/env python
"""Benchmark of the multi-RHS coarse stencil (the multigrid hot path's Mrhs apply).

Workload: coarse 8^4 lattice, nbasis 32, 32 right-hand sides, one M apply per
step (the multi-RHS coarse-stencil configuration: coarse operator of a 32^4
Wilson-clover lattice on 4^4 blocks).  Links are seeded Gaussian with the
gamma5-hermitian structure a Galerkin coarsening produces, RHS unit Gaussian.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line on rank 0.  `value` is whole-job TFLOP/s (algorithmic
flops 8 * V * 9 * N^2 * R per apply) with inputs resident in HBM and L2
flushed between steps; `e2e` is the same metric through the public C ABI call
with the RHS copied in from pinned host memory and the result copied back every
step.  --impl reference times the CPU implementation of the path (the FP64
oracle restatement, all host threads) on bounded site samples of the same
workload.  Multi-GPU runs are independent replicas (the path has no exchange
on one GPU per lattice), timed on the device as the max over ranks.
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "grid-mg-bench_b200"))

import numpy as np  # noqa: E402

DIMS = (8, 8, 8, 8)
NBASIS = 32
NRHS = 32
V = int(np.prod(DIMS))
FLOPS = 8.0 * V * 9 * NBASIS * NBASIS * NRHS  # 9.664 GFLOP per apply
METRIC = "coarse Mrhs stencil M apply throughput (8^4 coarse lattice, nbasis 32, 32 RHS)"
UNIT = "TFLOP/s"
VEC_BYTES_F32 = V * NRHS * NBASIS * 8  # one FP32 coarse field of 32 RHS
# algorithmic bytes of the dominant kernel (tensor-core stencil on packed BF16 input):
#   BF16 links 9*V*N^2*4 + packed BF16 input V*R*N*4 + FP32 output V*R*N*8
TC_KERNEL_BYTES = 9 * V * NBASIS * NBASIS * 4 + V * NRHS * NBASIS * 4 + V * NRHS * NBASIS * 8
# algorithmic bytes of the whole apply (BF16 links + FP32 in + FP32 out)
APPLY_BYTES = 9 * V * NBASIS * NBASIS * 4 + 2 * VEC_BYTES_F32
L2_FLUSH_BYTES = 256 << 20


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--form", choices=["bf16", "f16"], default="bf16")
    ap.add_argument("--suite", action="store_true",
                    help="per-row measurements (C1, C3, C4, fine operator) instead of the bench line")
    ap.add_argument("--rows", default="c1,c3,w_c4,c5", help="suite rows to run")
    ap.add_argument("--no-mg", action="store_true",
                    help="skip the 3-level MG solve measurement (32^4 Wilson-clover, 24 RHS) of the JSON line")
    ap.add_argument("--kernel-only", action="store_true",
                    help="only warm-up + timed applies (for profiler captures); prints a short line")
    ap.add_argument("--flush", choices=["write+read", "write"], default="write+read",
                    help="L2 flush between timed steps: 256 MiB written then another 256 MiB read (the default: "
                         "the written lines are written back before the step), or the write alone")
    return ap.parse_args()


def make_inputs():
    import inputs

    r = inputs.rng(stream=4242)
    A = inputs.random_links(DIMS, NBASIS, r)
    x = inputs.gaussian_field((V, NRHS, NBASIS), r)
    return A, x


# DRAM traffic (dram__bytes_read.sum + dram__bytes_write.sum) of one
# coarse_mrhs_tc_kernel launch on this workload, from one ncu capture of the
# kernel as built (a constant: an ncu capture cannot run inside the timed bench):
#   python bench.py --kernel-only --steps 3 --warmup 2 && \
#   ncu --set full --clock-control none -k regex:coarse_mrhs_tc -s 3 -c 1 -o prof_tc \
#       python bench.py --kernel-only --steps 3 --warmup 2
#   ncu -i prof_tc.ncu-rep --page raw --csv   (read 172.1 MB + write 21.4 MB)
TC_KERNEL_TRAFFIC = 193483008


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# ----------------------------------------------------------------------------- CPU side
def cpu_sample(A, x, target_s=12.0, max_reps=400, min_reps=5):
    """FP64 oracle apply on the host cores: full applies on all threads until
    ~target_s of work (at least min_reps), reported as the median repetition,
    then the same at 1 thread on a 1/16 site sample (median of min_reps)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as orc

    y = np.empty_like(x)
    threads = os.cpu_count()
    orc.set_threads(threads)
    orc.coarse_apply_range(DIMS, A, x, y, 0, V)  # warm-up
    times = []
    while len(times) < max_reps and (sum(times) < target_s or len(times) < min_reps):
        t0 = time.perf_counter()
        orc.coarse_apply_range(DIMS, A, x, y, 0, V)
        times.append(time.perf_counter() - t0)
    t_med = float(np.median(times))
    ns1 = V // 16
    orc.set_threads(1)
    orc.coarse_apply_range(DIMS, A, x, y, 0, ns1)
    t1 = []
    for _ in range(min_reps):
        t0 = time.perf_counter()
        orc.coarse_apply_range(DIMS, A, x, y, 0, ns1)
        t1.append(time.perf_counter() - t0)
    orc.set_threads(threads)
    one = FLOPS * ns1 / V / float(np.median(t1)) / 1e12
    return {
        "value": FLOPS / t_med / 1e12,
        "unit": UNIT,
        "cores": threads,
        "kind": "port",
        "sample": f"median of {len(times)} full M applies (8^4, nbasis 32, 32 RHS, FP64) with the C++/OpenMP "
                  f"oracle on {threads} threads ({sum(times):.1f} s in all)",
        "one_thread": {"value": one, "unit": UNIT,
                       "sample": f"median of {min_reps} applies over {ns1} of {V} output sites, 1 thread"},
    }, y


def max_over_ranks(v, dist, device):
    """The largest of every rank's v (a device time in ms): the job ends with its slowest rank."""
    if dist is None:
        return float(v)
    import torch

    t = torch.tensor([float(v)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def run_reference(args, rank):
    """CPU implementation of the path (FP64 oracle restatement) on bounded site samples."""
    if rank != 0:
        return 0
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as orc

    A, x = make_inputs()
    A = np.ascontiguousarray(A)
    y = np.empty_like(x)
    t0 = time.perf_counter()
    orc.coarse_apply_range(DIMS, A, x, y, 0, V)
    t_full = time.perf_counter() - t0
    budget = 150.0  # whole run within a few minutes
    per_step = min(t_full, budget / max(1, args.steps + args.warmup))
    nsites = max(16, min(V, int(V * per_step / t_full)))
    for i in range(args.warmup):
        s0 = (i * nsites) % (V - nsites + 1)
        orc.coarse_apply_range(DIMS, A, x, y, s0, s0 + nsites)
    tot = 0.0
    for i in range(args.steps):
        s0 = (i * nsites) % (V - nsites + 1)
        t0 = time.perf_counter()
        orc.coarse_apply_range(DIMS, A, x, y, s0, s0 + nsites)
        tot += time.perf_counter() - t0
    flops = FLOPS * nsites / V * args.steps
    val = flops / tot / 1e12
    line = {
        "metric": METRIC, "value": val, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": config_dict(),
        "form": "FP64 CPU restatement of CoarsenedMatrix::M (the oracle, C++/OpenMP)",
        "cpu_baseline": {"value": val, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
                         "sample": f"{nsites} of {V} output sites per step (all 32 RHS), FP64, "
                                   f"{os.cpu_count()} OpenMP threads; Grid, which the reference "
                                   f"needs, is not installable here"},
        "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def config_dict():
    """The workload, the same for both arms (how each arm computes it is in `form` and `dtype`)."""
    return {
        "workload": "multi-RHS coarse stencil M apply: coarse 8^4, nbasis 32, 32 RHS "
                    "(coarse operator of 32^4 Wilson-clover on 4^4 blocks)",
        "coarse_dims": list(DIMS), "nbasis": NBASIS, "nrhs": NRHS, "op": "M",
        "l2": "flushed between timed steps: 256 MiB written, then 256 MiB of a second buffer read, so that the "
              "flush's dirty lines are written back before the step starts; inputs and links are not in L2",
        "parallelism": "replicas",
    }


# ----------------------------------------------------------------------------- clocks
class ClockSampler:
    def __init__(self, gpu_index):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(gpu_index), f"--query-gpu={q}",
                                       "--format=csv,noheader,nounits", "-lms", "100"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        time.sleep(0.25)
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.f.flush()
        rows = []
        with open(self.f.name) as fh:
            for line in fh:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.f.name)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = max(float(r[2]) for r in rows if r[2].replace(".", "").isdigit())
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": reasons,
                "samples": len(rows)}


# ----------------------------------------------------------------------------- GPU side
def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank)
    if args.suite:
        import suite

        suite.run(tuple(args.rows.split(",")))
        return 0

    import torch

    import gmg

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local)
    A, x = make_inputs()
    cm = gmg.CoarsenedMatrix(DIMS, NBASIS)
    cm.set_links(A)
    cm.prepare(args.form)
    cm.prepare("f32")
    xin64 = torch.from_numpy(x).to(dev)
    xin = xin64.to(torch.complex64).contiguous()
    out = torch.zeros_like(xin)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    flush_rd = torch.ones(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    flush_sum = torch.empty((), dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream()

    def l2_flush(k, mode=None):
        """Evict the step's operands from L2: write 256 MiB; then (write+read) read another
        256 MiB, which writes the written lines back to DRAM before the step instead of
        during it (a write-only flush leaves ~126 MB of dirty lines that the next step's
        first kernel pays to evict)."""
        flush.fill_(float(k))
        if (mode or args.flush) == "write+read":
            torch.sum(flush_rd, dim=0, out=flush_sum)

    # accuracy of each form against the FP64 GPU path (itself pinned to the oracle)
    ref64 = torch.zeros_like(xin64)
    cm.M(xin64, ref64)
    forms = {}
    for form in (args.form, "f32"):
        o = torch.zeros_like(xin)
        cm.M(xin, o, compute=form)
        torch.cuda.synchronize()
        err = (torch.linalg.vector_norm(o.to(torch.complex128) - ref64) / torch.linalg.vector_norm(ref64)).item()
        forms[form] = {"rel_err_vs_fp64": err}

    def step(compute):
        cm.M(xin, out, compute=compute)

    for _ in range(args.warmup):
        step(args.form)
    torch.cuda.synchronize()
    if args.kernel_only:
        for k in range(args.steps):
            l2_flush(k)
            step(args.form)
        torch.cuda.synchronize()
        print(json.dumps({"kernel_only": True, "steps": args.steps, "form": args.form}))
        return 0

    # timed region: K steps, L2 flushed between steps (outside the per-step events).
    # The library's per-kernel events (gmg_profile_enable) put two more event
    # records inside every step, and each adds a gap of about 3 us between the
    # step's kernels; so the step time comes from this pass, without them, and
    # the kernels' own durations from a second pass of the same K steps with them.
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    if dist:
        dist.barrier()
    sampler = ClockSampler(local) if rank == 0 else None
    torch.cuda.synchronize()
    for k in range(args.steps):
        l2_flush(k)
        ev[k][0].record(stream)
        step(args.form)
        ev[k][1].record(stream)
    torch.cuda.synchronize()
    clocks = sampler.stop() if sampler else None
    t_ms = sum(a.elapsed_time(b) for a, b in ev)
    # the same steps after a write-only flush, for comparison (not the value)
    for k in range(args.steps):
        l2_flush(k, "write")
        ev[k][0].record(stream)
        step(args.form)
        ev[k][1].record(stream)
    torch.cuda.synchronize()
    t_write_only = sum(a.elapsed_time(b) for a, b in ev)
    if dist:
        dist.barrier()
    import ctypes

    # kernel-duration pass: the same K steps with the per-kernel events on
    gmg.lib().gmg_profile_enable(1)
    for k in range(args.steps):
        l2_flush(k)
        step(args.form)
    torch.cuda.synchronize()
    gmg.lib().gmg_profile_enable(0)
    kms, kn = ctypes.c_double(), ctypes.c_int64()
    gmg.lib().gmg_profile_read(b"coarse_mrhs_tc", ctypes.byref(kms), ctypes.byref(kn))
    pms, pn = ctypes.c_double(), ctypes.c_int64()
    gmg.lib().gmg_profile_read(b"pack_vec", ctypes.byref(pms), ctypes.byref(pn))
    code = np.zeros(1, dtype=np.int32)
    st = gmg.lib().gmg_coarse_device_error(cm._h, code.ctypes.data_as(ctypes.c_void_p))
    if st != 0:
        raise RuntimeError("tensor-core kernel reported a device error: " + gmg.lib().gmg_last_error().decode())
    t_ms = max_over_ranks(t_ms, dist, dev)
    value = world * FLOPS * args.steps / (t_ms * 1e-3) / 1e12

    # other forms (fewer steps): FP32 CUDA-core and FP64 CUDA-core
    for form, inp, o in (("f32", xin, torch.zeros_like(xin)), ("f64", xin64, torch.zeros_like(xin64))):
        n = max(5, min(50, args.steps // 10))
        for _ in range(3):
            cm.M(inp, o, compute=form)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        tt = 0.0
        for kk in range(n):
            l2_flush(kk)
            e0.record(stream)
            cm.M(inp, o, compute=form)
            e1.record(stream)
            e1.synchronize()
            tt += e0.elapsed_time(e1)
        forms.setdefault(form, {})["tflops"] = FLOPS * n / (tt * 1e-3) / 1e12
    forms[args.form]["tflops"] = FLOPS * args.steps / (t_ms * 1e-3) / 1e12 / 1.0
    forms["f64"]["rel_err_vs_fp64"] = 0.0

    # end to end through the public API with host buffers (pinned), every step:
    # copy the step's input in, apply, copy the result out.  Double-buffered
    # over three streams so that step k+1's copy-in and step k-1's copy-out
    # (separate copy engines) overlap step k's apply; every step still moves
    # its whole input and result across PCIe.
    s_in, s_cmp, s_out = torch.cuda.Stream(), torch.cuda.Stream(), torch.cuda.Stream()
    ne = max(10, min(200, args.steps // 10))

    def e2e_measure(compute, xhost):
        host_in = torch.from_numpy(xhost).pin_memory()
        host_out = torch.empty_like(host_in).pin_memory()
        dev_in = [torch.empty(host_in.shape, dtype=host_in.dtype, device=dev) for _ in range(2)]
        dev_out = [torch.empty_like(d) for d in dev_in]

        def run(nsteps, e0=None, e1=None):
            ev_in = [torch.cuda.Event() for _ in range(nsteps)]
            ev_cmp = [torch.cuda.Event() for _ in range(nsteps)]
            ev_out = [torch.cuda.Event() for _ in range(nsteps)]
            s_in.wait_stream(torch.cuda.current_stream())
            if e0 is not None:
                e0.record(s_in)
            for k in range(nsteps):
                b = k % 2
                with torch.cuda.stream(s_in):
                    if k >= 2:
                        s_in.wait_event(ev_cmp[k - 2])  # dev_in[b] no longer read
                    dev_in[b].copy_(host_in, non_blocking=True)
                    ev_in[k].record(s_in)
                with torch.cuda.stream(s_cmp):
                    s_cmp.wait_event(ev_in[k])
                    if k >= 2:
                        s_cmp.wait_event(ev_out[k - 2])  # dev_out[b] copied out
                    cm.M(dev_in[b], dev_out[b], compute=compute)
                    ev_cmp[k].record(s_cmp)
                with torch.cuda.stream(s_out):
                    s_out.wait_event(ev_cmp[k])
                    host_out.copy_(dev_out[b], non_blocking=True)
                    ev_out[k].record(s_out)
            s_out.wait_stream(s_in)
            s_out.wait_stream(s_cmp)
            if e1 is not None:
                e1.record(s_out)
            torch.cuda.synchronize()

        run(3)
        if dist:
            dist.barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        run(ne, e0, e1)
        te = max_over_ranks(e0.elapsed_time(e1), dist, dev)
        return world * FLOPS * ne / (te * 1e-3) / 1e12, int(host_in.numel() * host_in.element_size())

    e2e, e2e_bytes = e2e_measure(args.form, x.astype(np.complex64))
    # the same apply in FP64 (links and vectors), the reference's own arithmetic:
    # device-timed steps (L2 flushed) and end to end with complex128 host buffers
    n64 = max(5, min(100, args.steps))
    o64 = torch.zeros_like(xin64)
    for _ in range(3):
        cm.M(xin64, o64, compute="f64")
    ev64 = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(n64)]
    torch.cuda.synchronize()
    for k in range(n64):
        l2_flush(k)
        ev64[k][0].record(stream)
        cm.M(xin64, o64, compute="f64")
        ev64[k][1].record(stream)
    torch.cuda.synchronize()
    t64 = max_over_ranks(sum(a.elapsed_time(b) for a, b in ev64), dist, dev)
    e2e64, e2e64_bytes = e2e_measure("f64", x)
    f64_leg = {
        "value": world * FLOPS * n64 / (t64 * 1e-3) / 1e12, "unit": UNIT, "steps": n64,
        "ms_per_step": t64 / n64, "dtype": "f64",
        "form": "FP64 links and vectors on the CUDA cores (coarse_simt_pipe_kernel), the arithmetic of the reference "
                "and of its CPU arm",
        "e2e": {"value": e2e64, "unit": UNIT, "h2d_bytes_per_step": e2e64_bytes, "d2h_bytes_per_step": e2e64_bytes,
                "how": "public gmg_coarse_apply (compute F64) with pinned complex128 host input/output every step, "
                       "double-buffered as the headline e2e"},
    }

    hbm, src = peaks()
    kavg_s = (kms.value / max(kn.value, 1)) * 1e-3
    tc_ctas, tc_pps = ctypes.c_int(), ctypes.c_int()
    gmg.lib().gmg_coarse_tuned_shape(cm._h, NRHS, 9, gmg.PREC[args.form], ctypes.byref(tc_ctas),
                                     ctypes.byref(tc_pps))
    achieved = TC_KERNEL_BYTES / kavg_s / 1e9 if kn.value else None
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": args.form,
        "data": "synthetic (seeded Gaussian links with gamma5-hermitian structure, unit-Gaussian RHS)",
        "config": config_dict(),
        "form": f"{args.form} operands on tcgen05 tensor cores, FP32 accumulation, FP32 vectors",
        "tile": {"ctas_per_sm": tc_ctas.value, "points_per_stage": tc_pps.value,
                 "chosen_by": "autotuner (first apply times every shape that fits)"},
        "roofline": {
            "bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
            "frac": (achieved / hbm) if achieved else None, "traffic": TC_KERNEL_TRAFFIC,
            "traffic_source": "one ncu --set full capture of this kernel on this workload "
                              "(dram__bytes_read.sum + dram__bytes_write.sum)",
            "kernel": "coarse_mrhs_tc_kernel", "algorithmic_bytes_per_launch": TC_KERNEL_BYTES,
            "kernel_ms_avg": kavg_s * 1e3, "launches": kn.value,
            "timing": "CUDA events around every launch on its stream, over a second pass of the same K steps "
                      "(the step time comes from a pass without these events)",
            "pack_kernel_ms_avg": (pms.value / pn.value) if pn.value else None,
            "peak_source": f"MEASURED_PEAKS.json hbm_gbs ({src})",
        },
        "apply_roofline": {"algorithmic_bytes": APPLY_BYTES,
                           "achieved_gbs": APPLY_BYTES / (t_ms * 1e-3 / args.steps) / 1e9},
        "l2_flush": {"mode": args.flush,
                     "write_only_flush_ms_per_step": t_write_only / args.steps,
                     "note": "the same steps timed after a write-only flush, whose dirty lines the step evicts"},
        "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": e2e_bytes,
                "d2h_bytes_per_step": e2e_bytes,
                "how": "public gmg_coarse_apply with pinned host input/output every step; double-buffered on "
                       "three streams: step k+1's copy-in and step k-1's copy-out overlap step k"},
        "gpu_launches": 2 * args.steps,
        "clocks": clocks,
        "forms": forms,
        "f64_leg": f64_leg,
    }
    if rank == 0 and world == 1:
        cpu, _ = cpu_sample(A, x)
        line["cpu_baseline"] = cpu
    if not args.no_mg:
        # the MG solve half of the metric: 3-level K-cycle FGMRES on 32^4 Wilson-clover,
        # 24 RHS to 1e-10: the mixed BF16 multi-RHS form with the K-cycle replayed as a
        # CUDA graph (timed on its second solve; the first also captures), the same
        # form host-driven, and the plain FP64 single-RHS form on all 24 RHS one at a
        # time; setup not in the solve times
        torch.cuda.empty_cache()
        import suite

        mg = suite.c5_measure(nrhs=24, plain_rhs=24,
                              forms=("mixed_bf16_mrhs_graph", "mixed_bf16_mrhs", "plain_f64_single_rhs"))
        line["mg_solve"] = {
            "workload": "3-level K-cycle MG-preconditioned FGMRES, 32^4 Wilson-clover m=-0.35 csw 1, "
                        "nbasis 24 / 32 on 4^4 / 2^4 blocks, 8 MR smoother iterations per level, "
                        "24 RHS to 1e-10",
            "forms": {"mixed_bf16_mrhs": "outer FGMRES(8): every restart cycle starts from the FP64 residual "
                                         "b - A x and runs its Arnoldi process in FP32 (FP64 inner products, "
                                         "Hessenberg least squares and solution; tolerance checked on the FP64 "
                                         "residual); K-cycle with FP32 vectors, tensor-core BF16 coarse stencils "
                                         "and the fine MR smoother's residual fields in BF16 (FP32 arithmetic); "
                                         "24 RHS in one batch, converged RHS leave at their Arnoldi step",
                      "plain_f64_single_rhs": "the same algorithm with FP64 everywhere, one RHS per solve"},
            "unit": "s", "higher_is_better": False,
            "mixed_bf16_mrhs_graph_s": mg["mixed_bf16_mrhs_graph"]["solve_s_for_all_rhs"],
            "mixed_bf16_mrhs_graph_first_solve_s": mg["mixed_bf16_mrhs_graph"]["first_solve_s"],
            "mixed_bf16_mrhs_host_driven_s": mg["mixed_bf16_mrhs"]["solve_s_for_all_rhs"],
            "plain_f64_single_rhs_s": mg["plain_f64_single_rhs"]["solve_s_for_all_rhs"],
            "plain_f64_rhs_measured": mg["plain_f64_single_rhs"]["rhs_measured"],
            "speedup_vs_plain_f64": mg["mixed_bf16_mrhs_graph"]["speedup_vs_plain_f64"],
            "details": mg,
        }
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())

"""The allocation-free tensor-core apply, gmg_coarse_apply_noalloc, called through the C ABI.

Callers that cannot let the library allocate while they run (a solver loop
that must not stall the device, or an application whose device memory all
comes from its own pool) use this entry point: it keeps the packed
right-hand sides in a fixed 16 MiB device array instead of a buffer it would
cudaMalloc.  Its results must equal those of the allocating gmg_coarse_apply,
on two calls in a row (the array is shared and keeps the previous call's
contents), within the tensor-core tolerance: relative squared deviation 2e-5
for BF16 and 1e-6 for FP16.  The cases cover M and Mdag, a single stencil
point other than the self point, an active-RHS list shorter than the batch,
both operand kinds, and a fresh handle whose first tensor-core apply is the
allocation-free one (it does not tune, so it runs the heuristic launch shape
while the allocating apply afterwards tunes one).  Requests larger than the
array are rejected with GMG_ERR_UNSUPPORTED.  This file is collected last on
purpose.
"""
import ctypes

import numpy as np
import pytest
import torch

import gmg
import inputs

pytestmark = pytest.mark.gpu

TOL = {"bf16": 2e-5, "f16": 1e-6}
KIND = {"bf16": gmg.BF16, "f16": gmg.F16}
GMG_ERR_UNSUPPORTED = 6


def _noalloc(cm, op, x, out, point=8, kind="bf16", active=None):
    act, n_act = None, 0
    if active is not None:
        act, n_act = ctypes.c_void_p(active.data_ptr()), int(active.numel())
    return gmg.lib().gmg_coarse_apply_noalloc(cm._h, op, point, KIND[kind], x.shape[1],
                                              ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(out.data_ptr()),
                                              act, n_act, ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))


def _rel_sq(a, b):
    return float((torch.linalg.vector_norm(a - b) ** 2 / torch.linalg.vector_norm(a) ** 2).item())


def _device_error_clear(cm):
    code = np.zeros(1, dtype=np.int32)
    assert gmg.lib().gmg_coarse_device_error(cm._h, code.ctypes.data_as(ctypes.c_void_p)) == 0


def _handle(dims, N, stream, kind):
    cm = gmg.CoarsenedMatrix(dims, N)
    cm.set_links(inputs.random_links(dims, N, inputs.rng(stream=stream)))
    cm.prepare(kind)
    return cm


def _rhs(V, R, N, stream):
    return torch.from_numpy(inputs.gaussian_field((V, R, N), inputs.rng(stream=stream))).cuda().to(torch.complex64)


def test_noalloc_matches_allocating_apply_on_two_calls():
    dims, N, R = (4, 4, 8, 4), 32, 24
    cm = _handle(dims, N, 990, "bf16")
    V = int(np.prod(dims))
    # two different inputs and two ops in a row: the second call must not see the first one's data
    for op, stream in ((gmg.OP_M, 991), (gmg.OP_MDAG, 992)):
        x = _rhs(V, R, N, stream)
        ref = torch.zeros_like(x)
        cm.apply(op, x, ref, compute="bf16")
        got = torch.full_like(x, float("nan"))
        assert _noalloc(cm, op, x, got) == 0, gmg.lib().gmg_last_error().decode()
        torch.cuda.synchronize()
        assert _rel_sq(ref, got) < TOL["bf16"]
        assert torch.equal(ref, got)  # same kernels on the same packed data
    _device_error_clear(cm)


@pytest.mark.parametrize("kind", ["bf16", "f16"])
def test_noalloc_first_on_a_fresh_handle(kind):
    # the allocation-free apply is the handle's first tensor-core apply: no
    # launch shape is tuned yet, so it runs the heuristic one; the allocating
    # apply afterwards tunes and may pick another shape, which sums the same
    # products in the same order
    dims, N, R = (4, 4, 4, 4), 32, 32
    cm = _handle(dims, N, 994, kind)
    V = int(np.prod(dims))
    for op, stream in ((gmg.OP_M, 995), (gmg.OP_MDAG, 996)):
        x = _rhs(V, R, N, stream)
        got = torch.full_like(x, float("nan"))
        assert _noalloc(cm, op, x, got, kind=kind) == 0, gmg.lib().gmg_last_error().decode()
        ref = torch.zeros_like(x)
        cm.apply(op, x, ref, compute=kind)
        torch.cuda.synchronize()
        assert _rel_sq(ref, got) < TOL[kind]
    _device_error_clear(cm)


@pytest.mark.parametrize("kind", ["bf16", "f16"])
def test_noalloc_single_point_and_active_subset(kind):
    # Mdir at a hopping point (not the self point 8), then M over an active
    # list shorter than the batch, twice in a row each; slots outside the
    # active list stay untouched
    dims, N, R = (4, 2, 4, 4), 24, 12
    cm = _handle(dims, N, 997, kind)
    V = int(np.prod(dims))
    for point, stream in ((5, 998), (2, 999)):
        x = _rhs(V, R, N, stream)
        ref = torch.zeros_like(x)
        cm.apply(gmg.OP_MDIR, x, ref, point=point, compute=kind)
        got = torch.full_like(x, float("nan"))
        assert _noalloc(cm, gmg.OP_MDIR, x, got, point=point, kind=kind) == 0, gmg.lib().gmg_last_error().decode()
        torch.cuda.synchronize()
        assert _rel_sq(ref, got) < TOL[kind]
    active = torch.tensor([11, 0, 7, 3, 9], dtype=torch.int32, device="cuda")
    for stream in (1000, 1001):
        x = _rhs(V, R, N, stream)
        ref = torch.full_like(x, 5.0)
        cm.apply(gmg.OP_M, x, ref, compute=kind, active=active)
        got = torch.full_like(x, 5.0)
        assert _noalloc(cm, gmg.OP_M, x, got, kind=kind, active=active) == 0, gmg.lib().gmg_last_error().decode()
        torch.cuda.synchronize()
        sel = active.long()
        assert _rel_sq(ref[:, sel], got[:, sel]) < TOL[kind]
        rest = torch.ones(R, dtype=torch.bool, device="cuda")
        rest[sel] = False
        assert bool((got[:, rest] == 5.0).all())
    _device_error_clear(cm)


def test_noalloc_rejects_requests_beyond_the_static_array():
    dims, N, R = (8, 8, 8, 8), 32, 128  # packed RHS need 64 MiB > 16 MiB
    cm = _handle(dims, N, 993, "bf16")
    x = torch.zeros((4096, R, N), dtype=torch.complex64, device="cuda")
    out = torch.zeros_like(x)
    assert _noalloc(cm, gmg.OP_M, x, out) == GMG_ERR_UNSUPPORTED
    assert b"16 MiB" in gmg.lib().gmg_last_error()

"""The allocation-free tensor-core apply, gmg_coarse_apply_noalloc, called through the C ABI.

Callers that cannot let the library allocate while they run (a solver loop
that must not stall the device, or an application whose device memory all
comes from its own pool) use this entry point: it keeps the packed
right-hand sides in a fixed 16 MiB device array instead of a buffer it would
cudaMalloc.  Its results must equal those of the allocating gmg_coarse_apply,
on two calls in a row (the array is shared and keeps the previous call's
contents), within the tensor-core tolerance: relative squared deviation 2e-5
for BF16.  Requests larger than the array are rejected with
GMG_ERR_UNSUPPORTED.  This file is collected last on purpose.
"""
import ctypes

import numpy as np
import pytest
import torch

import gmg
import inputs

pytestmark = pytest.mark.gpu

TOL_BF16 = 2e-5
GMG_ERR_UNSUPPORTED = 6


def _noalloc(cm, op, x, out, point=8):
    return gmg.lib().gmg_coarse_apply_noalloc(cm._h, op, point, gmg.BF16, x.shape[1],
                                              ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(out.data_ptr()),
                                              None, 0, ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))


def _rel_sq(a, b):
    return float((torch.linalg.vector_norm(a - b) ** 2 / torch.linalg.vector_norm(a) ** 2).item())


def test_noalloc_matches_allocating_apply_on_two_calls():
    dims, N, R = (4, 4, 8, 4), 32, 24
    r = inputs.rng(stream=990)
    A = inputs.random_links(dims, N, r)
    cm = gmg.CoarsenedMatrix(dims, N)
    cm.set_links(A)
    cm.prepare("bf16")
    V = int(np.prod(dims))
    # two different inputs and two ops in a row: the second call must not see the first one's data
    for op, stream in ((gmg.OP_M, 991), (gmg.OP_MDAG, 992)):
        x = torch.from_numpy(inputs.gaussian_field((V, R, N), inputs.rng(stream=stream))).cuda().to(torch.complex64)
        ref = torch.zeros_like(x)
        cm.apply(op, x, ref, compute="bf16")
        got = torch.full_like(x, float("nan"))
        assert _noalloc(cm, op, x, got) == 0, gmg.lib().gmg_last_error().decode()
        torch.cuda.synchronize()
        assert _rel_sq(ref, got) < TOL_BF16
        assert torch.equal(ref, got)  # same kernels on the same packed data
    code = np.zeros(1, dtype=np.int32)
    assert gmg.lib().gmg_coarse_device_error(cm._h, code.ctypes.data_as(ctypes.c_void_p)) == 0


def test_noalloc_rejects_requests_beyond_the_static_array():
    dims, N, R = (8, 8, 8, 8), 32, 128  # packed RHS need 64 MiB > 16 MiB
    cm = gmg.CoarsenedMatrix(dims, N)
    cm.set_links(inputs.random_links(dims, N, inputs.rng(stream=993)))
    cm.prepare("bf16")
    x = torch.zeros((4096, R, N), dtype=torch.complex64, device="cuda")
    out = torch.zeros_like(x)
    assert _noalloc(cm, gmg.OP_M, x, out) == GMG_ERR_UNSUPPORTED
    assert b"16 MiB" in gmg.lib().gmg_last_error()

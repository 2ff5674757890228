"""Tensor-core block projection and promotion (BF16 hi+lo operands, FP32 accumulation) against the FP64 oracle.

Both operands are split into two BF16 parts (about 16 significant bits) and
three products are accumulated in FP32, so the stated bound on the relative
squared deviation |ref-res|^2/|ref|^2 is 1e-8 (1e-4 in norm); in practice it
sits near 1e-11.
"""
import numpy as np
import pytest
import torch

import gmg
import inputs
import oracle as orc

pytestmark = pytest.mark.gpu

TOL = 1e-8


@pytest.mark.parametrize("fd,cd,dof,N,R", [
    ((8, 8, 8, 8), (2, 2, 2, 2), 12, 32, 32),   # 4^4 blocks, nbasis 32, 32 RHS (the C3 shape, smaller lattice)
    ((8, 8, 4, 4), (2, 2, 2, 2), 12, 8, 5),     # ragged RHS count, 2 RHS tiles of padding
    ((4, 4, 4, 4), (2, 2, 2, 2), 24, 16, 16),   # coarse-of-coarse: site dof = nbasis of the level above
    ((8, 4, 4, 4), (2, 2, 2, 2), 40, 40, 3),    # nbasis 40 (M = 128 rows), dof 40
])
def test_project_tc_matches_oracle(fd, cd, dof, N, R):
    Vf = int(np.prod(fd))
    r = inputs.rng(stream=400 + N + R)
    B = inputs.gaussian_field((N, Vf, dof), r)
    B = orc.block_orthonormalise(fd, cd, B, passes=1)
    f = inputs.gaussian_field((Vf, R, dof), r)
    ag = gmg.Aggregation(fd, cd, dof, N)
    ag.set_basis(B)
    ref = orc.block_project(fd, cd, B, f)
    out = torch.zeros((int(np.prod(cd)), R, N), dtype=torch.complex64, device="cuda")
    ag.ProjectToSubspace(torch.from_numpy(f).cuda().to(torch.complex64), out, compute="bf16")
    torch.cuda.synchronize()
    got = out.cpu().numpy().astype(np.complex128)
    dev = orc.rel_dev_sq(ref, got)
    assert dev < TOL, dev


def test_project_tc_follows_basis_changes():
    fd, cd, dof, N, R = (4, 4, 4, 4), (2, 2, 2, 2), 12, 8, 4
    r = inputs.rng(stream=450)
    B1 = orc.block_orthonormalise(fd, cd, inputs.gaussian_field((N, 256, dof), r), passes=1)
    B2 = orc.block_orthonormalise(fd, cd, inputs.gaussian_field((N, 256, dof), r), passes=1)
    f = inputs.gaussian_field((256, R, dof), r)
    ag = gmg.Aggregation(fd, cd, dof, N)
    ag.set_basis(B1)
    x = torch.from_numpy(f).cuda().to(torch.complex64)
    out = torch.zeros((16, R, N), dtype=torch.complex64, device="cuda")
    ag.ProjectToSubspace(x, out, compute="bf16")
    ag.set_basis(B2)  # the packed tensor-core copy must be rebuilt
    ag.ProjectToSubspace(x, out, compute="bf16")
    torch.cuda.synchronize()
    assert orc.rel_dev_sq(orc.block_project(fd, cd, B2, f), out.cpu().numpy().astype(np.complex128)) < TOL


@pytest.mark.parametrize("fd,cd,dof,N,R", [
    ((8, 8, 8, 8), (2, 2, 2, 2), 12, 32, 32),   # K = 3072 fine dofs per block: 24 M tiles of 128
    ((8, 8, 4, 4), (2, 2, 2, 2), 12, 8, 5),     # 2N = 16, ragged RHS count
    ((4, 4, 4, 4), (2, 2, 2, 2), 24, 12, 16),   # 2N = 24: K padded to 32 with zero rows of B
    ((8, 4, 4, 4), (2, 2, 2, 2), 40, 40, 3),    # nbasis 40 (Mp = 128), K = 2560
])
def test_promote_tc_matches_oracle(fd, cd, dof, N, R):
    Vf, Vc = int(np.prod(fd)), int(np.prod(cd))
    r = inputs.rng(stream=500 + N + R)
    B = orc.block_orthonormalise(fd, cd, inputs.gaussian_field((N, Vf, dof), r), passes=1)
    c = inputs.gaussian_field((Vc, R, N), r)
    ag = gmg.Aggregation(fd, cd, dof, N)
    ag.set_basis(B)
    ref = orc.block_promote(fd, cd, B, c)
    out = torch.full((Vf, R, dof), float("nan"), dtype=torch.complex64, device="cuda")  # every entry is written
    ag.PromoteFromSubspace(torch.from_numpy(c).cuda().to(torch.complex64), out, compute="bf16")
    torch.cuda.synchronize()
    got = out.cpu().numpy().astype(np.complex128)
    assert np.isfinite(got).all()
    assert orc.rel_dev_sq(ref, got) < TOL


def test_promote_then_project_is_identity_tc():
    # P^dag P = 1 on the coarse space for an orthonormal basis
    fd, cd, dof, N, R = (8, 8, 4, 4), (2, 2, 2, 2), 12, 16, 8
    r = inputs.rng(stream=550)
    B = orc.block_orthonormalise(fd, cd, inputs.gaussian_field((N, 1024, dof), r), passes=2)
    c = torch.from_numpy(inputs.gaussian_field((16, R, N), r)).cuda().to(torch.complex64)
    ag = gmg.Aggregation(fd, cd, dof, N)
    ag.set_basis(B)
    f = torch.zeros((1024, R, dof), dtype=torch.complex64, device="cuda")
    back = torch.zeros_like(c)
    ag.PromoteFromSubspace(c, f, compute="bf16")
    ag.ProjectToSubspace(f, back, compute="bf16")
    torch.cuda.synchronize()
    d = (back - c).abs().pow(2).sum().item() / c.abs().pow(2).sum().item()
    assert d < TOL, d

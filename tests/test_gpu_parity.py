"""GPU parity of the CUDA path (through the C ABI) against the FP64 CPU oracle.

Tolerances are the reference's relative squared deviation |ref-res|^2/|ref|^2
(include/Benchmark_helpers.h:215-236): 1e-15 for FP64 (src/Benchmark_coarse_operator.cc:81)
and 1e-7 for FP32; tensor-core forms state their own bound in their tests.
"""
import numpy as np
import pytest
import torch

import gmg
import inputs
import oracle as orc

pytestmark = pytest.mark.gpu

TOL64 = 1e-15
TOL32 = 1e-7
DEV = "cuda:0"


def dev(a, dtype=torch.complex128):
    return torch.from_numpy(np.ascontiguousarray(a)).to(DEV).to(dtype)


def host(t):
    torch.cuda.synchronize()
    return t.cpu().numpy().astype(np.complex128)


# ---------------------------------------------------------------- coarse stencil
@pytest.fixture(scope="module")
def coarse44():
    dims, N = (4, 4, 4, 4), 24
    r = inputs.rng(stream=101)
    A = inputs.random_links(dims, N, r)
    x = inputs.gaussian_field((256, 5, N), r)
    cm = gmg.CoarsenedMatrix(dims, N)
    cm.set_links(A)
    return dims, N, A, x, cm


def test_neighbors_bit_exact(coarse44):
    dims, N, A, x, cm = coarse44
    assert np.array_equal(cm.neighbors(), orc.coarse_neighbors(dims))


def test_links_round_trip(coarse44):
    dims, N, A, x, cm = coarse44
    assert np.array_equal(cm.get_links(), A)


@pytest.mark.parametrize("nrhs", [1, 2, 5])
@pytest.mark.parametrize("op", ["M", "Mdag", "Mdiag"])
def test_coarse_ops_f64(coarse44, nrhs, op):
    dims, N, A, x, cm = coarse44
    xs = x[:, :nrhs]
    code = {"M": orc.OP_M, "Mdag": orc.OP_MDAG, "Mdiag": orc.OP_MDIAG}[op]
    ref = orc.coarse_apply(dims, A, xs, code)
    inp = dev(xs)
    out = torch.zeros_like(inp)
    getattr(cm, op)(inp, out)
    assert orc.rel_dev_sq(ref, host(out)) < TOL64


def test_coarse_mdir_and_mdirall_f64(coarse44):
    dims, N, A, x, cm = coarse44
    inp = dev(x[:, :2])
    outs = [torch.zeros_like(inp) for _ in range(8)]
    cm.MdirAll(inp, outs)
    for p in range(8):
        ref = orc.coarse_apply(dims, A, x[:, :2], orc.OP_MDIR, point=p)
        assert orc.rel_dev_sq(ref, host(outs[p])) < TOL64
        out = torch.zeros_like(inp)
        cm.Mdir(inp, out, p % 4, 1 if p < 4 else -1)
        assert orc.rel_dev_sq(ref, host(out)) < TOL64


def test_coarse_f32(coarse44):
    dims, N, A, x, cm = coarse44
    cm.prepare("f32")
    for code, name in ((orc.OP_M, "M"), (orc.OP_MDAG, "Mdag")):
        ref = orc.coarse_apply(dims, A, x, code)
        inp = dev(x, torch.complex64)
        out = torch.zeros_like(inp)
        getattr(cm, name)(inp, out)
        assert orc.rel_dev_sq(ref, host(out)) < TOL32


def test_coarse_active_rhs_subset(coarse44):
    dims, N, A, x, cm = coarse44
    inp = dev(x)
    out = torch.full_like(inp, 7.0)
    active = [4, 1, 3]
    cm.M(inp, out, active=active)
    ref = orc.coarse_apply(dims, A, x, orc.OP_M)
    got = host(out)
    for r in range(5):
        if r in active:
            assert orc.rel_dev_sq(ref[:, r], got[:, r]) < TOL64
        else:
            assert np.all(got[:, r] == 7.0)


def test_coarse_hermitian_mdag_is_m():
    dims, N = (2, 4, 2, 4), 8
    A = inputs.random_links(dims, N, inputs.rng(stream=102))
    cm = gmg.CoarsenedMatrix(dims, N, hermitian=1)
    cm.set_links(A)
    x = dev(inputs.gaussian_field((64, 3, N), inputs.rng(stream=103)))
    a, b = torch.zeros_like(x), torch.zeros_like(x)
    cm.M(x, a)
    cm.Mdag(x, b)
    assert torch.equal(a, b)


@pytest.mark.parametrize("dims,N", [((8, 8, 8, 8), 32), ((4, 4, 4, 4), 40)])
def test_coarse_mrhs_config_sizes(dims, N):
    # C2-shaped (8^4, N=32) and C4-shaped (N=40) applies with 8 RHS against the oracle
    r = inputs.rng(stream=104)
    A = inputs.random_links(dims, N, r)
    x = inputs.gaussian_field((int(np.prod(dims)), 8, N), r)
    cm = gmg.CoarsenedMatrix(dims, N)
    cm.set_links(A)
    ref = orc.coarse_apply(dims, A, x, orc.OP_M)
    out = torch.zeros(x.shape, dtype=torch.complex128, device=DEV)
    cm.M(dev(x), out)
    assert orc.rel_dev_sq(ref, host(out)) < TOL64


@pytest.mark.parametrize("prec", ["f64", "f32"])
@pytest.mark.parametrize("N,R", [(24, 4), (32, 12), (40, 8), (16, 32)])
def test_coarse_pipelined_simt_ops(prec, N, R):
    # the pipelined CUDA-core stencil (RHS counts the register tiles divide):
    # M, Mdag (dagger and G5C loop forms), Mdiag, one Mdir point, and an active
    # subset whose size the tiles divide, against the oracle
    dims = (4, 4, 4, 2)
    r = inputs.rng(stream=140 + N + R)
    A = inputs.random_links(dims, N, r)
    x = inputs.gaussian_field((int(np.prod(dims)), R + 2, N), r)
    cm = gmg.CoarsenedMatrix(dims, N)
    cm.set_links(A)
    dt, tol = (torch.complex128, TOL64) if prec == "f64" else (torch.complex64, TOL32)
    if prec == "f32":
        cm.prepare("f32")
    inp = dev(x[:, :R], dt)
    for code, name in ((orc.OP_M, "M"), (orc.OP_MDAG, "Mdag"), (orc.OP_MDIAG, "Mdiag")):
        ref = orc.coarse_apply(dims, A, x[:, :R], code)
        out = torch.zeros_like(inp)
        getattr(cm, name)(inp, out)
        assert orc.rel_dev_sq(ref, host(out)) < tol, (name, orc.rel_dev_sq(ref, host(out)))
    ref = orc.coarse_apply(dims, A, x[:, :R], orc.OP_MDIR, point=5)
    out = torch.zeros_like(inp)
    cm.Mdir(inp, out, 1, -1)
    assert orc.rel_dev_sq(ref, host(out)) < tol
    # active subset of R of the R + 2 columns
    full = dev(x, dt)
    outf = torch.full_like(full, 7.0)
    active = list(range(R + 1, 1, -1))[:R]  # R columns in reverse order, skipping columns 0 and 1
    cm.Mdag(full, outf, active=active)
    reff = orc.coarse_apply(dims, A, x, orc.OP_MDAG)
    got = host(outf)
    for c in range(R + 2):
        if c in active:
            assert orc.rel_dev_sq(reff[:, c], got[:, c]) < tol
        else:
            assert np.all(got[:, c] == 7.0)


def test_construct_remaining_links_matches_oracle():
    dims, N = (4, 2, 4, 2), 8
    A = inputs.gaussian_field((9, 64, N, N), inputs.rng(stream=105))
    for herm in (0, 1):
        cm = gmg.CoarsenedMatrix(dims, N, hermitian=herm)
        cm.set_links(A)
        cm.construct_remaining_links()
        ref = orc.construct_remaining_links(dims, A, herm)
        assert np.array_equal(cm.get_links(), ref)


def test_layout_links_matches_oracle():
    a = inputs.gaussian_field((6, 8, 8), inputs.rng(stream=106))
    t = dev(a)
    spin = gmg.layout_links(t, 2)
    assert np.array_equal(host(spin), orc.layout_link_flat_to_spin(a, 2))
    assert torch.equal(gmg.layout_links(spin, 2, inverse=True), t)


def test_layout_vectors_matches_oracle():
    v = inputs.gaussian_field((16, 3, 24), inputs.rng(stream=107))
    t = dev(v)
    spin = gmg.layout_vectors(t, 2)
    assert np.array_equal(host(spin).reshape(-1, 24), orc.layout_vec_flat_to_spin(v.reshape(-1, 24), 2))
    assert torch.equal(gmg.layout_vectors(spin, 2, inverse=True), t)


# ------------------------------------------------------------------ aggregation
@pytest.fixture(scope="module")
def agg8():
    fd, cd = (8, 8, 4, 4), (2, 2, 2, 2)
    h = inputs.gaussian_field((4, int(np.prod(fd)), 12), inputs.rng(stream=111))
    B0 = orc.chiral_double(h, 0.5)
    ag = gmg.Aggregation(fd, cd, 12, 8)
    ag.set_basis(B0)
    return fd, cd, B0, ag


def test_basis_round_trip(agg8):
    fd, cd, B0, ag = agg8
    assert np.array_equal(ag.get_basis(), B0)


def test_orthonormalise_matches_mgs(agg8):
    fd, cd, B0, ag = agg8
    ag2 = gmg.Aggregation(fd, cd, 12, 8)
    ag2.set_basis(B0)
    ag2.Orthogonalise(passes=1)
    got = ag2.get_basis()
    ref = orc.block_orthonormalise(fd, cd, B0, passes=1)
    assert orc.rel_dev_sq(ref, got) < 1e-24
    assert ag2.CheckOrthogonal() < 1e-13
    ag2.Orthogonalise(passes=2)
    assert ag2.CheckOrthogonal() < 1e-14


def test_orthonormalise_nearly_dependent_block_vectors(agg8):
    # smoothed test vectors can be nearly dependent inside a block: v_j = v_0 + 1e-7 noise
    # (condition number ~1e8, so a plain Cholesky-QR Gram matrix is numerically singular);
    # the result must still be orthonormal and span the same space as MGS's basis
    fd, cd, B0, ag = agg8
    r = inputs.rng(stream=119)
    B = np.repeat(B0[:1], 8, axis=0) + 1e-7 * inputs.gaussian_field(B0.shape, r)
    ag2 = gmg.Aggregation(fd, cd, 12, 8)
    ag2.set_basis(B)
    ag2.Orthogonalise(passes=2)
    assert ag2.CheckOrthogonal() < 1e-12
    got = ag2.get_basis()
    ref = orc.block_orthonormalise(fd, cd, B, passes=2)
    # same span block by block: projecting the MGS vectors onto the GPU basis keeps them
    back = orc.block_promote(fd, cd, got, orc.block_project(fd, cd, got, np.moveaxis(ref, 0, 1)))
    assert orc.rel_dev_sq(np.moveaxis(ref, 0, 1), back) < 1e-10


@pytest.mark.parametrize("fd,cd,dof,N", [
    ((8, 8, 8, 8), (2, 2, 2, 2), 12, 24),   # 4^4 blocks (K = 3072), nbasis 24
    ((8, 8, 8, 8), (2, 2, 2, 2), 12, 32),   # nbasis 32
    ((8, 8, 8, 8), (2, 2, 2, 2), 12, 40),   # nbasis 40 (the two-kernel path's largest)
    ((4, 4, 4, 4), (2, 2, 2, 2), 40, 40),   # coarse level: 2^4 blocks of dof 40 (K = 640)
    ((4, 4, 4, 4), (1, 2, 2, 2), 24, 48),   # nbasis 48: the one-CTA-per-block path
    ((4, 4, 2, 2), (2, 2, 1, 1), 12, 6),    # small nbasis, partial last chunk (K = 96)
])
def test_orthonormalise_sizes_match_mgs(fd, cd, dof, N):
    # Cholesky QR on the GPU against the oracle's modified Gram-Schmidt
    # (blockLutedOrthonormalise) on chirally doubled Gaussian vectors, one and
    # two passes, and the orthogonality check (CheckOrthogonal)
    h = inputs.gaussian_field((N // 2, int(np.prod(fd)), dof), inputs.rng(stream=190 + N + dof))
    B0 = orc.chiral_double(h, 0.5)
    ag = gmg.Aggregation(fd, cd, dof, N)
    ag.set_basis(B0)
    assert ag.CheckOrthogonal() > 0.5
    ag.Orthogonalise(passes=1)
    ref = orc.block_orthonormalise(fd, cd, B0, passes=1)
    assert orc.rel_dev_sq(ref, ag.get_basis()) < 1e-24
    assert ag.CheckOrthogonal() < 1e-13
    ag.set_basis(B0)
    ag.Orthogonalise(passes=2)
    ref2 = orc.block_orthonormalise(fd, cd, B0, passes=2)
    assert orc.rel_dev_sq(ref2, ag.get_basis()) < 1e-24
    assert ag.CheckOrthogonal() < 1e-14


def test_orthonormalise_shift_only_where_needed():
    # one block of 16 holds nearly dependent vectors, v_j = v_0 + 1e-9 noise
    # (the Gram matrix's condition number ~1e18 is beyond FP64, so plain
    # Cholesky QR breaks down there and the shifted factorisation plus two
    # extra plain passes run for that block alone); the other blocks must come
    # out as the plain pass leaves them
    fd, cd, N = (8, 8, 8, 8), (2, 2, 2, 2), 24
    V = int(np.prod(fd))
    h = inputs.gaussian_field((N // 2, V, 12), inputs.rng(stream=195))
    B0 = orc.chiral_double(h, 0.5)
    lut = gmg.lut_build(fd, cd)[0]
    sites = lut[5]  # block 5
    noise = 1e-9 * inputs.gaussian_field((N, len(sites), 12), inputs.rng(stream=196))
    B0[:, sites] = B0[:1, sites] + noise
    B0[N // 2:, sites, :6] = 0.0  # keep the chiral structure of the doubled basis
    B0[:N // 2, sites, 6:] = 0.0
    ag = gmg.Aggregation(fd, cd, 12, N)
    ag.set_basis(B0)
    ag.Orthogonalise(passes=1)
    assert ag.CheckOrthogonal() < 1e-12
    got = ag.get_basis()
    ref = orc.block_orthonormalise(fd, cd, B0, passes=1)
    other = np.setdiff1d(np.arange(V), sites)
    assert orc.rel_dev_sq(ref[:, other], got[:, other]) < 1e-24
    # block 5: same span as the Gram-Schmidt basis
    sub = got[:, sites]
    proj = np.einsum("ik,jk->ij", sub.reshape(N, -1).conj(), ref[:, sites].reshape(N, -1))
    back = np.einsum("ij,ik->jk", proj, sub.reshape(N, -1))
    assert orc.rel_dev_sq(ref[:, sites].reshape(N, -1), back) < 1e-10


@pytest.mark.parametrize("nrhs", [1, 3, 8])
def test_project_promote_f64(agg8, nrhs):
    fd, cd, B0, ag = agg8
    B = orc.block_orthonormalise(fd, cd, B0, passes=1)
    ag.set_basis(B)
    f = inputs.gaussian_field((int(np.prod(fd)), nrhs, 12), inputs.rng(stream=112))
    c = torch.zeros((16, nrhs, 8), dtype=torch.complex128, device=DEV)
    ag.ProjectToSubspace(dev(f), c)
    assert orc.rel_dev_sq(orc.block_project(fd, cd, B, f), host(c)) < TOL64
    vc = inputs.gaussian_field((16, nrhs, 8), inputs.rng(stream=113))
    fo = torch.zeros((int(np.prod(fd)), nrhs, 12), dtype=torch.complex128, device=DEV)
    ag.PromoteFromSubspace(dev(vc), fo)
    assert orc.rel_dev_sq(orc.block_promote(fd, cd, B, vc), host(fo)) < TOL64


@pytest.mark.parametrize("fd,cd,dof,N,R", [((8, 8, 8, 8), (2, 2, 2, 2), 12, 24, 12),
                                          ((8, 8, 8, 8), (4, 4, 4, 4), 12, 40, 20),
                                          ((4, 4, 4, 4), (2, 2, 2, 2), 16, 16, 4),
                                          ((4, 4, 4, 4), (2, 2, 2, 2), 40, 40, 40),
                                          ((8, 8, 8, 8), (2, 2, 2, 2), 12, 40, 40),
                                          ((8, 8, 8, 8), (4, 4, 4, 4), 12, 10, 7),
                                          ((6, 4, 4, 4), (2, 4, 4, 4), 12, 6, 5)])
def test_project_f64_shapes(fd, cd, dof, N, R):
    # FP64 projections of fine-site (dof 12) and coarse-site (dof 16, 40)
    # aggregations: several K chunks per block, register tiles cut by nbasis
    # and nrhs that are not multiples of the tile, and a block of 3 sites (the
    # pipelined kernel's last chunk of a block shorter than the others)
    Vf = int(np.prod(fd))
    B = inputs.gaussian_field((N, Vf, dof), inputs.rng(stream=180 + N))
    ag = gmg.Aggregation(fd, cd, dof, N)
    ag.set_basis(B)
    f = inputs.gaussian_field((Vf, R, dof), inputs.rng(stream=181 + R))
    c = torch.zeros((int(np.prod(cd)), R, N), dtype=torch.complex128, device=DEV)
    ag.ProjectToSubspace(dev(f), c)
    assert orc.rel_dev_sq(orc.block_project(fd, cd, B, f), host(c)) < TOL64


def test_project_promote_f32(agg8):
    fd, cd, B0, ag = agg8
    B = orc.block_orthonormalise(fd, cd, B0, passes=1)
    ag.set_basis(B)
    f = inputs.gaussian_field((int(np.prod(fd)), 4, 12), inputs.rng(stream=114))
    c = torch.zeros((16, 4, 8), dtype=torch.complex64, device=DEV)
    ag.ProjectToSubspace(dev(f, torch.complex64), c)
    assert orc.rel_dev_sq(orc.block_project(fd, cd, B, f), host(c)) < TOL32
    fo = torch.zeros((int(np.prod(fd)), 4, 12), dtype=torch.complex64, device=DEV)
    ag.PromoteFromSubspace(c, fo)
    assert orc.rel_dev_sq(orc.block_promote(fd, cd, B, host(c)), host(fo)) < TOL32


def test_transfer_identities_gpu(agg8):
    # P R v_i = v_i and R P v_c = v_c (MultigridPreconditioner.h:352-396)
    fd, cd, B0, ag = agg8
    ag.set_basis(B0)
    ag.Orthogonalise(passes=1)
    B = ag.get_basis()
    vi = dev(np.ascontiguousarray(np.transpose(B[:3], (1, 0, 2))))  # 3 basis vectors as RHS
    c = torch.zeros((16, 3, 8), dtype=torch.complex128, device=DEV)
    back = torch.zeros_like(vi)
    ag.ProjectToSubspace(vi, c)
    ag.PromoteFromSubspace(c, back)
    assert orc.rel_dev_sq(host(vi), host(back)) < TOL64
    vc = dev(inputs.gaussian_field((16, 2, 8), inputs.rng(stream=115)))
    f = torch.zeros((int(np.prod(fd)), 2, 12), dtype=torch.complex128, device=DEV)
    rp = torch.zeros_like(vc)
    ag.PromoteFromSubspace(vc, f)
    ag.ProjectToSubspace(f, rp)
    assert orc.rel_dev_sq(host(vc), host(rp)) < TOL64


# ----------------------------------------------------------------- wilson-clover
@pytest.fixture(scope="module")
def wil():
    dims = (4, 4, 4, 8)
    U = inputs.hot_gauge(dims, inputs.rng(stream=121))
    w = gmg.WilsonClover(dims, -0.1, 1.0, antiperiodic=True)
    w.set_gauge(U)
    cl = orc.clover_build(dims, U, 1.0)
    return dims, U, cl, w


def test_clover_matches_oracle(wil):
    dims, U, cl, w = wil
    assert orc.rel_dev_sq(cl, w.clover()) < TOL64


def test_clover_known_answer_uniform_abelian_field():
    # the device-built clover term on a uniform U(1) field (B01 = 2 pi / 8 in the
    # (0,1) plane, B23 = -2 pi / 8 in the (2,3) plane, identity colour) equals
    # the analytic -(c_sw/2) (sin B01 sigma_01 + sin B23 sigma_23) x 1_colour
    dims, csw = (8, 2, 8, 2), 1.3
    V = int(np.prod(dims))
    b01, b23 = 2 * np.pi / 8, -2 * np.pi / 8
    U = np.zeros((V, 4, 3, 3), dtype=np.complex128)
    for s in range(V):
        x0, x2 = s % 8, (s // 16) % 8
        for mu, ph in enumerate((1.0, np.exp(1j * b01 * x0), 1.0, np.exp(1j * b23 * x2))):
            U[s, mu] = ph * np.eye(3)
    g = [orc.gamma(mu) for mu in range(4)]
    sig = lambda a, b: 0.5j * (g[a] @ g[b] - g[b] @ g[a])  # noqa: E731
    full = np.kron(-0.5 * csw * (np.sin(b01) * sig(0, 1) + np.sin(b23) * sig(2, 3)), np.eye(3))
    expect = np.stack([full[:6, :6], full[6:, 6:]])
    w = gmg.WilsonClover(dims, -0.2, csw, antiperiodic=0)
    w.set_gauge(U)
    assert np.abs(w.clover() - expect[None]).max() < 1e-14


@pytest.mark.parametrize("op", ["M", "Mdag", "Mdiag"])
def test_wilson_ops_f64(wil, op):
    dims, U, cl, w = wil
    x = inputs.gaussian_field((512, 3, 12), inputs.rng(stream=122))
    code = {"M": orc.OP_M, "Mdag": orc.OP_MDAG, "Mdiag": orc.OP_MDIAG}[op]
    ref = orc.wilson_clover(dims, U, cl, -0.1, 1, x, code)
    out = torch.zeros((512, 3, 12), dtype=torch.complex128, device=DEV)
    getattr(w, op)(dev(x), out)
    assert orc.rel_dev_sq(ref, host(out)) < TOL64


@pytest.fixture
def forced(wil):
    """Force a Wilson kernel variant for one test, back to autotuning after it."""
    w = wil[3]
    yield w.set_kernel
    w.set_kernel("auto")


VARIANTS = ["site", "tile", "quad", "staged"]


@pytest.mark.parametrize("variant", VARIANTS)
@pytest.mark.parametrize("nrhs", [4, 7, 12, 13, 17, 20, 24, 40])
@pytest.mark.parametrize("op", ["M", "Mdag", "Mdiag"])
def test_wilson_multi_rhs_variants(wil, forced, variant, nrhs, op):
    # tile: 16 sites x min(nrhs, 16) threads; quad: rt = largest divisor of nrhs
    # up to 8 (13 -> 1, 7 -> 7, 20 -> 5); staged: RHS chunks of at most 24
    # (FP32) or 16 (FP64) of equal size (FP64 17 -> 9 + 8, 40 -> 14 + 13 + 13;
    # FP32 40 -> 20 + 20), partial warps in the last chunk
    dims, U, cl, w = wil
    forced(variant)
    x = inputs.gaussian_field((512, nrhs, 12), inputs.rng(stream=124 + nrhs))
    code = {"M": orc.OP_M, "Mdag": orc.OP_MDAG, "Mdiag": orc.OP_MDIAG}[op]
    ref = orc.wilson_clover(dims, U, cl, -0.1, 1, x, code)
    out = torch.zeros((512, nrhs, 12), dtype=torch.complex128, device=DEV)
    getattr(w, op)(dev(x), out)
    assert orc.rel_dev_sq(ref, host(out)) < TOL64
    out32 = torch.zeros((512, nrhs, 12), dtype=torch.complex64, device=DEV)
    getattr(w, op)(dev(x, torch.complex64), out32)
    assert orc.rel_dev_sq(ref, host(out32)) < TOL32


def test_wilson_autotuner_records_a_choice(wil):
    dims, U, cl, w = wil
    x = dev(inputs.gaussian_field((512, 12, 12), inputs.rng(stream=171)), torch.complex64)
    out = torch.zeros_like(x)
    w.M(x, out)
    assert w.tuned_kernel("f32", 12) in ("site", "tile", "quad", "staged")
    ref = orc.wilson_clover(dims, U, cl, -0.1, 1, host(x).astype(np.complex128), orc.OP_M)
    assert orc.rel_dev_sq(ref, host(out)) < TOL32


def test_wilson_mdir_f64_and_f32(wil):
    dims, U, cl, w = wil
    x = inputs.gaussian_field((512, 2, 12), inputs.rng(stream=123))
    for d in range(4):
        for disp in (1, -1):
            ref = orc.wilson_clover(dims, U, cl, -0.1, 1, x, orc.OP_MDIR, d, disp)
            out = torch.zeros((512, 2, 12), dtype=torch.complex128, device=DEV)
            w.Mdir(dev(x), out, d, disp)
            assert orc.rel_dev_sq(ref, host(out)) < TOL64
    ref = orc.wilson_clover(dims, U, cl, -0.1, 1, x, orc.OP_M)
    out = torch.zeros((512, 2, 12), dtype=torch.complex64, device=DEV)
    w.M(dev(x, torch.complex64), out)
    assert orc.rel_dev_sq(ref, host(out)) < TOL32


@pytest.mark.parametrize("variant", VARIANTS)
@pytest.mark.parametrize("dims,nrhs", [((6, 4, 2, 4), 9), ((2, 2, 2, 2), 4), ((10, 2, 2, 2), 16)])
def test_wilson_odd_lattices(dims, nrhs, variant):
    # tiles that start and end inside x rows (x halos), lattices of extent 2
    # (both hops of a direction reach the same site), a partial last RHS chunk
    V = int(np.prod(dims))
    U = inputs.hot_gauge(dims, inputs.rng(stream=161))
    w = gmg.WilsonClover(dims, -0.2, 1.0, antiperiodic=True)
    w.set_gauge(U)
    w.set_kernel(variant)
    cl = orc.clover_build(dims, U, 1.0)
    x = inputs.gaussian_field((V, nrhs, 12), inputs.rng(stream=162))
    for op, code in (("M", orc.OP_M), ("Mdag", orc.OP_MDAG)):
        ref = orc.wilson_clover(dims, U, cl, -0.2, 1, x, code)
        out = torch.zeros((V, nrhs, 12), dtype=torch.complex128, device=DEV)
        getattr(w, op)(dev(x), out)
        assert orc.rel_dev_sq(ref, host(out)) < TOL64, op
        out32 = torch.zeros((V, nrhs, 12), dtype=torch.complex64, device=DEV)
        getattr(w, op)(dev(x, torch.complex64), out32)
        assert orc.rel_dev_sq(ref, host(out32)) < TOL32, op
    assert w.device_error() == (0, 0)


def test_wilson_tile_kernel_several_tiles_per_cta():
    # 644 tiles of 16 sites (the last one partial): more than one resident
    # wave of CTAs holds (at most 4 x 148), so every CTA computes two or more
    # tiles, alternating between its two staging buffers.  M and Mdag in FP64
    # and FP32 at 16 and 24 RHS, and the BF16 smoother form with its products
    dims = (13, 11, 8, 9)
    V = int(np.prod(dims))
    U = inputs.hot_gauge(dims, inputs.rng(stream=231))
    w = gmg.WilsonClover(dims, -0.2, 1.0, antiperiodic=True)
    w.set_gauge(U)
    w.set_kernel("tile")
    cl = orc.clover_build(dims, U, 1.0)
    for nrhs in (16, 24):
        x = inputs.gaussian_field((V, nrhs, 12), inputs.rng(stream=232 + nrhs))
        for op, code in (("M", orc.OP_M), ("Mdag", orc.OP_MDAG)):
            ref = orc.wilson_clover(dims, U, cl, -0.2, 1, x, code)
            out = torch.zeros((V, nrhs, 12), dtype=torch.complex128, device=DEV)
            getattr(w, op)(dev(x), out)
            assert orc.rel_dev_sq(ref, host(out)) < TOL64, (op, nrhs)
            out32 = torch.zeros((V, nrhs, 12), dtype=torch.complex64, device=DEV)
            getattr(w, op)(dev(x, torch.complex64), out32)
            assert orc.rel_dev_sq(ref, host(out32)) < TOL32, (op, nrhs)
    # the BF16 smoother form (within BF16 rounding, as in the 512-site test)
    xb = torch.view_as_real(dev(x, torch.complex64)).to(torch.bfloat16).contiguous()
    xr = torch.view_as_complex(xb.float()).to(torch.complex128)
    ref = orc.wilson_clover(dims, U, cl, -0.2, 1, host(xr), orc.OP_M)
    outb = torch.zeros_like(xb)
    d1, d2 = w.M_mr(xb, outb)
    got = torch.view_as_complex(outb.float()).to(torch.complex128)
    assert orc.rel_dev_sq(ref, host(got)) < 4e-5
    d1_ref = np.einsum("srk,srk->r", ref.conj(), host(xr))
    d2_ref = np.einsum("srk,srk->r", ref.conj(), ref).real
    assert np.abs(d1.cpu().numpy() - d1_ref).max() / np.abs(d2_ref).max() < 1e-5
    assert np.abs(d2.cpu().numpy() - d2_ref).max() / np.abs(d2_ref).max() < 1e-5
    assert w.device_error() == (0, 0)


@pytest.mark.parametrize("variant", VARIANTS)
def test_wilson_multi_rhs_mdir(wil, forced, variant):
    # the single-hop form (CoarsenOperator's Mdir calls, nrhs >= 4) of every variant
    dims, U, cl, w = wil
    forced(variant)
    x = inputs.gaussian_field((512, 6, 12), inputs.rng(stream=141))
    for d in range(4):
        for disp in (1, -1):
            ref = orc.wilson_clover(dims, U, cl, -0.1, 1, x, orc.OP_MDIR, d, disp)
            out = torch.zeros((512, 6, 12), dtype=torch.complex128, device=DEV)
            w.Mdir(dev(x), out, d, disp)
            assert orc.rel_dev_sq(ref, host(out)) < TOL64, (d, disp)
            out32 = torch.zeros((512, 6, 12), dtype=torch.complex64, device=DEV)
            w.Mdir(dev(x, torch.complex64), out32, d, disp)
            assert orc.rel_dev_sq(ref, host(out32)) < TOL32, (d, disp)


@pytest.mark.parametrize("variant", ["tile", "quad", "staged"])
@pytest.mark.parametrize("nrhs", [1, 3, 12, 24, 30])
def test_wilson_apply_mr_products(wil, forced, variant, nrhs):
    # M with the minimal-residual inner products formed in the kernel's epilogue
    # (FP32 30 RHS: two chunks of 15 in the staged kernel)
    dims, U, cl, w = wil
    forced(variant)
    x = inputs.gaussian_field((512, nrhs, 12), inputs.rng(stream=150 + nrhs))
    ref = orc.wilson_clover(dims, U, cl, -0.1, 1, x, orc.OP_M)
    d1_ref = np.einsum("srk,srk->r", ref.conj(), x)
    d2_ref = np.einsum("srk,srk->r", ref.conj(), ref).real
    for dt, tol in ((torch.complex128, TOL64), (torch.complex64, TOL32)):
        out = torch.zeros((512, nrhs, 12), dtype=dt, device=DEV)
        d1, d2 = w.M_mr(dev(x, dt), out)
        assert orc.rel_dev_sq(ref, host(out)) < tol
        assert np.abs(d1.cpu().numpy() - d1_ref).max() / np.abs(d2_ref).max() < np.sqrt(tol)
        assert np.abs(d2.cpu().numpy() - d2_ref).max() / np.abs(d2_ref).max() < np.sqrt(tol)


# ------------------------------------------------------------- chiral doubling
@pytest.mark.parametrize("dof", [12, 24])
@pytest.mark.parametrize("factor", [0.5, 1.0])
def test_chiral_double_matches_oracle(dof, factor):
    # performChiralDoublingG5C (factor 1/2) and the G5R5 form (factor 1) on
    # spin-colour vectors (dof 12) and coarse vectors (dof 24), the setup's
    # multi-RHS input layout [V][nvec][dof], F64 and F32 inputs
    V, nvec = 300, 5
    h = inputs.gaussian_field((nvec, V, dof), inputs.rng(stream=160 + dof))
    ref = orc.chiral_double(h, factor)
    x = np.ascontiguousarray(h.transpose(1, 0, 2))
    got = gmg.chiral_double(dev(x), factor)
    assert np.array_equal(ref, host(got))  # sign selection and one product per element: exact
    x32 = dev(x, torch.complex64)
    got32 = host(gmg.chiral_double(x32, factor))
    ref32 = orc.chiral_double(x32.cpu().numpy().astype(np.complex128).transpose(1, 0, 2), factor)
    assert np.array_equal(ref32, got32)
    # the halves sum back to factor * 2 v (undoChiralDoubling up to the factor)
    assert np.allclose(got32[:nvec] + got32[nvec:], 2 * factor * x32.cpu().numpy().transpose(1, 0, 2), atol=0)


# --------------------------------------------------------------- CoarsenOperator
@pytest.fixture(scope="module")
def coarsen_setup():
    fd, cd = (8, 8, 8, 8), (2, 2, 2, 2)
    U = inputs.hot_gauge(fd, inputs.rng(stream=131))
    h = inputs.gaussian_field((4, int(np.prod(fd)), 12), inputs.rng(stream=132))
    B = orc.block_orthonormalise(fd, cd, orc.chiral_double(h, 0.5), passes=1)
    return fd, cd, U, B


@pytest.mark.parametrize("apbc", [0, 1])
def test_coarsen_wilson_matches_oracle(coarsen_setup, apbc):
    fd, cd, U, B = coarsen_setup
    mass = -0.1
    w = gmg.WilsonClover(fd, mass, 1.0, antiperiodic=apbc)
    w.set_gauge(U)
    ag = gmg.Aggregation(fd, cd, 12, 8)
    ag.set_basis(B)
    cm = gmg.CoarsenedMatrix(cd, 8)
    cm.CoarsenOperator(ag, w)
    cl = orc.clover_build(fd, U, 1.0)
    ref = orc.coarsen_wilson(fd, cd, B, U, cl, mass, apbc, 0, variant=0)  # Upstream semantics
    got = cm.get_links()
    for p in range(9):
        assert orc.rel_dev_sq(ref[p], got[p]) < TOL64, p


def test_coarsen_wilson_anisotropic_blocks_and_reuse():
    # blocks of a different extent per direction (each backward face its own
    # site list), and a second call on the same aggregation with a new basis
    # (the workspace kept from the first call) against the oracle both times
    fd, cd = (8, 4, 8, 8), (2, 2, 4, 2)
    U = inputs.hot_gauge(fd, inputs.rng(stream=135))
    w = gmg.WilsonClover(fd, -0.2, 1.0, antiperiodic=1)
    w.set_gauge(U)
    cl = orc.clover_build(fd, U, 1.0)
    ag = gmg.Aggregation(fd, cd, 12, 6)
    for stream in (136, 137):
        h = inputs.gaussian_field((3, int(np.prod(fd)), 12), inputs.rng(stream=stream))
        B = orc.block_orthonormalise(fd, cd, orc.chiral_double(h, 0.5), passes=1)
        ag.set_basis(B)
        cm = gmg.CoarsenedMatrix(cd, 6)
        cm.CoarsenOperator(ag, w)
        ref = orc.coarsen_wilson(fd, cd, B, U, cl, -0.2, 1, 0, variant=0)
        got = cm.get_links()
        for p in range(9):
            assert orc.rel_dev_sq(ref[p], got[p]) < TOL64, (stream, p)


def test_coarsen_coarse_matches_oracle(coarsen_setup):
    fd, cd, U, B = coarsen_setup
    c1 = (4, 4, 4, 4)
    h = inputs.gaussian_field((3, int(np.prod(fd)), 12), inputs.rng(stream=133))
    B1 = orc.block_orthonormalise(fd, c1, orc.chiral_double(h, 0.5), passes=1)
    cl = orc.clover_build(fd, U, 1.0)
    A1 = orc.coarsen_wilson(fd, c1, B1, U, cl, -0.1, 0, 0, variant=1)
    h2 = inputs.gaussian_field((2, 256, 6), inputs.rng(stream=134))
    B2 = orc.block_orthonormalise(c1, (2, 2, 2, 2), orc.chiral_double(h2, 0.5), passes=1)
    fine = gmg.CoarsenedMatrix(c1, 6)
    fine.set_links(A1)
    ag = gmg.Aggregation(c1, (2, 2, 2, 2), 6, 4)
    ag.set_basis(B2)
    cm = gmg.CoarsenedMatrix((2, 2, 2, 2), 4)
    cm.CoarsenOperator(ag, fine)
    ref = orc.coarsen_coarse(c1, (2, 2, 2, 2), B2, A1, variant=0)
    got = cm.get_links()
    for p in range(9):
        assert orc.rel_dev_sq(ref[p], got[p]) < TOL64, p


@pytest.mark.parametrize("nrhs", [1, 5, 24])
@pytest.mark.parametrize("dag", [False, True])
def test_wilson_f32_input_matches_converted_f64_apply(wil, forced, nrhs, dag):
    # the FP64 operator on an FP32 field, promoted on load, is bit for bit the
    # FP64 tile kernel on the field converted to FP64 (same kernel, same order
    # of operations), and within the FP64 bound of the oracle on that field
    dims, U, cl, w = wil
    forced("tile")
    x32 = dev(inputs.gaussian_field((512, nrhs, 12), inputs.rng(stream=190 + nrhs)), torch.complex64)
    x64 = x32.to(torch.complex128)
    want = torch.zeros_like(x64)
    (w.Mdag if dag else w.M)(x64, want)
    got = torch.zeros_like(x64)
    w.M_f32_in(x32, got, dag=dag)
    torch.cuda.synchronize()
    assert torch.equal(want, got)
    ref = orc.wilson_clover(dims, U, cl, -0.1, 1, host(x64), orc.OP_MDAG if dag else orc.OP_M)
    assert orc.rel_dev_sq(ref, host(got)) < TOL64


@pytest.mark.parametrize("nrhs", [4, 24])
def test_wilson_mr_products_bf16_fields(wil, nrhs):
    # the fine smoother's BF16 form: BF16 input records widened to FP32, M in
    # FP32, the result rounded to BF16, the MR products from the FP32 result.
    # Against the FP64 oracle on the BF16-rounded input: the output within
    # BF16 rounding (2^-8 relative per component, squared deviation < 4e-5),
    # the products to FP32 accuracy of the unrounded result
    dims, U, cl, w = wil
    x = inputs.gaussian_field((512, nrhs, 12), inputs.rng(stream=200 + nrhs))
    xb = torch.view_as_real(dev(x, torch.complex64)).to(torch.bfloat16).contiguous()
    xr = torch.view_as_complex(xb.float()).to(torch.complex128)
    ref = orc.wilson_clover(dims, U, cl, -0.1, 1, host(xr), orc.OP_M)
    out = torch.zeros_like(xb)
    d1, d2 = w.M_mr(xb, out)
    got = torch.view_as_complex(out.float()).to(torch.complex128)
    assert orc.rel_dev_sq(ref, host(got)) < 4e-5
    d1_ref = np.einsum("srk,srk->r", ref.conj(), host(xr))
    d2_ref = np.einsum("srk,srk->r", ref.conj(), ref).real
    assert np.abs(d1.cpu().numpy() - d1_ref).max() / np.abs(d2_ref).max() < 1e-5
    assert np.abs(d2.cpu().numpy() - d2_ref).max() / np.abs(d2_ref).max() < 1e-5

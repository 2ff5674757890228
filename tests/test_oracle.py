"""Pins the CPU oracle against the reference's own known-answer and identity checks.

The reference ships no golden vectors (its inputs come from Grid's RNG), so the
oracle is pinned by every check its test/benchmark programs assert, restated
at small sizes:

  geometry round trip ........................ src/Test_geom.cc:44-72
  LUT forward / reverse consistency .......... src/Test_coarsening_lookuptable.cc:37-87
  Mdag = G5C M G5C, Mdir point map ........... include/CoarsenedMatrixUpstream.h:609-742
  4-d looped == 5-d multi-RHS (exact) ........ src/Benchmark_mrhs_coarsening.cc:185-281
  M = Mdiag + sum Mdir (fine op) ............. include/MultigridPreconditioner.h:317-350
  chiral doubling halves sum back ............ src/Test_g5r5.cc:83-146
  CheckOrthogonal, P R v = v, R P v_c = v_c .. MultigridPreconditioner.h:352-396
  Upstream links == Dirsave links (1e-15) .... src/Benchmark_create_coarse_operator.cc:278-352
  coarse-of-coarse Upstream == Dirsave ....... src/Benchmark_create_coarse_coarse_operator.cc:217-381
  R D P v_c = D_c v_c, Im<v,Dc^+ Dc v> = 0 ... MultigridPreconditioner.h:398-443
"""
import numpy as np
import pytest

import oracle as orc
import inputs

TOL = 1e-15  # the reference's FP64 relative squared deviation tolerance


def lex(c, dims):
    return c[0] + dims[0] * (c[1] + dims[1] * (c[2] + dims[2] * c[3]))


def test_geometry_round_trip():
    for ndim in (4, 5):
        for faster in (False, True):
            dirs, disps = orc.geometry(ndim, faster)
            for p in range(9):
                assert orc.point_from_dir_disp(ndim, faster, dirs[p], disps[p]) == p
    dirs, disps = orc.geometry(4, True)
    assert dirs == [0, 1, 2, 3, 0, 1, 2, 3, 0]
    assert disps == [1, 1, 1, 1, -1, -1, -1, -1, 0]


def test_mdir_point_map():
    # CoarsenedMatrixUpstream.h:724-732: point = (1-disp)/2*4 + dir, (0,0) -> 8
    for d in range(4):
        for disp in (1, -1):
            assert orc.point_from_dir_disp(4, True, d, disp) == (1 - disp) // 2 * 4 + d
    assert orc.point_from_dir_disp(4, True, 0, 0) == 8


def test_neighbors_lexicographic():
    dims = (4, 3, 2, 5)
    nbr = orc.coarse_neighbors(dims)
    V = int(np.prod(dims))
    for s in range(V):
        c = [s % 4, (s // 4) % 3, (s // 12) % 2, s // 24]
        for p in range(9):
            cc = list(c)
            if p < 8:
                d = p % 4
                cc[d] = (cc[d] + (1 if p < 4 else -1)) % dims[d]
            assert nbr[p, s] == lex(cc, dims)
    assert np.array_equal(nbr, inputs.shift_index(dims))


@pytest.mark.parametrize("fdims,cdims", [((4, 4, 4, 4), (2, 2, 2, 2)), ((8, 4, 4, 8), (2, 2, 1, 2))])
def test_lut_consistency(fdims, cdims):
    l, sizes, rev = orc.lut(fdims, cdims)
    b = [f // c for f, c in zip(fdims, cdims)]
    bv = int(np.prod(b))
    Vc = int(np.prod(cdims))
    seen = np.zeros(int(np.prod(fdims)), dtype=int)
    for sc in range(Vc):
        assert sizes[sc] == bv
        cc = [sc % cdims[0], (sc // cdims[0]) % cdims[1], (sc // (cdims[0] * cdims[1])) % cdims[2],
              sc // (cdims[0] * cdims[1] * cdims[2])]
        for sb in range(bv):
            cb = [sb % b[0], (sb // b[0]) % b[1], (sb // (b[0] * b[1])) % b[2], sb // (b[0] * b[1] * b[2])]
            sf = lex([cc[d] * b[d] + cb[d] for d in range(4)], fdims)
            assert l[sc, sb] == sf  # lexicographic in-block order
            assert rev[sf] == sc
            seen[sf] += 1
    assert np.all(seen == 1)


def test_masked_lut_faces():
    fdims, cdims = (8, 8, 8, 8), (2, 2, 2, 2)
    for p in range(8):
        m = orc.outer_mask(fdims, cdims, p)
        l, sizes, rev = orc.lut(fdims, cdims, m)
        assert np.all(sizes == 64)  # one face of a 4^4 block
        for sc in range(16):
            for j in range(64):
                assert m[l[sc, j]] == 1 and rev[l[sc, j]] == sc
    assert np.all(orc.outer_mask(fdims, cdims, 8) == 0)
    e = orc.parity_mask(fdims, cdims, 0)
    o = orc.parity_mask(fdims, cdims, 1)
    assert np.all(e + o == 1) and e.sum() == o.sum()


def _coarse_setup(dims=(4, 4, 4, 4), N=8, R=3, seed=0):
    r = inputs.rng(stream=seed)
    A = inputs.random_links(dims, N, r)
    x = inputs.gaussian_field((int(np.prod(dims)), R, N), r)
    return A, x


def test_coarse_mdag_is_g5c_m_g5c_and_adjoint():
    dims = (4, 4, 4, 4)
    A, x = _coarse_setup(dims)
    y = orc.coarse_apply(dims, A, x, orc.OP_MDAG)
    g = np.ones(8); g[4:] = -1
    y2 = orc.coarse_apply(dims, A, x * g, orc.OP_M) * g
    assert orc.rel_dev_sq(y2, y) < TOL
    # with the gamma5-hermitian link structure Mdag is the true adjoint
    r = inputs.rng(stream=7)
    z = inputs.gaussian_field(x.shape, r)
    lhs = np.vdot(z, orc.coarse_apply(dims, A, x, orc.OP_M))
    rhs = np.vdot(orc.coarse_apply(dims, A, z, orc.OP_MDAG), x)
    assert abs(lhs - rhs) < 1e-12 * abs(lhs)


def test_coarse_m_is_sum_of_points_and_mrhs_equals_looped():
    dims = (4, 4, 4, 4)
    A, x = _coarse_setup(dims)
    y = orc.coarse_apply(dims, A, x, orc.OP_M)
    acc = orc.coarse_apply(dims, A, x, orc.OP_MDIAG)
    for p in range(8):
        acc = acc + orc.coarse_apply(dims, A, x, orc.OP_MDIR, point=p)
    assert orc.rel_dev_sq(y, acc) < TOL
    for r in range(x.shape[1]):  # 4-d looped == 5-d MRHS, exactly
        yr = orc.coarse_apply(dims, A, x[:, r:r + 1, :], orc.OP_M)
        assert np.array_equal(yr[:, 0], y[:, r])


def test_coarse_matches_dense_numpy():
    dims = (2, 2, 4, 2)
    A, x = _coarse_setup(dims, N=4, R=2)
    nbr = inputs.shift_index(dims)
    ref = np.einsum("psab,psrb->sra", A, x[nbr])
    assert orc.rel_dev_sq(ref, orc.coarse_apply(dims, A, x)) < TOL


def test_gamma_algebra():
    G = [orc.gamma(m) for m in range(4)]
    for a in range(4):
        assert np.allclose(G[a], G[a].conj().T)
        for b in range(4):
            assert np.allclose(G[a] @ G[b] + G[b] @ G[a], 2 * np.eye(4) * (a == b))
    assert np.allclose(G[0] @ G[1] @ G[2] @ G[3], np.diag([1, 1, -1, -1]))
    assert np.allclose(orc.gamma(4), np.diag([1, 1, -1, -1]))


@pytest.fixture(scope="module")
def wilson4():
    dims = (4, 4, 4, 4)
    r = inputs.rng(stream=11)
    U = inputs.hot_gauge(dims, r)
    cl = orc.clover_build(dims, U, 1.0)
    return dims, U, cl


def test_gauge_is_su3(wilson4):
    dims, U, _ = wilson4
    u = U.reshape(-1, 3, 3)
    assert np.allclose(u @ np.conj(np.swapaxes(u, -1, -2)), np.eye(3), atol=1e-13)
    assert np.allclose(np.linalg.det(u), 1.0, atol=1e-13)
    s = inputs.smooth_gauge(dims, inputs.rng(stream=3), 0.3).reshape(-1, 3, 3)
    assert np.allclose(s @ np.conj(np.swapaxes(s, -1, -2)), np.eye(3), atol=1e-13)
    assert np.allclose(np.linalg.det(s), 1.0, atol=1e-12)


def test_clover_hermitian(wilson4):
    dims, U, cl = wilson4
    assert np.allclose(cl, np.conj(np.swapaxes(cl, -1, -2)), atol=1e-14)
    assert np.abs(cl).max() > 0.01


@pytest.mark.parametrize("apbc", [0, 1])
def test_wilson_m_is_mdiag_plus_mdir(wilson4, apbc):
    dims, U, cl = wilson4
    x = inputs.gaussian_field((256, 2, 12), inputs.rng(stream=5))
    m = -0.1
    y = orc.wilson_clover(dims, U, cl, m, apbc, x, orc.OP_M)
    acc = orc.wilson_clover(dims, U, cl, m, apbc, x, orc.OP_MDIAG)
    for d in range(4):
        for disp in (1, -1):
            acc += orc.wilson_clover(dims, U, cl, m, apbc, x, orc.OP_MDIR, d, disp)
    dev = np.sqrt(orc.rel_dev_sq(y, acc))
    assert dev < 1e-13
    # gamma5-hermiticity: <z, M x> = <Mdag z, x>
    z = inputs.gaussian_field(x.shape, inputs.rng(stream=6))
    lhs = np.vdot(z, y)
    rhs = np.vdot(orc.wilson_clover(dims, U, cl, m, apbc, z, orc.OP_MDAG), x)
    assert abs(lhs - rhs) < 1e-12 * abs(lhs)


def test_wilson_free_field_plane_wave():
    # unit gauge, no clover: M on a constant spinor = (4+m) - 1/2 * sum_mu 2 = m
    dims = (4, 4, 4, 4)
    U = np.broadcast_to(np.eye(3, dtype=np.complex128), (256, 4, 3, 3)).copy()
    x = np.zeros((256, 1, 12), dtype=np.complex128)
    x[:, 0, :] = inputs.gaussian_field((12,), inputs.rng(stream=1))
    y = orc.wilson_clover(dims, U, None, 0.25, 0, x)
    assert np.allclose(y, 0.25 * x, atol=1e-13)


def test_chiral_doubling_halves_sum_back():
    V = 64
    h = inputs.gaussian_field((3, V, 12), inputs.rng(stream=2))
    d = orc.chiral_double(h, 0.5)
    assert np.allclose(d[:3] + d[3:], h, atol=1e-15)
    assert np.allclose(d[:3][..., 6:], 0) and np.allclose(d[3:][..., :6], 0)
    assert np.allclose(orc.undo_chiral_double(d), h)
    d1 = orc.chiral_double(h, 1.0)  # G5R5 in 4-d == gamma5 doubling (factor 1)
    assert np.allclose(d1, 2 * d)


def _basis(fdims, cdims, nb, stream, dof=12):
    V = int(np.prod(fdims))
    h = inputs.gaussian_field((nb, V, dof), inputs.rng(stream=stream))
    return orc.block_orthonormalise(fdims, cdims, orc.chiral_double(h, 0.5), passes=1)


def test_orthonormalise_and_transfer_identities():
    fdims, cdims = (8, 8, 4, 4), (2, 2, 2, 2)
    B = _basis(fdims, cdims, 4, 21)
    N = B.shape[0]
    Vc = 16
    # CheckOrthogonal: R v_i = e_i on every block
    for i in range(N):
        c = orc.block_project(fdims, cdims, B, B[i][:, None, :])
        e = np.zeros((Vc, 1, N), dtype=np.complex128)
        e[:, 0, i] = 1.0
        assert np.sum(np.abs(c - e) ** 2) < 1e-24
        # P R v_i = v_i
        back = orc.block_promote(fdims, cdims, B, c)
        assert orc.rel_dev_sq(B[i][:, None, :], back) < TOL
    # R P v_c = v_c
    vc = inputs.gaussian_field((Vc, 3, N), inputs.rng(stream=22))
    rp = orc.block_project(fdims, cdims, B, orc.block_promote(fdims, cdims, B, vc))
    assert orc.rel_dev_sq(vc, rp) < TOL


def test_project_matches_numpy():
    fdims, cdims = (4, 4, 4, 4), (2, 2, 2, 2)
    B = _basis(fdims, cdims, 2, 31)
    f = inputs.gaussian_field((256, 2, 12), inputs.rng(stream=32))
    _, _, rev = orc.lut(fdims, cdims)
    ref = np.zeros((16, 2, 4), dtype=np.complex128)
    for s in range(256):
        ref[rev[s]] += np.einsum("ia,ra->ri", np.conj(B[:, s, :]), f[s])
    assert orc.rel_dev_sq(ref, orc.block_project(fdims, cdims, B, f)) < TOL


@pytest.fixture(scope="module")
def coarse_from_wilson():
    fdims, cdims = (8, 8, 8, 8), (2, 2, 2, 2)
    r = inputs.rng(stream=41)
    U = inputs.hot_gauge(fdims, r)
    cl = orc.clover_build(fdims, U, 1.0)
    B = _basis(fdims, cdims, 4, 42)
    return fdims, cdims, U, cl, B


@pytest.mark.parametrize("apbc", [0, 1])
def test_coarsen_upstream_equals_dirsave(coarse_from_wilson, apbc):
    fdims, cdims, U, cl, B = coarse_from_wilson
    up = orc.coarsen_wilson(fdims, cdims, B, U, cl, -0.1, apbc, 0, variant=0)
    ds = orc.coarsen_wilson(fdims, cdims, B, U, cl, -0.1, apbc, 0, variant=1)
    for p in range(9):
        assert orc.rel_dev_sq(up[p], ds[p]) < TOL, p


def test_coarsen_hermitian_variants_agree(coarse_from_wilson):
    fdims, cdims, U, cl, B = coarse_from_wilson
    up = orc.coarsen_wilson(fdims, cdims, B, U, cl, -0.1, 0, 1, variant=0)
    ds = orc.coarsen_wilson(fdims, cdims, B, U, cl, -0.1, 0, 1, variant=1)
    for p in range(9):
        assert orc.rel_dev_sq(up[p], ds[p]) < TOL


def test_galerkin_identity_and_adjoint(coarse_from_wilson):
    fdims, cdims, U, cl, B = coarse_from_wilson
    m = -0.1
    A = orc.coarsen_wilson(fdims, cdims, B, U, cl, m, 1, 0, variant=1)
    vc = inputs.gaussian_field((16, 2, B.shape[0]), inputs.rng(stream=43))
    pv = orc.block_promote(fdims, cdims, B, vc)
    rdp = orc.block_project(fdims, cdims, B, orc.wilson_clover(fdims, U, cl, m, 1, pv))
    dc = orc.coarse_apply(cdims, A, vc)
    assert np.sqrt(orc.rel_dev_sq(rdp, dc)) < 1e-13
    dcv = orc.coarse_apply(cdims, A, vc[:, :1])
    dot = np.vdot(vc[:, :1], orc.coarse_apply(cdims, A, dcv, orc.OP_MDAG))
    assert abs(dot.imag) / abs(dot.real) < 1e-13


def test_coarse_of_coarse_upstream_equals_dirsave(coarse_from_wilson):
    fdims, cdims, U, cl, B = coarse_from_wilson
    # level-1 operator on the 2^4 coarse lattice, then 2^4 -> 1^4 blocks would be
    # degenerate; use a 4^4 coarse lattice from 8^4 with 2^4 blocks instead.
    c1 = (4, 4, 4, 4)
    B1 = _basis(fdims, c1, 3, 51)
    A1 = orc.coarsen_wilson(fdims, c1, B1, U, cl, -0.1, 0, 0, variant=1)
    N1 = B1.shape[0]
    h = inputs.gaussian_field((2, 256, N1), inputs.rng(stream=52))
    B2 = orc.block_orthonormalise(c1, (2, 2, 2, 2), orc.chiral_double(h, 0.5), passes=1)
    up = orc.coarsen_coarse(c1, (2, 2, 2, 2), B2, A1, variant=0)
    ds = orc.coarsen_coarse(c1, (2, 2, 2, 2), B2, A1, variant=1)
    for p in range(9):
        assert orc.rel_dev_sq(up[p], ds[p]) < TOL


def test_layout_maps():
    N, ncs = 8, 2
    x = inputs.gaussian_field((5, N), inputs.rng(stream=61))
    assert np.array_equal(orc.layout_vec_flat_to_spin(x, ncs), x)  # same memory order
    a = inputs.gaussian_field((5, N, N), inputs.rng(stream=62))
    y = orc.layout_link_flat_to_spin(a, ncs).reshape(5, ncs, ncs, N // ncs, N // ncs)
    for n1 in range(N):
        for n2 in range(N):
            assert y[:, n1 // 4, n2 // 4, n1 % 4, n2 % 4].tolist() == a[:, n1, n2].tolist()


# DeGrand-Rossi chiral basis (the basis Grid uses), written out from its definition
_I = 1j
_GAMMA_DR = [
    np.array([[0, 0, 0, _I], [0, 0, _I, 0], [0, -_I, 0, 0], [-_I, 0, 0, 0]]),
    np.array([[0, 0, 0, -1], [0, 0, 1, 0], [0, 1, 0, 0], [-1, 0, 0, 0]], dtype=complex),
    np.array([[0, 0, _I, 0], [0, 0, 0, -_I], [-_I, 0, 0, 0], [0, _I, 0, 0]]),
    np.array([[0, 0, 1, 0], [0, 0, 0, 1], [1, 0, 0, 0], [0, 1, 0, 0]], dtype=complex),
]


def _abelian_gauge(dims, n01, n23):
    """U(1) x identity-colour links with a uniform field strength: U_1(x) = exp(i B01 x_0),
    U_3(x) = exp(i B23 x_2), U_0 = U_2 = 1, with B01 = 2 pi n01 / L_0 and B23 = 2 pi n23 / L_2
    (whole flux quanta, so the field is uniform across the periodic boundary too).
    Every plaquette in the (0,1) plane is exp(i B01), in the (2,3) plane exp(i B23),
    in the other four planes 1."""
    V = int(np.prod(dims))
    U = np.zeros((V, 4, 3, 3), dtype=np.complex128)
    b01, b23 = 2 * np.pi * n01 / dims[0], 2 * np.pi * n23 / dims[2]
    for s in range(V):
        x0 = s % dims[0]
        x2 = (s // (dims[0] * dims[1])) % dims[2]
        ph = [1.0, np.exp(1j * b01 * x0), 1.0, np.exp(1j * b23 * x2)]
        for mu in range(4):
            U[s, mu] = ph[mu] * np.eye(3)
    return U, b01, b23


@pytest.mark.parametrize("n01,n23", [(1, 0), (1, 1), (1, -1), (2, 1)])
def test_clover_known_answer_uniform_abelian_field(n01, n23):
    # Clover term on an analytic background: the clover-leaf field strength of a
    # uniform U(1) field is F_{mu nu} = (Q - Q^dag)/(8i) = sin(B_{mu nu}) exactly
    # (four equal leaves exp(i B)), so Cl = -(c_sw/2) sum_{mu<nu} sigma_{mu nu} F_{mu nu}
    # with sigma_{mu nu} = (i/2)[gamma_mu, gamma_nu] is
    #   Cl = -(c_sw/2) (sin B01 sigma_01 + sin B23 sigma_23) (x) 1_colour
    # at every site: this pins the normalisation (1/8 of the leaf sum, 1/2 of
    # c_sw) and the sign.  In the chiral basis sigma_01 = diag(1,-1,1,-1) and
    # sigma_23 = diag(-1,1,1,-1), so a self-dual field (B01 = B23) leaves the
    # gamma5 = +1 block untouched and an anti-self-dual one the gamma5 = -1 block.
    dims, csw, m = (8, 2, 8, 2), 1.3, -0.2
    for mu in range(4):
        assert np.array_equal(orc.gamma(mu), _GAMMA_DR[mu])
    U, b01, b23 = _abelian_gauge(dims, n01, n23)
    cl = orc.clover_build(dims, U, csw)
    sig01 = 0.5j * (_GAMMA_DR[0] @ _GAMMA_DR[1] - _GAMMA_DR[1] @ _GAMMA_DR[0])
    sig23 = 0.5j * (_GAMMA_DR[2] @ _GAMMA_DR[3] - _GAMMA_DR[3] @ _GAMMA_DR[2])
    spin = -0.5 * csw * (np.sin(b01) * sig01 + np.sin(b23) * sig23)
    full = np.kron(spin, np.eye(3))  # index 3 * spin + colour
    expect = np.stack([full[:6, :6], full[6:, 6:]])
    assert np.abs(full[:6, 6:]).max() == 0 and np.abs(full[6:, :6]).max() == 0
    assert np.abs(cl - expect[None]).max() < 1e-14
    if n01 == n23:
        assert np.abs(cl[:, 0]).max() < 1e-14 and np.abs(cl[:, 1]).max() > 0.1
    if n01 == -n23:
        assert np.abs(cl[:, 1]).max() < 1e-14 and np.abs(cl[:, 0]).max() > 0.1
    # Mdiag on a Gaussian spinor field = (4 + m) x + Cl x
    x = inputs.gaussian_field((int(np.prod(dims)), 2, 12), inputs.rng(stream=77))
    y = orc.wilson_clover(dims, U, cl, m, 0, x, orc.OP_MDIAG)
    assert np.abs(y - ((4 + m) * x + np.einsum("ab,srb->sra", full, x))).max() < 1e-13

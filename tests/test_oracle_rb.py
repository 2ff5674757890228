"""Pins the red-black (checkerboarded) coarse operator of the oracle against the
identities the reference asserts for Rework::CoarsenedMatrix
(src/Test_coarse_red_black.cc:170-530, tolerance 1e-15 relative squared deviation):

  Dhop + Mdiag = M ........................................ :176-205
  Meo + Moe = Dhop ........................................ :207-247
  Im<v, M^dag M v> = 0 .................................... :249-272
  MooeeInv Mooee = 1 (full grid, each checkerboard) ....... :274-300, 334-389
  <phi|Meo chi>* = <chi|Meo^dag phi> ...................... :302-346
  MooeeDag MooeeInvDag = 1 (each checkerboard) ............ :391-431
  Meo + Moe + Moo + Mee = M ............................... :433-482
  MpcDagMpc hermitian (NonHermitianSchurDiagMooeeOperator) :484-530

The coarse operator comes from a Galerkin coarsening of Wilson-clover, as in
the reference test.  Half fields: sites of parity (x+y+z+t) % 2, half index
x/2 + (Lx/2)(y + Ly(z + Lz t)) (Grid's red-black grid).
"""
import numpy as np
import pytest

import oracle as orc
import inputs

TOL = 1e-15


@pytest.fixture(scope="module")
def rb():
    fdims, cdims = (8, 8, 8, 8), (4, 4, 4, 4)
    r = inputs.rng(stream=61)
    U = inputs.hot_gauge(fdims, r)
    cl = orc.clover_build(fdims, U, 1.0)
    h = inputs.gaussian_field((4, int(np.prod(fdims)), 12), inputs.rng(stream=62))
    B = orc.block_orthonormalise(fdims, cdims, orc.chiral_double(h, 0.5), passes=1)
    A = orc.coarsen_wilson(fdims, cdims, B, U, cl, 0.1, 0, 0, variant=1)
    inv = orc.invert_self_links(A)
    src = inputs.gaussian_field((256, 2, A.shape[2]), inputs.rng(stream=63))
    return cdims, A, inv, src


def halves(dims, x):
    return orc.pick_checkerboard(dims, 0, x), orc.pick_checkerboard(dims, 1, x)


def full(dims, e, o):
    f = np.zeros((2 * e.shape[0],) + e.shape[1:], dtype=np.complex128)
    orc.set_checkerboard(dims, 0, e, f)
    orc.set_checkerboard(dims, 1, o, f)
    return f


def test_pick_set_round_trip(rb):
    dims, A, inv, src = rb
    e, o = halves(dims, src)
    assert np.array_equal(full(dims, e, o), src)
    # the half index of a site: x/2 + (Lx/2) (y + Ly (z + Lz t))
    s = 1 + 4 * (2 + 4 * (3 + 4 * 1))  # (1, 2, 3, 1): parity 1
    h = 0 + 2 * (2 + 4 * (3 + 4 * 1))
    assert np.array_equal(o[h], src[s])


def test_dhop_plus_mdiag_is_m(rb):
    dims, A, inv, src = rb
    ref = orc.coarse_apply(dims, A, src)
    res = orc.coarse_dhop(dims, A, src) + orc.coarse_apply(dims, A, src, op=orc.OP_MDIAG)
    assert orc.rel_dev_sq(ref, res) < TOL


def test_meo_plus_moe_is_dhop(rb):
    dims, A, inv, src = rb
    e, o = halves(dims, src)
    r_o = orc.coarse_rb_apply(dims, A, e, orc.RB_MEOOE, 0)
    r_e = orc.coarse_rb_apply(dims, A, o, orc.RB_MEOOE, 1)
    assert orc.rel_dev_sq(orc.coarse_dhop(dims, A, src), full(dims, r_e, r_o)) < TOL


def test_im_vdag_mdagm_v_is_zero(rb):
    dims, A, inv, src = rb
    v = src[:, :1]
    phi = orc.coarse_apply(dims, A, orc.coarse_apply(dims, A, v), op=orc.OP_MDAG)
    dot = np.vdot(v, phi)
    assert abs(dot.imag) / abs(dot.real) < TOL


def test_mooee_inverse_full_and_checkerboards(rb):
    dims, A, inv, src = rb
    y = orc.coarse_mooee(dims, A, orc.coarse_mooee(dims, A, src, orc.RB_MOOEE), orc.RB_MOOEE_INV, inv)
    assert orc.rel_dev_sq(src, y) < TOL
    for cb, x in enumerate(halves(dims, src)):
        y = orc.coarse_rb_apply(dims, A, orc.coarse_rb_apply(dims, A, x, orc.RB_MOOEE, cb), orc.RB_MOOEE_INV, cb, inv)
        assert orc.rel_dev_sq(x, y) < TOL
        y = orc.coarse_rb_apply(dims, A, orc.coarse_rb_apply(dims, A, x, orc.RB_MOOEE_INV_DAG, cb, inv),
                                orc.RB_MOOEE_DAG, cb)
        assert orc.rel_dev_sq(x, y) < TOL


def test_meooe_dagger(rb):
    dims, A, inv, src = rb
    r = inputs.rng(stream=64)
    phi = inputs.gaussian_field(src.shape, r)
    chi = inputs.gaussian_field(src.shape, r)
    chi_e, chi_o = halves(dims, chi)
    phi_e, phi_o = halves(dims, phi)
    dchi_o = orc.coarse_rb_apply(dims, A, chi_e, orc.RB_MEOOE, 0)
    dphi_e = orc.coarse_rb_apply(dims, A, phi_o, orc.RB_MEOOE_DAG, 1)
    a, b = np.vdot(phi_o, dchi_o), np.vdot(chi_e, dphi_e)
    assert abs(a - np.conj(b)) / abs(a) < 1e-13


def test_sum_of_blocks_is_m(rb):
    dims, A, inv, src = rb
    e, o = halves(dims, src)
    moe = orc.coarse_rb_apply(dims, A, e, orc.RB_MEOOE, 0)
    meo = orc.coarse_rb_apply(dims, A, o, orc.RB_MEOOE, 1)
    mee = orc.coarse_rb_apply(dims, A, e, orc.RB_MOOEE, 0)
    moo = orc.coarse_rb_apply(dims, A, o, orc.RB_MOOEE, 1)
    assert orc.rel_dev_sq(orc.coarse_apply(dims, A, src), full(dims, mee + meo, moo + moe)) < TOL


def mpc(dims, A, inv, x, cb, dag=False):
    """NonHermitianSchurDiagMooeeOperator: Mpc = Mcc - Mc,c' Mc'c'^-1 Mc',c on parity cb."""
    hop, diag, dinv = ((orc.RB_MEOOE_DAG, orc.RB_MOOEE_DAG, orc.RB_MOOEE_INV_DAG) if dag else
                       (orc.RB_MEOOE, orc.RB_MOOEE, orc.RB_MOOEE_INV))
    t = orc.coarse_rb_apply(dims, A, x, hop, cb)
    t = orc.coarse_rb_apply(dims, A, t, dinv, 1 - cb, inv)
    t = orc.coarse_rb_apply(dims, A, t, hop, 1 - cb)
    return orc.coarse_rb_apply(dims, A, x, diag, cb) - t


def test_mpcdagmpc_hermitian(rb):
    dims, A, inv, src = rb
    r = inputs.rng(stream=65)
    for cb in (0, 1):
        phi = orc.pick_checkerboard(dims, cb, inputs.gaussian_field(src.shape, r))
        chi = orc.pick_checkerboard(dims, cb, inputs.gaussian_field(src.shape, r))
        dchi = mpc(dims, A, inv, mpc(dims, A, inv, chi, cb), cb, dag=True)
        dphi = mpc(dims, A, inv, mpc(dims, A, inv, phi, cb), cb, dag=True)
        a, b = np.vdot(phi, dchi), np.vdot(chi, dphi)
        assert abs(a - np.conj(b)) / abs(a) < 1e-13


def test_invert_self_links_matches_numpy(rb):
    dims, A, inv, src = rb
    assert np.allclose(inv, np.linalg.inv(A[8]), rtol=0, atol=1e-12 * np.abs(inv).max())

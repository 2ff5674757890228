"""GPU parity of the coarse-operator construction at the benchmark configurations.

Each case runs the chain a user runs on the GPU, through the C ABI, and the
same chain in the FP64 CPU oracle on the same seeded inputs:

  Gaussian test vectors -> chiral doubling -> block orthonormalisation ->
  CoarsenOperator (all 9 link fields) [-> coarse M / Mdag on a Gaussian vector]

The links are compared with the oracle's Upstream-semantics construction
(CoarsenedMatrixUpstream.h:755-931), one link field at a time, at the
reference's FP64 bound of 1e-15 relative squared deviation
(src/Benchmark_create_coarse_operator.cc:278-352,
src/Benchmark_create_coarse_coarse_operator.cc:217-381).  The coarse applies
use the bound of src/Benchmark_coarse_operator.cc:119-246 (1e-15).

Cases:
  - the plain coarse operator configuration: fine 16^4, Wilson-clover m=-0.1,
    c_sw=1, Haar-random SU(3) links, 12 vectors doubled to nbasis 24 on 4^4
    blocks, periodic and antiperiodic t, then M and Mdag on one coarse vector;
  - nbasis 40 on 4^4 blocks (the coarse-operator construction configuration's
    block and basis size) on a fine 8^4 lattice;
  - coarse-of-coarse at nbasis 40 on 2^4 blocks (the construction
    configuration's second level) on 8^4 -> 4^4 -> 2^4;
  - the construction in several batches of basis vectors (forced smaller than
    the basis, uneven last batch), for the Wilson-clover and the coarse fine
    operator;
  - the two-spin (Rework) subspace and link forms against the Upstream ones,
    on a Wilson-clover and on a coarse fine level.
"""
import numpy as np
import pytest
import torch

import gmg
import inputs
import oracle as orc

pytestmark = pytest.mark.gpu

TOL64 = 1e-15


def _gpu_basis(fd, cd, h, dof):
    """Chiral doubling (G5C, factor 1/2) and one block-orthonormalisation pass on
    the GPU; h [nvec][V][dof].  Returns the aggregation and the oracle's basis
    built from the same vectors."""
    nvec, V, _ = h.shape
    x = torch.from_numpy(np.ascontiguousarray(h.transpose(1, 0, 2))).cuda()
    B = gmg.chiral_double(x, 0.5)
    ag = gmg.Aggregation(fd, cd, dof, 2 * nvec)
    ag.set_basis(B)
    ag.Orthogonalise(passes=1)
    ref_B = orc.block_orthonormalise(fd, cd, orc.chiral_double(h, 0.5), passes=1)
    got_B = ag.get_basis()
    # Cholesky QR (GPU) and modified Gram-Schmidt (oracle) give the same basis up to rounding
    assert orc.rel_dev_sq(ref_B, got_B) < 1e-24
    assert ag.CheckOrthogonal() < 1e-13
    return ag, ref_B


def _check_links(ref, got, what):
    for p in range(9):
        d = orc.rel_dev_sq(ref[p], got[p])
        assert d < TOL64, (what, p, d)


@pytest.mark.parametrize("apbc", [0, 1])
def test_plain_coarse_operator_config_end_to_end(apbc):
    fd, cd, mass, csw = (16, 16, 16, 16), (4, 4, 4, 4), -0.1, 1.0
    U = inputs.hot_gauge(fd, inputs.rng(stream=171))
    h = inputs.gaussian_field((12, int(np.prod(fd)), 12), inputs.rng(stream=172))
    ag, B = _gpu_basis(fd, cd, h, 12)
    w = gmg.WilsonClover(fd, mass, csw, antiperiodic=apbc)
    w.set_gauge(U)
    cm = gmg.CoarsenedMatrix(cd, 24)
    cm.CoarsenOperator(ag, w)
    cl = orc.clover_build(fd, U, csw)
    ref = orc.coarsen_wilson(fd, cd, B, U, cl, mass, apbc, 0, variant=0)
    got = cm.get_links()
    _check_links(ref, got, "16^4 -> 4^4, nbasis 24")
    # M and Mdag on one unit-Gaussian coarse vector, each side with its own links
    x = inputs.gaussian_field((256, 1, 24), inputs.rng(stream=173))
    xd = torch.from_numpy(x).cuda()
    for op, fn in ((orc.OP_M, cm.M), (orc.OP_MDAG, cm.Mdag)):
        want = orc.coarse_apply(cd, ref, x, op)
        out = torch.zeros_like(xd)
        fn(xd, out)
        torch.cuda.synchronize()
        assert orc.rel_dev_sq(want, out.cpu().numpy()) < TOL64, op


def test_coarsen_nbasis40_on_4x4_blocks():
    fd, cd, mass = (8, 8, 8, 8), (2, 2, 2, 2), -0.3
    U = inputs.smooth_gauge(fd, inputs.rng(stream=174), 0.3)
    h = inputs.gaussian_field((20, int(np.prod(fd)), 12), inputs.rng(stream=175))
    ag, B = _gpu_basis(fd, cd, h, 12)
    w = gmg.WilsonClover(fd, mass, 1.0, antiperiodic=1)
    w.set_gauge(U)
    cm = gmg.CoarsenedMatrix(cd, 40)
    cm.CoarsenOperator(ag, w)
    ref = orc.coarsen_wilson(fd, cd, B, U, orc.clover_build(fd, U, 1.0), mass, 1, 0, variant=0)
    _check_links(ref, cm.get_links(), "8^4 -> 2^4, nbasis 40")


def test_coarse_of_coarse_nbasis40_on_2x4_blocks():
    fd, c1, c2, mass = (8, 8, 8, 8), (4, 4, 4, 4), (2, 2, 2, 2), -0.3
    U = inputs.smooth_gauge(fd, inputs.rng(stream=176), 0.3)
    h = inputs.gaussian_field((20, int(np.prod(fd)), 12), inputs.rng(stream=177))
    ag, B = _gpu_basis(fd, c1, h, 12)
    w = gmg.WilsonClover(fd, mass, 1.0, antiperiodic=1)
    w.set_gauge(U)
    cm = gmg.CoarsenedMatrix(c1, 40)
    cm.CoarsenOperator(ag, w)
    A1 = orc.coarsen_wilson(fd, c1, B, U, orc.clover_build(fd, U, 1.0), mass, 1, 0, variant=0)
    _check_links(A1, cm.get_links(), "8^4 -> 4^4, nbasis 40")
    # second level: 20 coarse vectors doubled with G5C to nbasis 40 on 2^4 blocks,
    # the GPU level-1 operator as the fine operator
    h2 = inputs.gaussian_field((20, 256, 40), inputs.rng(stream=178))
    ag2, B2 = _gpu_basis(c1, c2, h2, 40)
    cc = gmg.CoarsenedMatrix(c2, 40)
    cc.CoarsenOperator(ag2, cm)
    ref = orc.coarsen_coarse(c1, c2, B2, A1, variant=0)
    _check_links(ref, cc.get_links(), "4^4 -> 2^4, nbasis 40")


@pytest.mark.parametrize("batch", [3, 5])
def test_coarsen_in_forced_batches(batch):
    # the basis split into batches of `batch` vectors (8 = 3 + 3 + 2 or 5 + 3):
    # every batch writes its own columns of the nine link fields
    fd, cd = (8, 8, 8, 8), (2, 2, 2, 2)
    U = inputs.hot_gauge(fd, inputs.rng(stream=179))
    h = inputs.gaussian_field((4, int(np.prod(fd)), 12), inputs.rng(stream=180))
    ag, B = _gpu_basis(fd, cd, h, 12)
    ag.set_coarsen_batch(batch)
    w = gmg.WilsonClover(fd, -0.1, 1.0, antiperiodic=1)
    w.set_gauge(U)
    cm = gmg.CoarsenedMatrix(cd, 8)
    cm.CoarsenOperator(ag, w)
    cl = orc.clover_build(fd, U, 1.0)
    ref = orc.coarsen_wilson(fd, cd, B, U, cl, -0.1, 1, 0, variant=0)
    _check_links(ref, cm.get_links(), f"Wilson-clover, batches of {batch}")
    # the same aggregation back at the default batch: same links
    ag.set_coarsen_batch(0)
    cm2 = gmg.CoarsenedMatrix(cd, 8)
    cm2.CoarsenOperator(ag, w)
    _check_links(ref, cm2.get_links(), "default batch")
    # coarse-of-coarse in batches: 2^4 coarse lattice of the level above as the fine operator
    c1 = (4, 4, 4, 4)
    h1 = inputs.gaussian_field((3, int(np.prod(fd)), 12), inputs.rng(stream=181))
    ag1, B1 = _gpu_basis(fd, c1, h1, 12)
    A1 = orc.coarsen_wilson(fd, c1, B1, U, cl, -0.1, 1, 0, variant=0)
    fine = gmg.CoarsenedMatrix(c1, 6)
    fine.set_links(A1)
    h2 = inputs.gaussian_field((4, 256, 6), inputs.rng(stream=182))
    ag2, B2 = _gpu_basis(c1, (2, 2, 2, 2), h2, 6)
    ag2.set_coarsen_batch(batch)
    cc = gmg.CoarsenedMatrix((2, 2, 2, 2), 8)
    cc.CoarsenOperator(ag2, fine)
    _check_links(orc.coarsen_coarse(c1, (2, 2, 2, 2), B2, A1, variant=0), cc.get_links(),
                 f"coarse-of-coarse, batches of {batch}")


@pytest.mark.parametrize("level", ["fine", "coarse"])
def test_two_spin_surface_matches_upstream(level):
    # The Rework (two-spin) forms through the C ABI, as
    # src/Benchmark_create_coarse_operator.cc:355-467 checks them: the Upstream
    # subspace with its chiral doubling undone goes into the two-spin subspace
    # (and comes back unchanged), the coarse operator built from it has
    # Y_[p] = convertLayout(A[p]) for every point, and the links set in the
    # two-spin form read back in the flat one
    if level == "fine":
        fd, cd, dof, nvec = (8, 8, 8, 8), (2, 2, 2, 2), 12, 6
    else:
        fd, cd, dof, nvec = (4, 4, 4, 4), (2, 2, 2, 2), 8, 5
    V = int(np.prod(fd))
    h = inputs.gaussian_field((nvec, V, dof), inputs.rng(stream=185))
    up = orc.block_orthonormalise(fd, cd, orc.chiral_double(h, 0.5), passes=1)
    undone = orc.undo_chiral_double(up)
    ag2 = gmg.Aggregation(fd, cd, dof, 2 * nvec)
    ag2.set_subspace_spins(undone, 2)
    assert np.array_equal(ag2.get_basis(), up)  # the chiral halves have disjoint supports: exact
    assert np.array_equal(ag2.get_subspace_spins(2), undone)
    if level == "fine":
        U = inputs.hot_gauge(fd, inputs.rng(stream=186))
        w = gmg.WilsonClover(fd, -0.1, 1.0, antiperiodic=1)
        w.set_gauge(U)
        cm = gmg.CoarsenedMatrix(cd, 2 * nvec)
        cm.CoarsenOperator(ag2, w)
        ref = orc.coarsen_wilson(fd, cd, up, U, orc.clover_build(fd, U, 1.0), -0.1, 1, 0, variant=0)
    else:
        fine = gmg.CoarsenedMatrix(fd, dof)
        A1 = inputs.random_links(fd, dof, inputs.rng(stream=187))
        fine.set_links(A1)
        cm = gmg.CoarsenedMatrix(cd, 2 * nvec)
        cm.CoarsenOperator(ag2, fine)
        ref = orc.coarsen_coarse(fd, cd, up, A1, variant=0)
    got = cm.get_links()
    _check_links(ref, got, f"two-spin subspace, {level} level")
    Y = np.stack([cm.get_links_spins(p, 2) for p in range(9)])
    for p in range(9):
        want = orc.layout_link_flat_to_spin(got[p], 2).reshape(Y[p].shape)
        assert np.array_equal(want, Y[p])
    cm2 = gmg.CoarsenedMatrix(cd, 2 * nvec)
    cm2.set_links_spins(Y, 2)
    assert np.array_equal(cm2.get_links(), got)

"""numpy/ctypes front end of the CPU FP64 oracle (oracle/gmg_oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
cpu_baseline leg of bench.py as the checker of the CUDA library.  Parity with
the reference is pinned by the reference's identity / known-answer checks;
absolute values of Grid's fine operator are parity unpinned (Grid is absent).

All arrays are complex128 numpy arrays in the layouts documented in
oracle/gmg_oracle.h.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

OP_M, OP_MDAG, OP_MDIAG, OP_MDIR = 0, 1, 2, 3


def build():
    subprocess.check_call(["make", "-s", "-C", _HERE])


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        _LIB = ctypes.CDLL(path)
    return _LIB


def _i4(dims):
    return (ctypes.c_int * 4)(*[int(d) for d in dims])


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p) if a is not None else None


def _c(a):
    a = np.ascontiguousarray(a, dtype=np.complex128)
    return a


def vol(dims):
    return int(np.prod(dims))


def point_from_dir_disp(ndim, dirs_faster, d, disp):
    return lib().orc_point_from_dir_disp(ndim, int(dirs_faster), d, disp)


def geometry(ndim, dirs_faster=True):
    dirs = (ctypes.c_int * 9)()
    disps = (ctypes.c_int * 9)()
    lib().orc_geometry(ndim, int(dirs_faster), dirs, disps)
    return list(dirs), list(disps)


def coarse_neighbors(dims):
    out = np.zeros((9, vol(dims)), dtype=np.int32)
    lib().orc_coarse_neighbors(_i4(dims), _p(out))
    return out


def lut(fdims, cdims, mask=None):
    b = [f // c for f, c in zip(fdims, cdims)]
    bv = int(np.prod(b))
    Vc, Vf = vol(cdims), vol(fdims)
    l = np.zeros((Vc, bv), dtype=np.int32)
    sizes = np.zeros(Vc, dtype=np.int32)
    rev = np.zeros(Vf, dtype=np.int32)
    m = None if mask is None else np.ascontiguousarray(mask, dtype=np.int8)
    lib().orc_lut_populate(_i4(fdims), _i4(cdims), _p(m), _p(l), _p(sizes), _p(rev))
    return l, sizes, rev


def outer_mask(fdims, cdims, point):
    m = np.zeros(vol(fdims), dtype=np.int8)
    lib().orc_outer_mask(_i4(fdims), _i4(cdims), point, _p(m))
    return m


def parity_mask(fdims, cdims, parity):
    m = np.zeros(vol(fdims), dtype=np.int8)
    lib().orc_block_parity_mask(_i4(fdims), _i4(cdims), parity, _p(m))
    return m


def coarse_apply(dims, links, x, op=OP_M, point=8, hermitian=0):
    """links [9][V][N][N], x [V][R][N] -> y [V][R][N]."""
    links = _c(links)
    x = _c(x)
    V, R, N = x.shape
    y = np.empty_like(x)
    lib().orc_coarse_apply(_i4(dims), N, R, _p(links), _p(x), _p(y), op, point, hermitian)
    return y


def set_threads(n):
    """OpenMP threads of the oracle's parallel loops (n <= 0: all host threads); returns the previous count."""
    return lib().orc_set_threads(int(n))


def coarse_apply_range(dims, links, x, y, s0, s1, op=OP_M, point=8, hermitian=0):
    """In-place y[s0:s1] = op(x) on output sites [s0, s1) (bounded timing samples)."""
    V, R, N = x.shape
    lib().orc_coarse_apply_range(_i4(dims), N, R, _p(links), _p(x), _p(y), op, point, hermitian,
                                 ctypes.c_int64(s0), ctypes.c_int64(s1))
    return y


def block_project(fdims, cdims, basis, fine, mask=None):
    """basis [N][Vf][dof], fine [Vf][R][dof] -> coarse [Vc][R][N]."""
    basis = _c(basis)
    fine = _c(fine)
    N, Vf, dof = basis.shape
    R = fine.shape[1]
    out = np.zeros((vol(cdims), R, N), dtype=np.complex128)
    m = None if mask is None else np.ascontiguousarray(mask, dtype=np.int8)
    lib().orc_block_project(_i4(fdims), _i4(cdims), dof, N, R, _p(basis), _p(fine), _p(out), _p(m))
    return out


def block_promote(fdims, cdims, basis, coarse):
    basis = _c(basis)
    coarse = _c(coarse)
    N, Vf, dof = basis.shape
    R = coarse.shape[1]
    out = np.zeros((Vf, R, dof), dtype=np.complex128)
    lib().orc_block_promote(_i4(fdims), _i4(cdims), dof, N, R, _p(basis), _p(coarse), _p(out))
    return out


def block_orthonormalise(fdims, cdims, basis, passes=1):
    b = _c(basis).copy()
    N, Vf, dof = b.shape
    lib().orc_block_orthonormalise(_i4(fdims), _i4(cdims), dof, N, _p(b), passes)
    return b


def chiral_double(basis_half, factor=0.5):
    """basis_half [nb][V][dof] -> doubled [2nb][V][dof] (G5C: factor 1/2, G5R5: 1)."""
    h = _c(basis_half)
    nb, V, dof = h.shape
    out = np.zeros((2 * nb, V, dof), dtype=np.complex128)
    out[:nb] = h
    lib().orc_chiral_double(ctypes.c_int64(V), dof, nb, _p(out), ctypes.c_double(factor))
    return out


def undo_chiral_double(basis):
    b = _c(basis).copy()
    n2, V, dof = b.shape
    lib().orc_undo_chiral_double(ctypes.c_int64(V), dof, n2 // 2, _p(b))
    return b[: n2 // 2]


def gamma(mu):
    g = np.zeros((4, 4), dtype=np.complex128)
    lib().orc_gamma(mu, _p(g))
    return g


def clover_build(dims, U, csw):
    U = _c(U)
    cl = np.zeros((vol(dims), 2, 6, 6), dtype=np.complex128)
    lib().orc_clover_build(_i4(dims), _p(U), ctypes.c_double(csw), _p(cl))
    return cl


def wilson_clover(dims, U, clover, mass, antiperiodic, x, op=OP_M, d=0, disp=0):
    """x [V][R][12] -> y [V][R][12]."""
    U = _c(U)
    x = _c(x)
    cl = None if clover is None else _c(clover)
    V, R, _ = x.shape
    y = np.zeros_like(x)
    lib().orc_wilson_clover_apply(_i4(dims), _p(U), _p(cl), ctypes.c_double(mass), int(antiperiodic),
                                  R, _p(x), _p(y), op, d, disp)
    return y


def coarsen_wilson(fdims, cdims, basis, U, clover, mass, antiperiodic, hermitian=0, variant=1):
    basis = _c(basis)
    N = basis.shape[0]
    links = np.zeros((9, vol(cdims), N, N), dtype=np.complex128)
    cl = None if clover is None else _c(clover)
    lib().orc_coarsen_wilson(_i4(fdims), _i4(cdims), N, _p(basis), _p(_c(U)), _p(cl),
                             ctypes.c_double(mass), int(antiperiodic), hermitian, variant, _p(links))
    return links


def coarsen_coarse(fdims, cdims, basis, flinks, fhermitian=0, hermitian=0, variant=1):
    basis = _c(basis)
    flinks = _c(flinks)
    N, Vf, Nf = basis.shape
    links = np.zeros((9, vol(cdims), N, N), dtype=np.complex128)
    lib().orc_coarsen_coarse(_i4(fdims), _i4(cdims), Nf, N, _p(basis), _p(flinks), fhermitian,
                             hermitian, variant, _p(links))
    return links


def construct_remaining_links(dims, links, hermitian=0):
    l = _c(links).copy()
    N = l.shape[-1]
    lib().orc_construct_remaining_links(_i4(dims), N, _p(l), hermitian)
    return l


def layout_vec_flat_to_spin(x, ncs):
    x = _c(x)
    V, N = x.shape[0] * (x.size // (x.shape[0] * x.shape[-1])), x.shape[-1]
    out = np.empty_like(x)
    lib().orc_layout_vec_flat_to_spin(ctypes.c_int64(V), N, ncs, _p(x), _p(out))
    return out


def layout_link_flat_to_spin(a, ncs):
    a = _c(a)
    N = a.shape[-1]
    V = a.size // (N * N)
    out = np.empty_like(a)
    lib().orc_layout_link_flat_to_spin(ctypes.c_int64(V), N, ncs, _p(a), _p(out))
    return out


def rel_dev_sq(ref, res):
    """Reference's relative squared deviation |ref-res|^2/|ref|^2 (Benchmark_helpers.h:215-236)."""
    ref = np.asarray(ref)
    res = np.asarray(res)
    return float(np.sum(np.abs(ref - res) ** 2) / np.sum(np.abs(ref) ** 2))


# ----------------------------------------------------------------------------
# red-black coarse operator (CoarsenedMatrixRework.h:178-245, 288-394, 617-679)
# ----------------------------------------------------------------------------
RB_MEOOE, RB_MEOOE_DAG, RB_MOOEE, RB_MOOEE_DAG, RB_MOOEE_INV, RB_MOOEE_INV_DAG = range(6)


def pick_checkerboard(dims, cb, full):
    """full [V][...] -> half [V/2][...] (sites of parity cb, half index x/2 + Lx/2 * (...))."""
    full = _c(full)
    per = int(np.prod(full.shape[1:])) if full.ndim > 1 else 1
    half = np.zeros((full.shape[0] // 2,) + full.shape[1:], dtype=np.complex128)
    lib().orc_pick_checkerboard(_i4(dims), cb, ctypes.c_int64(per), _p(full), _p(half))
    return half


def set_checkerboard(dims, cb, half, full):
    """Writes the half field into the parity-cb sites of full (in place)."""
    half = _c(half)
    per = int(np.prod(half.shape[1:])) if half.ndim > 1 else 1
    lib().orc_set_checkerboard(_i4(dims), cb, ctypes.c_int64(per), _p(half), _p(full))
    return full


def invert_self_links(links):
    """links [9][V][N][N] -> inverse of the self link per site, [V][N][N]."""
    links = _c(links)
    V, N = links.shape[1], links.shape[2]
    a8 = np.ascontiguousarray(links[8])
    inv = np.zeros_like(a8)
    lib().orc_invert_self_links.restype = ctypes.c_int
    bad = lib().orc_invert_self_links(ctypes.c_int64(V), N, _p(a8), _p(inv))
    if bad:
        raise ValueError(f"{bad} singular self links")
    return inv


def coarse_rb_apply(dims, links, x_half, op, cb, self_inv=None):
    """Half field x (parity cb) -> Meooe / Mooee family output half field."""
    links = _c(links)
    x_half = _c(x_half)
    Vh, R, N = x_half.shape
    y = np.zeros_like(x_half)
    si = None if self_inv is None else _c(self_inv)
    lib().orc_coarse_rb_apply(_i4(dims), N, R, _p(links), _p(si), op, cb, _p(x_half), _p(y))
    return y


def coarse_dhop(dims, links, x, dag=0):
    links = _c(links)
    x = _c(x)
    V, R, N = x.shape
    y = np.zeros_like(x)
    lib().orc_coarse_dhop(_i4(dims), N, R, _p(links), int(dag), _p(x), _p(y))
    return y


def coarse_mooee(dims, links, x, op, self_inv=None):
    """Full-grid Mooee family (op RB_MOOEE..RB_MOOEE_INV_DAG)."""
    links = _c(links)
    x = _c(x)
    V, R, N = x.shape
    y = np.zeros_like(x)
    si = None if self_inv is None else _c(self_inv)
    lib().orc_coarse_mooee(_i4(dims), N, R, _p(links), _p(si), op, _p(x), _p(y))
    return y

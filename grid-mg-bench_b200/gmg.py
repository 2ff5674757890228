"""Python binding of libgmg_b200.so (ctypes over the C ABI in include/gmg.h).

Mirrors the reference's class surface so that tests read like the reference's
own drivers:

  CoarsenedMatrix   M, Mdag, Mdiag, Mdir, MdirAll, CoarsenOperator, links A
                    (include/CoarsenedMatrixUpstream.h:515-931); red-black
                    Dhop, Meooe[Dag], Mooee[Inv][Dag], InvertSelfStencilPoint
                    (include/CoarsenedMatrixRework.h:178-245, 617-679)
  Aggregation       Orthogonalise, CheckOrthogonal, ProjectToSubspace,
                    PromoteFromSubspace, subspace (...LutMRHS.h:293-352)
  WilsonClover      Op/AdjOp/OpDiag/OpDir of the fine operator
                    (MdagMLinearOperator over WilsonCloverFermionR)

Vectors are torch CUDA tensors: complex128 (FP64) or complex64 (FP32) with
shape [sites, nrhs, dof].  There is no CPU fallback: without the built
library or a GPU every call raises.
"""
import ctypes
import os

import numpy as np
import torch

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libgmg_b200.so")
_LIB = None

F64, F32, BF16, F16 = 0, 1, 2, 3
OP_M, OP_MDAG, OP_MDIAG, OP_MDIR = 0, 1, 2, 3
RB_MEOOE, RB_MEOOE_DAG, RB_MOOEE, RB_MOOEE_DAG, RB_MOOEE_INV, RB_MOOEE_INV_DAG = range(6)
EVEN, ODD = 0, 1
PREC = {"f64": F64, "f32": F32, "bf16": BF16, "f16": F16}


class GmgError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"gmg status {status}: {msg}")
        self.status = status


def lib():
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with grid-mg-bench_b200/build.py")
        _LIB = ctypes.CDLL(LIB_PATH)
        _LIB.gmg_last_error.restype = ctypes.c_char_p
        _LIB.gmg_version.restype = ctypes.c_char_p
    return _LIB


def _chk(st):
    if st != 0:
        raise GmgError(st, lib().gmg_last_error().decode())


def _dims(d):
    return (ctypes.c_int * 4)(*[int(x) for x in d])


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def _vec_prec(t):
    if t.dtype == torch.complex128:
        return F64
    if t.dtype == torch.complex64:
        return F32
    raise TypeError(f"vectors must be complex128 or complex64, got {t.dtype}")


def _check_vec(t, V, dof, name):
    if not t.is_cuda or not t.is_contiguous():
        raise ValueError(f"{name} must be a contiguous CUDA tensor")
    if t.dim() != 3 or t.shape[0] != V or t.shape[2] != dof:
        raise ValueError(f"{name} must have shape [{V}, nrhs, {dof}], got {tuple(t.shape)}")


def vol(d):
    return int(np.prod(d))


class CoarsenedMatrix:
    """CoarsenedMatrix(CoarseGrid, hermitian) over the 9-point coarse stencil."""

    def __init__(self, dims, nbasis, hermitian=0):
        self.dims = tuple(int(x) for x in dims)
        self.N = int(nbasis)
        self.hermitian = int(hermitian)
        self.V = vol(self.dims)
        h = ctypes.c_void_p()
        _chk(lib().gmg_coarse_create(_dims(self.dims), self.N, self.hermitian, ctypes.byref(h)))
        self._h = h

    def __del__(self):
        if getattr(self, "_h", None) and _LIB is not None:
            _LIB.gmg_coarse_destroy(self._h)
            self._h = None

    # link fields A[p], exchange layout [9][V][N][N]
    def set_links(self, A):
        if isinstance(A, torch.Tensor):
            A = A.to(torch.complex128).contiguous()
            _chk(lib().gmg_coarse_set_links(self._h, _ptr(A), 1 if A.is_cuda else 0, _stream()))
            torch.cuda.current_stream().synchronize()
        else:
            a = np.ascontiguousarray(A, dtype=np.complex128)
            assert a.shape == (9, self.V, self.N, self.N)
            _chk(lib().gmg_coarse_set_links(self._h, a.ctypes.data_as(ctypes.c_void_p), 0, _stream()))

    def get_links(self):
        a = np.zeros((9, self.V, self.N, self.N), dtype=np.complex128)
        _chk(lib().gmg_coarse_get_links(self._h, a.ctypes.data_as(ctypes.c_void_p), 0, _stream()))
        return a

    def get_links_spins(self, point, ncoarse_spins=2):
        """Rework link field Y_[point] as [V][Ns_c][Ns_c][Nc_c][Nc_c] complex128."""
        nc = self.N // ncoarse_spins
        y = np.zeros((self.V, ncoarse_spins, ncoarse_spins, nc, nc), dtype=np.complex128)
        _chk(lib().gmg_coarse_get_links_spins(self._h, int(ncoarse_spins), int(point),
                                              y.ctypes.data_as(ctypes.c_void_p), 0, _stream()))
        return y

    def set_links_spins(self, Y, ncoarse_spins=2):
        y = np.ascontiguousarray(Y, dtype=np.complex128)
        _chk(lib().gmg_coarse_set_links_spins(self._h, int(ncoarse_spins), y.ctypes.data_as(ctypes.c_void_p), 0,
                                              _stream()))

    def prepare(self, compute):
        _chk(lib().gmg_coarse_prepare(self._h, PREC.get(compute, compute), _stream()))

    def apply(self, op, inp, out, point=8, compute=None, active=None):
        _check_vec(inp, self.V, self.N, "in")
        _check_vec(out, self.V, self.N, "out")
        vp = _vec_prec(inp)
        if _vec_prec(out) != vp or out.shape != inp.shape:
            raise ValueError("in and out must match in shape and dtype")
        c = vp if compute is None else PREC.get(compute, compute)
        act = None
        n_act = 0
        if active is not None:
            act = active if isinstance(active, torch.Tensor) else torch.tensor(active, dtype=torch.int32,
                                                                               device=inp.device)
            assert act.dtype == torch.int32 and act.is_cuda
            n_act = act.numel()
        _chk(lib().gmg_coarse_apply(self._h, op, point, c, vp, inp.shape[1], _ptr(inp), _ptr(out),
                                    _ptr(act) if act is not None else None, n_act, _stream()))
        return out

    def M(self, inp, out, **kw):
        return self.apply(OP_M, inp, out, **kw)

    def Mdag(self, inp, out, **kw):
        return self.apply(OP_MDAG, inp, out, **kw)

    def Mdiag(self, inp, out, **kw):
        return self.apply(OP_MDIAG, inp, out, **kw)

    def Mdir(self, inp, out, d, disp, **kw):
        p = lib().gmg_point_from_dir_disp(4, 1, d, disp)
        if p < 0:
            raise ValueError("bad direction / displacement")
        return self.apply(OP_MDIR, inp, out, point=p, **kw)

    def MdirAll(self, inp, outs, compute=None):
        assert len(outs) == 8
        vp = _vec_prec(inp)
        c = vp if compute is None else PREC.get(compute, compute)
        arr = (ctypes.c_void_p * 8)(*[o.data_ptr() for o in outs])
        _chk(lib().gmg_coarse_mdir_all(self._h, c, vp, inp.shape[1], _ptr(inp), arr, _stream()))
        return outs

    def construct_remaining_links(self):
        _chk(lib().gmg_coarse_construct_remaining_links(self._h, _stream()))

    # ---------------------------------------------------- red-black interface
    # Half fields: [V/2, nrhs, N], sites of one parity (x+y+z+t) % 2 at half
    # index x/2 + (Lx/2)(y + Ly(z + Lz t)).
    def InvertSelfStencilPoint(self):
        _chk(lib().gmg_coarse_invert_self(self._h, _stream()))

    def _rb(self, op, cb, inp, out, compute):
        _check_vec(inp, self.V // 2, self.N, "in")
        _check_vec(out, self.V // 2, self.N, "out")
        vp = _vec_prec(inp)
        if _vec_prec(out) != vp or out.shape != inp.shape:
            raise ValueError("in and out must match in shape and dtype")
        c = vp if compute is None else PREC.get(compute, compute)
        _chk(lib().gmg_coarse_apply_rb(self._h, op, int(cb), c, vp, inp.shape[1], _ptr(inp), _ptr(out), _stream()))
        return out

    def Meooe(self, inp, out, cb, compute=None):
        """in: half field of parity cb -> out: parity 1 - cb (DhopOE for cb even, DhopEO for odd)."""
        return self._rb(RB_MEOOE, cb, inp, out, compute)

    def MeooeDag(self, inp, out, cb, compute=None):
        return self._rb(RB_MEOOE_DAG, cb, inp, out, compute)

    def _mooee(self, op, inp, out, cb, compute):
        if cb is not None:
            return self._rb(op, cb, inp, out, compute)
        _check_vec(inp, self.V, self.N, "in")
        _check_vec(out, self.V, self.N, "out")
        vp = _vec_prec(inp)
        c = vp if compute is None else PREC.get(compute, compute)
        _chk(lib().gmg_coarse_mooee(self._h, op, c, vp, inp.shape[1], _ptr(inp), _ptr(out), _stream()))
        return out

    def Mooee(self, inp, out, cb=None, compute=None):
        """Self point; cb None = full grid, else a half field of parity cb."""
        return self._mooee(RB_MOOEE, inp, out, cb, compute)

    def MooeeDag(self, inp, out, cb=None, compute=None):
        return self._mooee(RB_MOOEE_DAG, inp, out, cb, compute)

    def MooeeInv(self, inp, out, cb=None, compute=None):
        return self._mooee(RB_MOOEE_INV, inp, out, cb, compute)

    def MooeeInvDag(self, inp, out, cb=None, compute=None):
        return self._mooee(RB_MOOEE_INV_DAG, inp, out, cb, compute)

    def Dhop(self, inp, out, dag=0, compute=None):
        _check_vec(inp, self.V, self.N, "in")
        _check_vec(out, self.V, self.N, "out")
        vp = _vec_prec(inp)
        c = vp if compute is None else PREC.get(compute, compute)
        _chk(lib().gmg_coarse_dhop(self._h, int(dag), c, vp, inp.shape[1], _ptr(inp), _ptr(out), _stream()))
        return out

    def neighbors(self):
        n = np.zeros((9, self.V), dtype=np.int32)
        _chk(lib().gmg_coarse_neighbors(self._h, n.ctypes.data_as(ctypes.c_void_p)))
        return n

    def CoarsenOperator(self, agg, linop):
        if isinstance(linop, WilsonClover):
            _chk(lib().gmg_coarsen_wilson(self._h, agg._h, linop._h, _stream()))
        elif isinstance(linop, CoarsenedMatrix):
            _chk(lib().gmg_coarsen_coarse(self._h, agg._h, linop._h, _stream()))
        else:
            raise TypeError("linop must be WilsonClover or CoarsenedMatrix")


def pick_checkerboard(dims, cb, full, half):
    """Grid's pickCheckerboard on device fields [V, ...] -> [V/2, ...] (complex128 / complex64)."""
    per = int(np.prod(full.shape[1:])) if full.dim() > 1 else 1
    _chk(lib().gmg_pick_checkerboard(_dims(dims), int(cb), per, _vec_prec(full), _ptr(full), _ptr(half), _stream()))
    return half


def set_checkerboard(dims, cb, half, full):
    per = int(np.prod(half.shape[1:])) if half.dim() > 1 else 1
    _chk(lib().gmg_set_checkerboard(_dims(dims), int(cb), per, _vec_prec(half), _ptr(half), _ptr(full), _stream()))
    return full


class Aggregation:
    """Aggregation(CoarseGrid, FineGrid): block basis, project / promote / orthonormalise."""

    def __init__(self, fine_dims, coarse_dims, site_dof, nbasis):
        self.fdims = tuple(int(x) for x in fine_dims)
        self.cdims = tuple(int(x) for x in coarse_dims)
        self.dof = int(site_dof)
        self.N = int(nbasis)
        self.Vf, self.Vc = vol(self.fdims), vol(self.cdims)
        h = ctypes.c_void_p()
        _chk(lib().gmg_agg_create(_dims(self.fdims), _dims(self.cdims), self.dof, self.N, ctypes.byref(h)))
        self._h = h

    def __del__(self):
        if getattr(self, "_h", None) and _LIB is not None:
            _LIB.gmg_agg_destroy(self._h)
            self._h = None

    def set_subspace_spins(self, vecs, ncoarse_spins=2):
        """Rework subspace in: vecs [nbasis / ncoarse_spins][Vf][dof] (complex128, host or device)."""
        if isinstance(vecs, torch.Tensor):
            v = vecs.to(torch.complex128).contiguous()
            _chk(lib().gmg_agg_set_subspace_spins(self._h, int(ncoarse_spins), _ptr(v), 1 if v.is_cuda else 0,
                                                  _stream()))
            torch.cuda.current_stream().synchronize()
        else:
            v = np.ascontiguousarray(vecs, dtype=np.complex128)
            _chk(lib().gmg_agg_set_subspace_spins(self._h, int(ncoarse_spins), v.ctypes.data_as(ctypes.c_void_p), 0,
                                                  _stream()))

    def get_subspace_spins(self, ncoarse_spins=2):
        v = np.zeros((self.N // ncoarse_spins, self.Vf, self.dof), dtype=np.complex128)
        _chk(lib().gmg_agg_get_subspace_spins(self._h, int(ncoarse_spins), v.ctypes.data_as(ctypes.c_void_p), 0,
                                              _stream()))
        return v

    def set_coarsen_batch(self, max_batch):
        """Cap the basis vectors per CoarsenOperator batch (0: sized from free memory)."""
        _chk(lib().gmg_agg_set_coarsen_batch(self._h, int(max_batch)))

    def set_basis(self, B):
        if isinstance(B, torch.Tensor):
            B = B.to(torch.complex128).contiguous()
            _chk(lib().gmg_agg_set_basis(self._h, _ptr(B), 1 if B.is_cuda else 0, _stream()))
            torch.cuda.current_stream().synchronize()
        else:
            b = np.ascontiguousarray(B, dtype=np.complex128)
            assert b.shape == (self.N, self.Vf, self.dof)
            _chk(lib().gmg_agg_set_basis(self._h, b.ctypes.data_as(ctypes.c_void_p), 0, _stream()))

    def get_basis(self):
        b = np.zeros((self.N, self.Vf, self.dof), dtype=np.complex128)
        _chk(lib().gmg_agg_get_basis(self._h, b.ctypes.data_as(ctypes.c_void_p), 0, _stream()))
        return b

    def Orthogonalise(self, passes=1):
        _chk(lib().gmg_agg_orthonormalise(self._h, passes, _stream()))

    def CheckOrthogonal(self):
        e = ctypes.c_double()
        _chk(lib().gmg_agg_check_orthogonal(self._h, ctypes.byref(e), _stream()))
        return e.value

    def ProjectToSubspace(self, fine, coarse, compute=None):
        _check_vec(fine, self.Vf, self.dof, "fine")
        _check_vec(coarse, self.Vc, self.N, "coarse")
        vp = _vec_prec(fine)
        c = vp if compute is None else PREC.get(compute, compute)
        _chk(lib().gmg_agg_project(self._h, c, vp, fine.shape[1], _ptr(fine), _ptr(coarse), _stream()))
        return coarse

    def PromoteFromSubspace(self, coarse, fine, compute=None):
        _check_vec(fine, self.Vf, self.dof, "fine")
        _check_vec(coarse, self.Vc, self.N, "coarse")
        vp = _vec_prec(fine)
        c = vp if compute is None else PREC.get(compute, compute)
        _chk(lib().gmg_agg_promote(self._h, c, vp, coarse.shape[1], _ptr(coarse), _ptr(fine), _stream()))
        return fine


class WilsonClover:
    """Fine Wilson-clover operator: Op (M), AdjOp (Mdag), OpDiag, OpDir."""

    def __init__(self, dims, mass, csw, antiperiodic=False):
        self.dims = tuple(int(x) for x in dims)
        self.V = vol(self.dims)
        h = ctypes.c_void_p()
        _chk(lib().gmg_wilson_create(_dims(self.dims), ctypes.c_double(mass), ctypes.c_double(csw),
                                     int(bool(antiperiodic)), ctypes.byref(h)))
        self._h = h

    def __del__(self):
        if getattr(self, "_h", None) and _LIB is not None:
            _LIB.gmg_wilson_destroy(self._h)
            self._h = None

    def set_gauge(self, U):
        if isinstance(U, torch.Tensor):
            u = U.to(torch.complex128).contiguous()
            assert tuple(u.shape) == (self.V, 4, 3, 3)
            _chk(lib().gmg_wilson_set_gauge(self._h, _ptr(u), 1 if u.is_cuda else 0, _stream()))
            torch.cuda.current_stream().synchronize()
            return
        u = np.ascontiguousarray(U, dtype=np.complex128)
        assert u.shape == (self.V, 4, 3, 3)
        _chk(lib().gmg_wilson_set_gauge(self._h, u.ctypes.data_as(ctypes.c_void_p), 0, _stream()))

    def clover(self):
        c = np.zeros((self.V, 2, 6, 6), dtype=np.complex128)
        _chk(lib().gmg_wilson_get_clover(self._h, c.ctypes.data_as(ctypes.c_void_p), 0, _stream()))
        return c

    def apply(self, op, inp, out, d=0, disp=0):
        _check_vec(inp, self.V, 12, "in")
        _check_vec(out, self.V, 12, "out")
        _chk(lib().gmg_wilson_apply(self._h, op, d, disp, _vec_prec(inp), inp.shape[1], _ptr(inp), _ptr(out),
                                    _stream()))
        return out

    def M(self, inp, out):
        return self.apply(OP_M, inp, out)

    def Mdag(self, inp, out):
        return self.apply(OP_MDAG, inp, out)

    def Mdiag(self, inp, out):
        return self.apply(OP_MDIAG, inp, out)

    def Mdir(self, inp, out, d, disp):
        return self.apply(OP_MDIR, inp, out, d, disp)

    KERNELS = {"auto": -1, "site": 0, "tile": 1, "quad": 2, "staged": 3}

    def set_kernel(self, name):
        """Force a kernel variant ("site", "tile", "quad", "staged") or "auto"."""
        _chk(lib().gmg_wilson_set_kernel(self._h, self.KERNELS[name]))

    def tuned_kernel(self, prec, nrhs, fused_mr=False, single_hop=False):
        k = ctypes.c_int()
        _chk(lib().gmg_wilson_tuned_kernel(self._h, PREC[prec], nrhs, int(fused_mr), int(single_hop),
                                           ctypes.byref(k)))
        return {v: n for n, v in self.KERNELS.items()}[k.value]

    def device_error(self):
        code = ctypes.c_int()
        st = lib().gmg_wilson_device_error(self._h, ctypes.byref(code))
        return st, code.value

    def M_f32_in(self, inp, out, dag=False):
        """out (complex128) = M in (or Mdag) with in complex64: FP64 arithmetic on the promoted input."""
        assert inp.dtype == torch.complex64 and out.dtype == torch.complex128
        _check_vec(inp, self.V, 12, "in")
        _check_vec(out, self.V, 12, "out")
        _chk(lib().gmg_wilson_apply_f32_in(self._h, OP_MDAG if dag else OP_M, inp.shape[1], _ptr(inp), _ptr(out),
                                           _stream()))
        return out

    def M_mr(self, inp, out):
        """out = M inp and the MR-step inner products <out, inp>, <out, out> per RHS.  BF16 fields
        are torch.bfloat16 tensors of shape [V, nrhs, 12, 2] (real, imaginary)."""
        if inp.dtype == torch.bfloat16:
            if inp.dim() != 4 or inp.shape[0] != self.V or inp.shape[2:] != (12, 2) or not inp.is_contiguous():
                raise ValueError("BF16 fields must be contiguous [V, nrhs, 12, 2]")
            assert out.dtype == torch.bfloat16 and out.shape == inp.shape and out.is_contiguous()
            prec = BF16
        else:
            _check_vec(inp, self.V, 12, "in")
            _check_vec(out, self.V, 12, "out")
            prec = _vec_prec(inp)
        d = torch.zeros((2, inp.shape[1]), dtype=torch.complex128, device=inp.device)
        _chk(lib().gmg_wilson_apply_mr(self._h, prec, inp.shape[1], _ptr(inp), _ptr(out), _ptr(d[0]), _ptr(d[1]),
                                       _stream()))
        return d[0], d[1].real


class GaugeInfo(ctypes.Structure):
    _fields_ = [("dims", ctypes.c_int * 4), ("two_row", ctypes.c_int), ("precision", ctypes.c_int),
                ("big_endian", ctypes.c_int), ("plaquette", ctypes.c_double), ("link_trace", ctypes.c_double),
                ("checksum", ctypes.c_uint32), ("checksum_data", ctypes.c_uint32)]

    def as_dict(self):
        return {"dims": tuple(self.dims), "two_row": self.two_row, "precision": self.precision,
                "big_endian": self.big_endian, "plaquette": self.plaquette, "link_trace": self.link_trace,
                "checksum": self.checksum, "checksum_data": self.checksum_data}


def read_nersc(path, verify=True):
    """NerscIO::readConfiguration: (links [V, 4, 3, 3] complex128, header info)."""
    info = GaugeInfo()
    _chk(lib().gmg_gauge_read_nersc(str(path).encode(), ctypes.byref(info), None, 0))
    U = np.zeros((vol(tuple(info.dims)), 4, 3, 3), dtype=np.complex128)
    _chk(lib().gmg_gauge_read_nersc(str(path).encode(), ctypes.byref(info), U.ctypes.data_as(ctypes.c_void_p),
                                    int(verify)))
    return U, info.as_dict()


def write_nersc(path, dims, U, two_row=False, precision=64, ensemble_id="synthetic", sequence_number=0):
    """NerscIO::writeConfiguration of host links [V, 4, 3, 3] complex128."""
    U = np.ascontiguousarray(U, dtype=np.complex128)
    _chk(lib().gmg_gauge_write_nersc(str(path).encode(), _dims(dims), U.ctypes.data_as(ctypes.c_void_p),
                                     int(two_row), int(precision), ensemble_id.encode(), int(sequence_number)))


def read_ildg(path):
    """IldgReader::readConfiguration: (links [V, 4, 3, 3] complex128, header info)."""
    info = GaugeInfo()
    _chk(lib().gmg_gauge_read_ildg(str(path).encode(), ctypes.byref(info), None))
    U = np.zeros((vol(tuple(info.dims)), 4, 3, 3), dtype=np.complex128)
    _chk(lib().gmg_gauge_read_ildg(str(path).encode(), ctypes.byref(info), U.ctypes.data_as(ctypes.c_void_p)))
    return U, info.as_dict()


def plaquette(dims, U):
    """(average plaquette, average link trace) of links on the host or the device, on the GPU."""
    p, t = ctypes.c_double(), ctypes.c_double()
    if isinstance(U, torch.Tensor) and U.is_cuda:
        _chk(lib().gmg_gauge_plaquette(_dims(dims), _ptr(U), 1, ctypes.byref(p), ctypes.byref(t), _stream()))
    else:
        U = np.ascontiguousarray(U, dtype=np.complex128)
        _chk(lib().gmg_gauge_plaquette(_dims(dims), U.ctypes.data_as(ctypes.c_void_p), 0, ctypes.byref(p),
                                       ctypes.byref(t), _stream()))
    return p.value, t.value


class MGParams(ctypes.Structure):
    _fields_ = [("nlevels", ctypes.c_int), ("block", (ctypes.c_int * 4) * 2), ("nvec", ctypes.c_int * 2),
                ("setup_iters", ctypes.c_int), ("smoother_iters", ctypes.c_int), ("wrapper_iters", ctypes.c_int),
                ("wrapper_tol", ctypes.c_double), ("coarsest_iters", ctypes.c_int), ("coarsest_tol", ctypes.c_double),
                ("coarsest_restart", ctypes.c_int), ("outer_restart", ctypes.c_int), ("prec", ctypes.c_int),
                ("seed", ctypes.c_uint64), ("setup_solver", ctypes.c_int), ("setup_tol", ctypes.c_double),
                ("setup_passes", ctypes.c_int), ("setup_null", ctypes.c_int), ("graph", ctypes.c_int),
                ("refine_iters", ctypes.c_int * 2), ("recursive_updates", ctypes.c_int),
                ("drop_in_cycle", ctypes.c_int), ("smoother_bf16", ctypes.c_int), ("outer_dcgs", ctypes.c_int),
                ("arnoldi_f32", ctypes.c_int)]


class MultiGrid:
    """MG-preconditioned FGMRES solve of the fine Wilson-clover operator (MultiGridPreconditioner)."""

    def __init__(self, fine, max_rhs, **params):
        p = MGParams()
        _chk(lib().gmg_mg_params_default(ctypes.byref(p)))
        for k, v in params.items():
            if k == "block":
                for i, blk in enumerate(v):
                    for d in range(4):
                        p.block[i][d] = blk[d]
            elif k in ("nvec", "refine_iters"):
                arr = getattr(p, k)
                for i, n in enumerate(v):
                    arr[i] = n
            elif k == "prec":
                p.prec = PREC.get(v, v)
            else:
                setattr(p, k, v)
        self.params = p
        self.fine = fine
        h = ctypes.c_void_p()
        _chk(lib().gmg_mg_create(fine._h, ctypes.byref(p), int(max_rhs), ctypes.byref(h)))
        self._h = h

    def __del__(self):
        if getattr(self, "_h", None) and _LIB is not None:
            _LIB.gmg_mg_destroy(self._h)
            self._h = None

    def setup(self):
        _chk(lib().gmg_mg_setup(self._h, _stream()))

    def refine(self):
        """refinementSetup: params.refine_iters passes per transition (see gmg_mg_refine)."""
        _chk(lib().gmg_mg_refine(self._h, _stream()))

    def graphs(self):
        """(captured K-cycle graphs, 1 if a capture failed and the host-driven cycle was kept)."""
        n, fb = ctypes.c_int(), ctypes.c_int()
        _chk(lib().gmg_mg_graphs(self._h, ctypes.byref(n), ctypes.byref(fb)))
        return n.value, fb.value

    def solve(self, b, x, tol=1e-10, maxiter=500):
        """b, x: complex128 CUDA tensors [V, nrhs, 12]; returns (outer iterations, max relative residual)."""
        _check_vec(b, self.fine.V, 12, "b")
        _check_vec(x, self.fine.V, 12, "x")
        it, rr = ctypes.c_int(), ctypes.c_double()
        _chk(lib().gmg_mg_solve(self._h, b.shape[1], _ptr(b), _ptr(x), ctypes.c_double(tol), int(maxiter),
                                ctypes.byref(it), ctypes.byref(rr), _stream()))
        return it.value, rr.value

    def apply(self, inp, out):
        """One K-cycle, out = M^-1 inp (MultiGridPreconditioner::operator()); complex128 CUDA
        tensors [V, nrhs, 12]."""
        _check_vec(inp, self.fine.V, 12, "inp")
        _check_vec(out, self.fine.V, 12, "out")
        _chk(lib().gmg_mg_apply(self._h, inp.shape[1], _ptr(inp), _ptr(out), _stream()))

    def solve_stats(self, nrhs):
        """Per-RHS (outer iteration at which its residual estimate met the tolerance, final true
        relative residual) of the last solve."""
        it = np.zeros(nrhs, dtype=np.int32)
        rr = np.zeros(nrhs, dtype=np.float64)
        _chk(lib().gmg_mg_solve_stats(self._h, int(nrhs), it.ctypes.data_as(ctypes.c_void_p),
                                      rr.ctypes.data_as(ctypes.c_void_p)))
        return it, rr

    def solve_batches(self):
        """Active-batch size of every outer Arnoldi step of the last solve."""
        n = ctypes.c_int()
        _chk(lib().gmg_mg_solve_batches(self._h, 0, None, ctypes.byref(n)))
        out = np.zeros(max(n.value, 1), dtype=np.int32)
        _chk(lib().gmg_mg_solve_batches(self._h, n.value, out.ctypes.data_as(ctypes.c_void_p), ctypes.byref(n)))
        return out[: n.value]

    def level(self, l):
        op, ag = ctypes.c_void_p(), ctypes.c_void_p()
        _chk(lib().gmg_mg_level(self._h, l, ctypes.byref(op), ctypes.byref(ag)))
        return op, ag


def chiral_double(vecs, factor=1.0):
    """Chirally doubled basis [2 nvec][V][dof] complex128 from vecs [V][nvec][dof]
    (complex128 or complex64 on the GPU): factor (1 + G5) v_n, then factor (1 - G5) v_n
    (performChiralDoublingG5C with factor 1/2, G5R5 with factor 1)."""
    V, nvec, dof = vecs.shape
    out = torch.empty((2 * nvec, V, dof), dtype=torch.complex128, device=vecs.device)
    _chk(lib().gmg_chiral_double(ctypes.c_int64(V), dof, nvec, _vec_prec(vecs), _ptr(vecs),
                                 ctypes.c_double(factor), _ptr(out), _stream()))
    return out


def lut_build(fine_dims, coarse_dims, mask_kind=-1):
    b = [f // c for f, c in zip(fine_dims, coarse_dims)]
    bv = int(np.prod(b))
    Vc, Vf = vol(coarse_dims), vol(fine_dims)
    l = np.zeros((Vc, bv), dtype=np.int32)
    s = np.zeros(Vc, dtype=np.int32)
    r = np.zeros(Vf, dtype=np.int32)
    _chk(lib().gmg_lut_build(_dims(fine_dims), _dims(coarse_dims), mask_kind, l.ctypes.data_as(ctypes.c_void_p),
                             s.ctypes.data_as(ctypes.c_void_p), r.ctypes.data_as(ctypes.c_void_p)))
    return l, s, r


def point_from_dir_disp(ndim, dirs_faster, d, disp):
    return lib().gmg_point_from_dir_disp(ndim, int(dirs_faster), d, disp)


def layout_vectors(vecs, ncs, inverse=False):
    """Device coarse vectors [..][N] (complex128 tensor) flat <-> Rework spin-split layout."""
    out = torch.empty_like(vecs)
    N = vecs.shape[-1]
    rows = vecs.numel() // N
    _chk(lib().gmg_layout_vectors(ctypes.c_int64(rows), N, ncs, _ptr(vecs), _ptr(out), int(inverse), _stream()))
    return out


def layout_links(links, ncs, inverse=False):
    """Device links [V][N][N] (complex128 tensor) flat <-> Rework spin-split layout."""
    out = torch.empty_like(links)
    N = links.shape[-1]
    V = links.numel() // (N * N)
    _chk(lib().gmg_layout_links(ctypes.c_int64(V), N, ncs, _ptr(links), _ptr(out), int(inverse), _stream()))
    return out

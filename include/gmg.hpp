// gmg.hpp -- C++ class surface of libgmg_b200 over the C ABI of gmg.h.
//
// Mirrors the reference's classes so that its multigrid driver code can be
// pointed at the GPU implementation:
//
//   gmg::CoarsenedMatrix      CoarsenedMatrix<Fobj,CComplex,nbasis>
//                             (include/CoarsenedMatrixUpstream.h:515-998):
//                             M, Mdag, Mdiag, Mdir, MdirAll, CoarsenOperator,
//                             ConstructRemainingLinks, public link access
//   gmg::Aggregation          Aggregation<Fobj,CComplex,nbasis>
//                             (...LutMRHS.h:293-352): Orthogonalise,
//                             CheckOrthogonal, ProjectToSubspace,
//                             PromoteFromSubspace, subspace set/get
//   gmg::WilsonCloverFermion  the fine matrix (Grid's WilsonCloverFermionR)
//   gmg::LinearOperatorBase   Op / AdjOp / HermOp / OpDiag / OpDir / OpDirAll
//   gmg::MdagMLinearOperator  Grid's MdagMLinearOperator<Matrix, Field> over any
//                             of the sparse matrices above
//   gmg::MultiGridPreconditioner
//                             MultiGridPreconditioner (include/MultigridPreconditioner.h:44-660):
//                             initialSetup, refinementSetup, and the outer
//                             FGMRES solve of Test_wilsonclover_mg[_mp].cc
//
// Fields are device buffers described by gmg::Field (pointer, sites, nrhs,
// dof, precision); the library never owns them.  Errors throw gmg::Error
// carrying the status and gmg_last_error() text (the reference aborts).
#pragma once

#include <array>
#include <stdexcept>
#include <string>
#include <vector>

#include "gmg.h"

namespace gmg {

class Error : public std::runtime_error {
 public:
  Error(gmg_status s, const std::string& what) : std::runtime_error(what), status(s) {}
  gmg_status status;
};

inline void check(gmg_status s) {
  if (s != GMG_OK) throw Error(s, gmg_last_error());
}

typedef std::array<int, 4> Coordinate;

// A caller-owned device field [sites][nrhs][dof], complex, F64 or F32.
struct Field {
  void* data = nullptr;
  long sites = 0;
  int nrhs = 1;
  int dof = 0;
  gmg_prec prec = GMG_F64;
  int checkerboard = -1;  // half fields: the parity of their sites (0 Even, 1 Odd), as Grid's Checkerboard()
};

// Grid's pickCheckerboard / setCheckerboard on device fields: full (V sites)
// <-> half (the V/2 sites of parity cb), see gmg_pick_checkerboard.
inline void PickCheckerboard(int cb, const std::array<int, 4>& dims, const Field& full, Field& half,
                             gmg_stream s = nullptr);
inline void SetCheckerboard(const std::array<int, 4>& dims, const Field& half, int cb, Field& full,
                            gmg_stream s = nullptr);

class LinearOperatorBase {
 public:
  virtual ~LinearOperatorBase() {}
  virtual void Op(const Field& in, Field& out) = 0;
  virtual void AdjOp(const Field& in, Field& out) = 0;
  virtual void OpDiag(const Field& in, Field& out) = 0;
  virtual void OpDir(const Field& in, Field& out, int dir, int disp) = 0;
  virtual void OpDirAll(const Field& in, std::vector<Field>& out) = 0;
  // HermOp = AdjOp(Op(in)); needs a temporary field of the same shape
  virtual void HermOp(const Field& in, Field& out, Field& tmp) {
    Op(in, tmp);
    AdjOp(tmp, out);
  }
};

class CoarsenedMatrix {
 public:
  CoarsenedMatrix(const Coordinate& coarse_dims, int nbasis, int hermitian = 0, gmg_stream s = nullptr)
      : dims_(coarse_dims), nbasis_(nbasis), hermitian_(hermitian), stream_(s) {
    check(gmg_coarse_create(dims_.data(), nbasis, hermitian, &h_));
  }
  ~CoarsenedMatrix() { gmg_coarse_destroy(h_); }
  CoarsenedMatrix(const CoarsenedMatrix&) = delete;
  CoarsenedMatrix& operator=(const CoarsenedMatrix&) = delete;

  gmg_coarse* handle() const { return h_; }
  int nbasis() const { return nbasis_; }
  const Coordinate& Grid() const { return dims_; }

  // the public A[p] link fields, [9][V][N][N] complex128
  void SetLinks(const double* links, bool on_device) { check(gmg_coarse_set_links(h_, links, on_device, stream_)); }
  void GetLinks(double* links, bool on_device) { check(gmg_coarse_get_links(h_, links, on_device, stream_)); }
  void Prepare(gmg_prec compute) { check(gmg_coarse_prepare(h_, compute, stream_)); }
  void SetCompute(gmg_prec compute) { compute_ = compute; }

  void M(const Field& in, Field& out) { apply(GMG_OP_M, 8, in, out); }
  void Mdag(const Field& in, Field& out) { apply(GMG_OP_MDAG, 8, in, out); }
  void Mdiag(const Field& in, Field& out) { apply(GMG_OP_MDIAG, 8, in, out); }
  void Mdir(const Field& in, Field& out, int dir, int disp) {
    const int p = gmg_point_from_dir_disp(4, 1, dir, disp);
    if (p < 0) throw Error(GMG_ERR_ARGUMENT, "Mdir: bad direction / displacement");
    apply(GMG_OP_MDIR, p, in, out);
  }
  void MdirAll(const Field& in, std::vector<Field>& out) {
    if (out.size() != 8 && out.size() != 9) throw Error(GMG_ERR_ARGUMENT, "MdirAll: need 8 outputs");
    void* o[8];
    for (int p = 0; p < 8; ++p) o[p] = out[p].data;
    check(gmg_coarse_mdir_all(h_, compute_or(in), in.prec, in.nrhs, in.data, o, stream_));
  }
  // restrict to a subset of RHS slots (device int32 list)
  void MActive(const Field& in, Field& out, const int32_t* active, int n_active) {
    check(gmg_coarse_apply(h_, GMG_OP_M, 8, compute_or(in), in.prec, in.nrhs, in.data, out.data, active,
                           n_active, stream_));
  }

  void ConstructRemainingLinks() { check(gmg_coarse_construct_remaining_links(h_, stream_)); }

  // Red-black (Schur) interface of Rework::CoarsenedMatrix (CoarsenedMatrixRework.h:178-245).
  // Half fields hold V/2 sites of one parity; `cb` is the parity of `in`
  // (Grid's in.Checkerboard()), 0 = Even, 1 = Odd.
  int ConstEE() const { return 0; }
  void InvertSelfStencilPoint() { check(gmg_coarse_invert_self(h_, stream_)); }
  void Dhop(const Field& in, Field& out, int dag) {
    check(gmg_coarse_dhop(h_, dag, compute_or(in), in.prec, in.nrhs, in.data, out.data, stream_));
  }
  void Meooe(const Field& in, Field& out, int cb) { rb(GMG_RB_MEOOE, cb, in, out); }
  void MeooeDag(const Field& in, Field& out, int cb) { rb(GMG_RB_MEOOE_DAG, cb, in, out); }
  void DhopOE(const Field& in_even, Field& out_odd, int dag) { rb(dag ? GMG_RB_MEOOE_DAG : GMG_RB_MEOOE, 0, in_even, out_odd); }
  void DhopEO(const Field& in_odd, Field& out_even, int dag) { rb(dag ? GMG_RB_MEOOE_DAG : GMG_RB_MEOOE, 1, in_odd, out_even); }
  void Mooee(const Field& in, Field& out, int cb) { rb(GMG_RB_MOOEE, cb, in, out); }
  void MooeeDag(const Field& in, Field& out, int cb) { rb(GMG_RB_MOOEE_DAG, cb, in, out); }
  void MooeeInv(const Field& in, Field& out, int cb) { rb(GMG_RB_MOOEE_INV, cb, in, out); }
  void MooeeInvDag(const Field& in, Field& out, int cb) { rb(GMG_RB_MOOEE_INV_DAG, cb, in, out); }
  // the full-grid forms of the self-point family
  void Mooee(const Field& in, Field& out) { mooee(GMG_RB_MOOEE, in, out); }
  void MooeeDag(const Field& in, Field& out) { mooee(GMG_RB_MOOEE_DAG, in, out); }
  void MooeeInv(const Field& in, Field& out) { mooee(GMG_RB_MOOEE_INV, in, out); }
  void MooeeInvDag(const Field& in, Field& out) { mooee(GMG_RB_MOOEE_INV_DAG, in, out); }

  // CoarsenOperator(FineGrid, linop, Subspace)
  inline void CoarsenOperator(class Aggregation& agg, class WilsonCloverFermion& fine);
  inline void CoarsenOperator(class Aggregation& agg, CoarsenedMatrix& fine);

 private:
  gmg_prec compute_or(const Field& in) const { return compute_ == (gmg_prec)-1 ? in.prec : compute_; }
  void rb(gmg_rb_op op, int cb, const Field& in, Field& out) {
    check(gmg_coarse_apply_rb(h_, op, cb, compute_or(in), in.prec, in.nrhs, in.data, out.data, stream_));
  }
  void mooee(gmg_rb_op op, const Field& in, Field& out) {
    check(gmg_coarse_mooee(h_, op, compute_or(in), in.prec, in.nrhs, in.data, out.data, stream_));
  }
  void apply(gmg_op op, int point, const Field& in, Field& out) {
    check(gmg_coarse_apply(h_, op, point, compute_or(in), in.prec, in.nrhs, in.data, out.data, nullptr, 0,
                           stream_));
  }
  Coordinate dims_;
  int nbasis_, hermitian_;
  gmg_stream stream_;
  gmg_prec compute_ = (gmg_prec)-1;
  gmg_coarse* h_ = nullptr;
};

class Aggregation {
 public:
  Aggregation(const Coordinate& coarse_dims, const Coordinate& fine_dims, int site_dof, int nbasis,
              gmg_stream s = nullptr)
      : stream_(s) {
    check(gmg_agg_create(fine_dims.data(), coarse_dims.data(), site_dof, nbasis, &h_));
  }
  ~Aggregation() { gmg_agg_destroy(h_); }
  Aggregation(const Aggregation&) = delete;
  Aggregation& operator=(const Aggregation&) = delete;
  gmg_agg* handle() const { return h_; }

  void SetSubspace(const double* basis, bool on_device) { check(gmg_agg_set_basis(h_, basis, on_device, stream_)); }
  void GetSubspace(double* basis, bool on_device) { check(gmg_agg_get_basis(h_, basis, on_device, stream_)); }
  void Orthogonalise(int checkOrthogonality = 1, int passes = 2) {
    check(gmg_agg_orthonormalise(h_, passes, stream_));
    if (checkOrthogonality) CheckOrthogonal();
  }
  double CheckOrthogonal() {
    double e = 0;
    check(gmg_agg_check_orthogonal(h_, &e, stream_));
    return e;
  }
  void ProjectToSubspace(Field& coarse, const Field& fine) {
    check(gmg_agg_project(h_, fine.prec, fine.prec, fine.nrhs, fine.data, coarse.data, stream_));
  }
  void PromoteFromSubspace(const Field& coarse, Field& fine) {
    check(gmg_agg_promote(h_, fine.prec, fine.prec, coarse.nrhs, coarse.data, fine.data, stream_));
  }

 private:
  gmg_stream stream_;
  gmg_agg* h_ = nullptr;
};

class WilsonCloverFermion {
 public:
  WilsonCloverFermion(const Coordinate& dims, double mass, double csw, bool antiperiodic_t,
                      gmg_stream s = nullptr)
      : stream_(s) {
    check(gmg_wilson_create(dims.data(), mass, csw, antiperiodic_t, &h_));
  }
  ~WilsonCloverFermion() { gmg_wilson_destroy(h_); }
  WilsonCloverFermion(const WilsonCloverFermion&) = delete;
  WilsonCloverFermion& operator=(const WilsonCloverFermion&) = delete;
  gmg_wilson* handle() const { return h_; }

  void ImportGauge(const double* U, bool on_device) { check(gmg_wilson_set_gauge(h_, U, on_device, stream_)); }
  void M(const Field& in, Field& out) { apply(GMG_OP_M, 0, 0, in, out); }
  void Mdag(const Field& in, Field& out) { apply(GMG_OP_MDAG, 0, 0, in, out); }
  void Mdiag(const Field& in, Field& out) { apply(GMG_OP_MDIAG, 0, 0, in, out); }
  void Mdir(const Field& in, Field& out, int dir, int disp) { apply(GMG_OP_MDIR, dir, disp, in, out); }
  void MdirAll(const Field& in, std::vector<Field>& out) {
    for (int p = 0; p < 8; ++p) Mdir(in, out[p], p % 4, p < 4 ? 1 : -1);
  }

 private:
  void apply(gmg_op op, int dir, int disp, const Field& in, Field& out) {
    check(gmg_wilson_apply(h_, op, dir, disp, in.prec, in.nrhs, in.data, out.data, stream_));
  }
  gmg_stream stream_;
  gmg_wilson* h_ = nullptr;
};

inline void CoarsenedMatrix::CoarsenOperator(Aggregation& agg, WilsonCloverFermion& fine) {
  check(gmg_coarsen_wilson(h_, agg.handle(), fine.handle(), stream_));
}
inline void CoarsenedMatrix::CoarsenOperator(Aggregation& agg, CoarsenedMatrix& fine) {
  check(gmg_coarsen_coarse(h_, agg.handle(), fine.handle(), stream_));
}

// Grid's MdagMLinearOperator<Matrix, Field>: Op -> M, AdjOp -> Mdag,
// OpDiag -> Mdiag, OpDir -> Mdir, OpDirAll -> MdirAll.
template <class Matrix>
class MdagMLinearOperator : public LinearOperatorBase {
 public:
  explicit MdagMLinearOperator(Matrix& m) : m_(m) {}
  Matrix& matrix() { return m_; }
  void Op(const Field& in, Field& out) override { m_.M(in, out); }
  void AdjOp(const Field& in, Field& out) override { m_.Mdag(in, out); }
  void OpDiag(const Field& in, Field& out) override { m_.Mdiag(in, out); }
  void OpDir(const Field& in, Field& out, int dir, int disp) override { m_.Mdir(in, out, dir, disp); }
  void OpDirAll(const Field& in, std::vector<Field>& out) override { m_.MdirAll(in, out); }

 private:
  Matrix& m_;
};

// The multigrid hierarchy over the fine Wilson-clover matrix.  Parameters
// are MultiGridParams (MultigridParams.h:95-113) as gmg_mg_params; Params()
// gives the defaults.  Solve() runs the FP64 outer FGMRES preconditioned by
// the K-cycle on device fields [V][nrhs][12] (F64) and returns the outer
// iteration count.
class MultiGridPreconditioner {
 public:
  static gmg_mg_params Params() {
    gmg_mg_params p;
    check(gmg_mg_params_default(&p));
    return p;
  }
  MultiGridPreconditioner(WilsonCloverFermion& fine, const gmg_mg_params& p, int max_rhs, gmg_stream s = nullptr)
      : stream_(s) {
    check(gmg_mg_create(fine.handle(), &p, max_rhs, &h_));
  }
  ~MultiGridPreconditioner() { gmg_mg_destroy(h_); }
  MultiGridPreconditioner(const MultiGridPreconditioner&) = delete;
  MultiGridPreconditioner& operator=(const MultiGridPreconditioner&) = delete;
  gmg_mg* handle() const { return h_; }

  void initialSetup() { check(gmg_mg_setup(h_, stream_)); }
  void refinementSetup() { check(gmg_mg_refine(h_, stream_)); }
  // one K-cycle: out = M^-1 in (F64 fields)
  void operator()(const Field& in, Field& out) {
    check(gmg_mg_apply(h_, in.nrhs, static_cast<const double*>(in.data), static_cast<double*>(out.data), stream_));
  }
  int Solve(const Field& b, Field& x, double tol, int maxiter, double* max_relres = nullptr) {
    int it = 0;
    double rr = 0;
    check(gmg_mg_solve(h_, b.nrhs, static_cast<const double*>(b.data), static_cast<double*>(x.data), tol, maxiter,
                       &it, &rr, stream_));
    if (max_relres) *max_relres = rr;
    return it;
  }
  // the coarse operator of level > 0 and the aggregation from level to level+1
  // (owned by the hierarchy)
  gmg_coarse* CoarseMatrix(int level) {
    gmg_coarse* op = nullptr;
    check(gmg_mg_level(h_, level, &op, nullptr));
    return op;
  }
  gmg_agg* Aggregates(int level) {
    gmg_agg* agg = nullptr;
    check(gmg_mg_level(h_, level, nullptr, &agg));
    return agg;
  }

 private:
  gmg_stream stream_;
  gmg_mg* h_ = nullptr;
};

inline void PickCheckerboard(int cb, const std::array<int, 4>& dims, const Field& full, Field& half, gmg_stream s) {
  check(gmg_pick_checkerboard(dims.data(), cb, full.nrhs * full.dof, full.prec, full.data, half.data, s));
}
inline void SetCheckerboard(const std::array<int, 4>& dims, const Field& half, int cb, Field& full, gmg_stream s) {
  check(gmg_set_checkerboard(dims.data(), cb, half.nrhs * half.dof, half.prec, half.data, full.data, s));
}

}  // namespace gmg

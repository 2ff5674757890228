// gmg_rework.hpp -- the Rework class surface of libgmg_b200: the policy-typed
// two-spin coarse operator and aggregation of grid-mg-bench's buildable
// multigrid path (MultigridPreconditioner.h:88-95, 150-154 with
// USE_NEW_COARSENING), over the C ABI of gmg.h.
//
//   gmg::Rework::CoarseningPolicy<Ns_f, Nc_f, Nbasis, Ncoarse_spins>
//       CoarseningPolicy<FineFermionField, Nbasis, Ncoarse_spins>
//       (include/CoarseningPolicyRework.h:56-109): the compile-time sizes
//   gmg::Rework::Aggregation<Policy>
//       Aggregation<Policy> (include/AggregationRework.h:43-146): Subspace,
//       Create(basis vectors), Orthogonalise, CheckOrthogonal,
//       ProjectToSubspace / PromoteFromSubspace, UseFastProjects
//   gmg::Rework::CoarsenedMatrix<Policy>
//       CoarsenedMatrix<Policy> (include/CoarsenedMatrixRework.h:43-680):
//       the (Grid, RBGrid, speedLevel, hermitian) constructor, M, Mdag,
//       Mdiag, Mdir, Meooe[Dag], Mooee[Inv][Dag], Dhop, DhopOE / DhopEO,
//       DhopDir, ConstEE, CoarsenOperator (which ends with the self-link
//       inverse, as the reference's InvertSelfStencilPoint), and the link
//       fields Y_[p] in their [Ns_c][Ns_c][Nc_c][Nc_c] block form
//
// The library stores the Rework coarse space as the Upstream one with
// nbasis = Ns_c * Nc_c and flat index n = s * Nc_c + c (the chirally doubled
// basis; see gmg_agg_set_subspace_spins), so a Rework coarse field
// [sites][nrhs][Ns_c][Nc_c] is the same memory as the flat field and every
// operator call goes to the same kernels.  The reference's speed levels
// (0 / 1 / 2) select implementations of CoarsenOperator that it asserts give
// equal links (src/Benchmark_create_coarse_operator.cc:355-467); here there is
// one implementation, and SpeedLevel() returns the level the object was made
// with.  The fast / slow projection switch (UseFastProjects) is recorded the
// same way.  Red-black fields carry their parity in Field::checkerboard
// (0 Even, 1 Odd), which Meooe / Mooee read and set like Grid's
// Checkerboard().
#pragma once

#include <cuda_runtime.h>

#include "gmg.hpp"

namespace gmg {
namespace Rework {

template <int Ns_f_, int Nc_f_, int Nbasis_, int Ncoarse_spins_>
struct CoarseningPolicy {
  static constexpr int Ns_f = Ns_f_;   // fine spins (4 for Wilson, 2 for a coarse fine level)
  static constexpr int Nc_f = Nc_f_;   // fine colours (3, or the basis size of the level above)
  static constexpr int Ns_c = Ncoarse_spins_;
  static constexpr int Nc_c = Nbasis_;
  static constexpr int Ns_b = Ns_f / Ns_c;  // spin blocking
  static constexpr int FineDof = Ns_f * Nc_f;
  static constexpr int CoarseDof = Ns_c * Nc_c;  // the flat nbasis of the library
  static_assert(Ns_f >= Ns_c, "Number of spin dofs incorrect");
  static_assert(Ns_f % Ns_c == 0, "coarse spins must block the fine spins evenly");
};

// Wilson-clover fine fields (4 spins x 3 colours) coarsened with two spins
template <int Nbasis>
using WilsonTwoSpinPolicy = CoarseningPolicy<4, 3, Nbasis, 2>;

template <class Policy>
class Aggregation {
 public:
  static constexpr int Ns_c = Policy::Ns_c, Nc_c = Policy::Nc_c;

  // Aggregation(CoarseGrid, FineGrid, CheckerBoard, UseFastProjects) (AggregationRework.h:64-73)
  Aggregation(const Coordinate& coarse_dims, const Coordinate& fine_dims, int checkerboard = 0,
              int use_fast_projects = 0, gmg_stream s = nullptr)
      : coarse_(coarse_dims), fine_(fine_dims), cb_(checkerboard), fast_(use_fast_projects), stream_(s) {
    check(gmg_agg_create(fine_dims.data(), coarse_dims.data(), Policy::FineDof, Policy::CoarseDof, &h_));
  }
  ~Aggregation() { gmg_agg_destroy(h_); }
  Aggregation(const Aggregation&) = delete;
  Aggregation& operator=(const Aggregation&) = delete;
  gmg_agg* handle() const { return h_; }
  const Coordinate& CoarseGrid() const { return coarse_; }
  const Coordinate& FineGrid() const { return fine_; }
  int CheckerBoard() const { return cb_; }

  void UseFastProjects(bool yes) { fast_ = yes; }
  bool FastProjects() const { return fast_; }

  // Subspace(): the Nc_c vectors [Nc_c][Vf][FineDof] complex128 (copied out / in)
  void GetSubspace(double* vecs, bool on_device) {
    check(gmg_agg_get_subspace_spins(h_, Ns_c, vecs, on_device, stream_));
  }
  void SetSubspace(const double* vecs, bool on_device) {
    check(gmg_agg_set_subspace_spins(h_, Ns_c, vecs, on_device, stream_));
  }

  // Orthogonalise(checkOrthogonality, passes): per block and coarse spin
  // (aggregateOrthogonalise, AggregationKernelsRework.h:266-341); the spins
  // have disjoint supports, so this is the flat basis's block orthonormalisation
  double Orthogonalise(int checkOrthogonality = 1, int passes = 2) {
    check(gmg_agg_orthonormalise(h_, passes, stream_));
    return checkOrthogonality ? CheckOrthogonal() : 0.0;
  }
  // max over blocks of |B^dag B - 1| (the reference prints the norm of R v_i - e_i per i)
  double CheckOrthogonal() {
    double e = 0;
    check(gmg_agg_check_orthogonal(h_, &e, stream_));
    return e;
  }

  // Create(MGBasisVectors) (:127-146): copy the Nc_c basis vectors in and orthogonalise
  double Create(const double* basis_vectors, bool on_device) {
    SetSubspace(basis_vectors, on_device);
    return Orthogonalise();
  }

  // coarse [Vc][nrhs][Ns_c][Nc_c], fine [Vf][nrhs][FineDof]
  void ProjectToSubspace(Field& coarse, const Field& fine) const {
    check(gmg_agg_project(h_, fine.prec, fine.prec, fine.nrhs, fine.data, coarse.data, stream_));
  }
  void PromoteFromSubspace(const Field& coarse, Field& fine) const {
    check(gmg_agg_promote(h_, fine.prec, fine.prec, coarse.nrhs, coarse.data, fine.data, stream_));
  }

 private:
  Coordinate coarse_, fine_;
  int cb_;
  bool fast_;
  gmg_stream stream_;
  gmg_agg* h_ = nullptr;
};

template <class Policy>
class CoarsenedMatrix {
 public:
  static constexpr int Ns_c = Policy::Ns_c, Nc_c = Policy::Nc_c;

  // CoarsenedMatrix(CoarseGrid, CoarseRBGrid, speedLevel, hermitian) (CoarsenedMatrixRework.h:82-101).
  // rb_dims is the checkerboarded grid: the coarse extents with x halved.
  CoarsenedMatrix(const Coordinate& coarse_dims, const Coordinate& rb_dims, int speedLevel = 0, int hermitian = 0,
                  gmg_stream s = nullptr)
      : dims_(coarse_dims), rb_(rb_dims), speed_(speedLevel), stream_(s) {
    if (rb_dims[0] * 2 != coarse_dims[0] || rb_dims[1] != coarse_dims[1] || rb_dims[2] != coarse_dims[2] ||
        rb_dims[3] != coarse_dims[3])
      throw Error(GMG_ERR_SHAPE, "Rework::CoarsenedMatrix: the red-black grid must be the grid with x halved");
    check(gmg_coarse_create(dims_.data(), Policy::CoarseDof, hermitian, &h_));
  }
  ~CoarsenedMatrix() { gmg_coarse_destroy(h_); }
  CoarsenedMatrix(const CoarsenedMatrix&) = delete;
  CoarsenedMatrix& operator=(const CoarsenedMatrix&) = delete;
  gmg_coarse* handle() const { return h_; }

  const Coordinate& Grid() const { return dims_; }
  const Coordinate& RedBlackGrid() const { return rb_; }
  int ConstEE() const { return 0; }
  int SpeedLevel() const { return speed_; }
  void SetCompute(gmg_prec compute) { compute_ = compute; }
  void Prepare(gmg_prec compute) { check(gmg_coarse_prepare(h_, compute, stream_)); }

  // the link fields Y_[p], [V][Ns_c][Ns_c][Nc_c][Nc_c] complex128 per point (all 9 for Set)
  void GetLinks(int point, double* links, bool on_device) {
    check(gmg_coarse_get_links_spins(h_, Ns_c, point, links, on_device, stream_));
  }
  void SetLinks(const double* links9, bool on_device) {
    check(gmg_coarse_set_links_spins(h_, Ns_c, links9, on_device, stream_));
  }

  void M(const Field& in, Field& out) { apply(GMG_OP_M, 8, in, out); }
  void Mdag(const Field& in, Field& out) { apply(GMG_OP_MDAG, 8, in, out); }
  void Mdiag(const Field& in, Field& out) { Mooee(in, out); }
  void Mdir(const Field& in, Field& out, int dir, int disp) { DhopDir(in, out, dir, disp); }
  void DhopDir(const Field& in, Field& out, int dir, int disp) {
    const int p = gmg_point_from_dir_disp(4, 1, dir, disp);
    if (p < 0 || p == 8) throw Error(GMG_ERR_ARGUMENT, "DhopDir: bad direction / displacement");
    apply(GMG_OP_MDIR, p, in, out);
  }
  void MdirAll(const Field& in, std::vector<Field>& out) {
    if (out.size() < 8) throw Error(GMG_ERR_ARGUMENT, "MdirAll: need 8 outputs");
    void* o[8];
    for (int p = 0; p < 8; ++p) o[p] = out[p].data;
    check(gmg_coarse_mdir_all(h_, compute_or(in), in.prec, in.nrhs, in.data, o, stream_));
  }

  // full-grid hopping term and self-point family
  void Dhop(const Field& in, Field& out, int dag) {
    check(gmg_coarse_dhop(h_, dag, compute_or(in), in.prec, in.nrhs, in.data, out.data, stream_));
    out.checkerboard = in.checkerboard;
  }
  void Mooee(const Field& in, Field& out) { self(GMG_RB_MOOEE, in, out); }
  void MooeeDag(const Field& in, Field& out) { self(GMG_RB_MOOEE_DAG, in, out); }
  void MooeeInv(const Field& in, Field& out) { self(GMG_RB_MOOEE_INV, in, out); }
  void MooeeInvDag(const Field& in, Field& out) { self(GMG_RB_MOOEE_INV_DAG, in, out); }

  // red-black: in.checkerboard selects DhopEO (Odd in) or DhopOE (Even in)
  void Meooe(const Field& in, Field& out) { hop(GMG_RB_MEOOE, in, out); }
  void MeooeDag(const Field& in, Field& out) { hop(GMG_RB_MEOOE_DAG, in, out); }
  void DhopOE(const Field& in, Field& out, int dag) {
    if (in.checkerboard != 0) throw Error(GMG_ERR_ARGUMENT, "DhopOE: input must be on the Even checkerboard");
    hop(dag ? GMG_RB_MEOOE_DAG : GMG_RB_MEOOE, in, out);
  }
  void DhopEO(const Field& in, Field& out, int dag) {
    if (in.checkerboard != 1) throw Error(GMG_ERR_ARGUMENT, "DhopEO: input must be on the Odd checkerboard");
    hop(dag ? GMG_RB_MEOOE_DAG : GMG_RB_MEOOE, in, out);
  }

  // CoarsenOperator(FineGrid, LinOp, Projector) (CoarsenedMatrixRework.h:401-611):
  // the Galerkin links, then the self-link inverse the red-black operators use
  void CoarsenOperator(const Coordinate& fine_grid, MdagMLinearOperator<WilsonCloverFermion>& linop,
                       Aggregation<Policy>& projector) {
    same_fine(fine_grid, projector);
    check(gmg_coarsen_wilson(h_, projector.handle(), linop.matrix().handle(), stream_));
    InvertSelfStencilPoint();
  }
  template <class FinePolicy>
  void CoarsenOperator(const Coordinate& fine_grid, MdagMLinearOperator<CoarsenedMatrix<FinePolicy>>& linop,
                       Aggregation<Policy>& projector) {
    same_fine(fine_grid, projector);
    check(gmg_coarsen_coarse(h_, projector.handle(), linop.matrix().handle(), stream_));
    InvertSelfStencilPoint();
  }
  void InvertSelfStencilPoint() { check(gmg_coarse_invert_self(h_, stream_)); }

 private:
  gmg_prec compute_or(const Field& in) const { return compute_ == (gmg_prec)-1 ? in.prec : compute_; }
  void apply(gmg_op op, int point, const Field& in, Field& out) {
    check(gmg_coarse_apply(h_, op, point, compute_or(in), in.prec, in.nrhs, in.data, out.data, nullptr, 0,
                           stream_));
    out.checkerboard = in.checkerboard;
  }
  void self(gmg_rb_op op, const Field& in, Field& out) {
    const Coordinate& d = dims_;
    const long V = (long)d[0] * d[1] * d[2] * d[3];
    if (in.sites == V) {
      check(gmg_coarse_mooee(h_, op, compute_or(in), in.prec, in.nrhs, in.data, out.data, stream_));
    } else {
      if (in.checkerboard != 0 && in.checkerboard != 1)
        throw Error(GMG_ERR_ARGUMENT, "Mooee: a half field needs its checkerboard (0 Even, 1 Odd)");
      check(gmg_coarse_apply_rb(h_, op, in.checkerboard, compute_or(in), in.prec, in.nrhs, in.data, out.data,
                                stream_));
    }
    out.checkerboard = in.checkerboard;
  }
  void hop(gmg_rb_op op, const Field& in, Field& out) {
    if (in.checkerboard != 0 && in.checkerboard != 1)
      throw Error(GMG_ERR_ARGUMENT, "Meooe: the input needs its checkerboard (0 Even, 1 Odd)");
    check(gmg_coarse_apply_rb(h_, op, in.checkerboard, compute_or(in), in.prec, in.nrhs, in.data, out.data,
                              stream_));
    out.checkerboard = 1 - in.checkerboard;
  }
  void same_fine(const Coordinate& fine_grid, const Aggregation<Policy>& projector) const {
    if (fine_grid != projector.FineGrid())
      throw Error(GMG_ERR_SHAPE, "CoarsenOperator: the fine grid differs from the aggregation's");
  }
  Coordinate dims_, rb_;
  int speed_;
  gmg_stream stream_;
  gmg_prec compute_ = (gmg_prec)-1;
  gmg_coarse* h_ = nullptr;
};

}  // namespace Rework
}  // namespace gmg

// surface_check.cpp -- exercises the C++ class surface (include/gmg.hpp) the way
// the reference's drivers use CoarsenedMatrix / Aggregation / linear operators.
//
// Restates the MG correctness checks of MultiGridPreconditioner::runChecks
// (include/MultigridPreconditioner.h:311-446) on the GPU implementation:
//   (1) 0 == (M - (Mdiag + sum_mu Mdir_mu)) v          fine operator
//   (2) 0 == (1 - P R) v_i                              basis vectors
//   (3) 0 == (1 - R P) v_c
//   (4) 0 == (R D P - D_c) v_c                           Galerkin identity
//   (5) 0 == Im(v_c^dag D_c^dag D_c v_c)                 Mdag is the adjoint
// and the red-black identities of src/Test_coarse_red_black.cc:170-482:
//   (6) M = Dhop + Mdiag   (7) MooeeInv Mooee = 1   (8) M = Meo + Moe + Mee + Moo
// and the MG driver of src/Test_wilsonclover_mg.cc:115-140 (initialSetup,
// refinementSetup, outer FGMRES):
//   (9) |b - D x| / |b| of the solve after the refinement setup
//   (10) (R D P - D_c) v_c on the operators the refinement rebuilt
// and the Rework (two-spin, policy-typed) surface of include/gmg_rework.hpp the
// way src/Benchmark_create_coarse_operator.cc:355-467 checks it:
//   (11) the Upstream subspace with its chiral doubling undone, copied into the
//        two-spin aggregation, comes back unchanged and orthonormal
//   (12) Y_[p] of the two-spin CoarsenOperator against A[p] of the Upstream
//        one through the layout map (convertLayout), every point
//   (13) the two-spin M / Mdag / Meooe / MooeeInv Mooee on the same coarse fields
//   (14) Create(basis vectors) gives an orthonormal two-spin subspace
// Prints one line per check and exits non-zero if any check fails.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdio>
#include <random>
#include <vector>

#include "gmg_rework.hpp"

typedef std::complex<double> cplx;

struct DevField {
  gmg::Field f;
  DevField(long sites, int nrhs, int dof) {
    f.sites = sites;
    f.nrhs = nrhs;
    f.dof = dof;
    f.prec = GMG_F64;
    cudaMalloc(&f.data, bytes());
    cudaMemset(f.data, 0, bytes());
  }
  ~DevField() { cudaFree(f.data); }
  size_t bytes() const { return sizeof(cplx) * f.sites * f.nrhs * f.dof; }
  std::vector<cplx> get() const {
    std::vector<cplx> h(f.sites * f.nrhs * f.dof);
    cudaMemcpy(h.data(), f.data, bytes(), cudaMemcpyDeviceToHost);
    return h;
  }
  void set(const std::vector<cplx>& h) { cudaMemcpy(f.data, h.data(), bytes(), cudaMemcpyHostToDevice); }
};

static std::vector<cplx> gaussian(size_t n, std::mt19937_64& g) {
  std::normal_distribution<double> d(0.0, std::sqrt(0.5));
  std::vector<cplx> v(n);
  for (auto& x : v) x = cplx(d(g), d(g));
  return v;
}

static double rel_dev(const std::vector<cplx>& a, const std::vector<cplx>& b) {
  double num = 0, den = 0;
  for (size_t i = 0; i < a.size(); ++i) {
    num += std::norm(a[i] - b[i]);
    den += std::norm(a[i]);
  }
  return std::sqrt(num / den);
}

static bool report(const char* name, double dev, double tol) {
  const bool ok = dev < tol;
  std::printf("%-44s deviation %.3e  (tol %.0e)  %s\n", name, dev, tol, ok ? "passed" : "FAILED");
  return ok;
}

int main() {
  const gmg::Coordinate fdims{8, 8, 8, 8}, cdims{2, 2, 2, 2};
  const long Vf = 4096, Vc = 16;
  const int nb = 4, N = 2 * nb;
  std::mt19937_64 gen(1234);

  // random unitary gauge links (Gram-Schmidt of Gaussian 3x3 matrices)
  std::vector<cplx> U(Vf * 4 * 9);
  for (long l = 0; l < Vf * 4; ++l) {
    auto m = gaussian(9, gen);
    for (int r = 0; r < 3; ++r) {
      for (int q = 0; q < r; ++q) {
        cplx d = 0;
        for (int c = 0; c < 3; ++c) d += std::conj(m[q * 3 + c]) * m[r * 3 + c];
        for (int c = 0; c < 3; ++c) m[r * 3 + c] -= d * m[q * 3 + c];
      }
      double n = 0;
      for (int c = 0; c < 3; ++c) n += std::norm(m[r * 3 + c]);
      for (int c = 0; c < 3; ++c) m[r * 3 + c] /= std::sqrt(n);
    }
    for (int k = 0; k < 9; ++k) U[l * 9 + k] = m[k];
  }

  bool ok = true;
  try {
    gmg::WilsonCloverFermion D(fdims, -0.2, 1.0, true);
    D.ImportGauge(reinterpret_cast<const double*>(U.data()), false);
    gmg::MdagMLinearOperator<gmg::WilsonCloverFermion> FineOp(D);

    // (1) M = Mdiag + sum Mdir
    DevField v(Vf, 1, 12), Mv(Vf, 1, 12), t(Vf, 1, 12);
    v.set(gaussian(Vf * 12, gen));
    FineOp.Op(v.f, Mv.f);
    FineOp.OpDiag(v.f, t.f);
    std::vector<cplx> acc = t.get();
    for (int dir = 0; dir < 4; ++dir)
      for (int disp : {+1, -1}) {
        FineOp.OpDir(v.f, t.f, dir, disp);
        auto h = t.get();
        for (size_t i = 0; i < acc.size(); ++i) acc[i] += h[i];
      }
    ok &= report("M - (Mdiag + sum Mdir)", rel_dev(Mv.get(), acc), 1e-13);

    // basis: nb Gaussian vectors, chirally doubled (G5C, factor 1/2), block-orthonormalised
    std::vector<cplx> B(N * Vf * 12);
    auto h = gaussian(nb * Vf * 12, gen);
    for (int n = 0; n < nb; ++n)
      for (long s = 0; s < Vf; ++s)
        for (int a = 0; a < 12; ++a) {
          const cplx x = h[(n * Vf + s) * 12 + a];
          B[(n * Vf + s) * 12 + a] = a < 6 ? x : 0.0;
          B[((n + nb) * Vf + s) * 12 + a] = a < 6 ? 0.0 : x;
        }
    gmg::Aggregation Aggs(cdims, fdims, 12, N);
    Aggs.SetSubspace(reinterpret_cast<const double*>(B.data()), false);
    Aggs.Orthogonalise(0, 1);
    ok &= report("CheckOrthogonal max |B^dag B - 1|", Aggs.CheckOrthogonal(), 1e-13);

    gmg::CoarsenedMatrix Dc(cdims, N, 0);
    Dc.CoarsenOperator(Aggs, D);
    gmg::MdagMLinearOperator<gmg::CoarsenedMatrix> CoarseOp(Dc);

    // (2) (1 - P R) v_i for the first basis vector
    std::vector<cplx> Bo(N * Vf * 12);
    Aggs.GetSubspace(reinterpret_cast<double*>(Bo.data()), false);
    DevField vi(Vf, 1, 12), back(Vf, 1, 12);
    DevField c(Vc, 1, N), c2(Vc, 1, N), c3(Vc, 1, N);
    vi.set(std::vector<cplx>(Bo.begin(), Bo.begin() + Vf * 12));
    Aggs.ProjectToSubspace(c.f, vi.f);
    Aggs.PromoteFromSubspace(c.f, back.f);
    ok &= report("(1 - P R) v_0", rel_dev(vi.get(), back.get()), 1e-13);

    // (3) (1 - R P) v_c
    c.set(gaussian(Vc * N, gen));
    Aggs.PromoteFromSubspace(c.f, back.f);
    Aggs.ProjectToSubspace(c2.f, back.f);
    ok &= report("(1 - R P) v_c", rel_dev(c.get(), c2.get()), 1e-13);

    // (4) (R D P - D_c) v_c
    FineOp.Op(back.f, Mv.f);
    Aggs.ProjectToSubspace(c2.f, Mv.f);
    CoarseOp.Op(c.f, c3.f);
    ok &= report("(R D P - D_c) v_c", rel_dev(c2.get(), c3.get()), 1e-12);

    // (5) Im(v_c^dag D_c^dag D_c v_c) / Re(...)
    CoarseOp.Op(c.f, c2.f);
    CoarseOp.AdjOp(c2.f, c3.f);
    auto a = c.get(), b = c3.get();
    cplx dot = 0;
    for (size_t i = 0; i < a.size(); ++i) dot += std::conj(a[i]) * b[i];
    ok &= report("Im(v^dag Dc^dag Dc v) / Re(...)", std::abs(dot.imag()) / std::abs(dot.real()), 1e-12);

    // red-black interface (src/Test_coarse_red_black.cc:170-482)
    // (6) Dhop + Mdiag = M
    Dc.Dhop(c.f, c2.f, 0);
    Dc.Mdiag(c.f, c3.f);
    {
      auto x = c2.get(), y = c3.get();
      for (size_t i = 0; i < x.size(); ++i) x[i] += y[i];
      Dc.M(c.f, c3.f);
      ok &= report("M - (Dhop + Mdiag)", rel_dev(c3.get(), x), 1e-13);
    }
    // (7) MooeeInv Mooee = 1 on each checkerboard, (8) Meo + Moe + Mee + Moo = M
    Dc.InvertSelfStencilPoint();
    DevField he(Vc / 2, 1, N), ho(Vc / 2, 1, N), t1(Vc / 2, 1, N), t2(Vc / 2, 1, N), full(Vc, 1, N);
    gmg::PickCheckerboard(0, cdims, c.f, he.f);
    gmg::PickCheckerboard(1, cdims, c.f, ho.f);
    Dc.Mooee(he.f, t1.f, 0);
    Dc.MooeeInv(t1.f, t2.f, 0);
    ok &= report("(1 - MooeeInv Mooee) v_e", rel_dev(he.get(), t2.get()), 1e-13);
    Dc.Meooe(he.f, t1.f, 0);  // -> odd
    Dc.Mooee(ho.f, t2.f, 1);
    {
      auto x = t1.get(), y = t2.get();
      for (size_t i = 0; i < x.size(); ++i) x[i] += y[i];
      t1.set(x);
    }
    gmg::SetCheckerboard(cdims, t1.f, 1, full.f);
    Dc.Meooe(ho.f, t1.f, 1);  // -> even
    Dc.Mooee(he.f, t2.f, 0);
    {
      auto x = t1.get(), y = t2.get();
      for (size_t i = 0; i < x.size(); ++i) x[i] += y[i];
      t1.set(x);
    }
    gmg::SetCheckerboard(cdims, t1.f, 0, full.f);
    Dc.M(c.f, c3.f);
    ok &= report("M - (Meo + Moe + Mee + Moo)", rel_dev(c3.get(), full.get()), 1e-13);

    // MG driver: 2 levels, test-vector setup, one refinement pass
    gmg_mg_params P = gmg::MultiGridPreconditioner::Params();
    P.nlevels = 2;
    P.nvec[0] = 4;
    P.setup_iters = 30;
    P.setup_null = 0;
    P.coarsest_iters = 30;
    P.refine_iters[0] = 1;
    gmg::MultiGridPreconditioner MG(D, P, 2);
    MG.initialSetup();
    MG.refinementSetup();
    DevField bb(Vf, 2, 12), xx(Vf, 2, 12), r(Vf, 2, 12);
    auto bh = gaussian(Vf * 2 * 12, gen);
    bb.set(bh);
    double rr = 0;
    const int its = MG.Solve(bb.f, xx.f, 1e-10, 300, &rr);
    FineOp.Op(xx.f, r.f);
    {
      auto Dx = r.get();
      double worst = 0;
      for (int k = 0; k < 2; ++k) {
        double num = 0, den = 0;
        for (long s2 = 0; s2 < Vf; ++s2)
          for (int a2 = 0; a2 < 12; ++a2) {
            const size_t i = ((size_t)s2 * 2 + k) * 12 + a2;
            num += std::norm(bh[i] - Dx[i]);
            den += std::norm(bh[i]);
          }
        worst = std::max(worst, std::sqrt(num / den));
      }
      std::printf("MG solve after refinementSetup: %d outer iterations\n", its);
      ok &= report("|b - D x| / |b| after refinementSetup", worst, 2e-10);
    }
    {
      gmg_agg* ag = MG.Aggregates(0);
      gmg_coarse* op = MG.CoarseMatrix(1);
      const int Nm = 2 * P.nvec[0];
      DevField vc(Vc, 1, Nm), rc(Vc, 1, Nm), dc(Vc, 1, Nm), pf(Vf, 1, 12), dpf(Vf, 1, 12);
      vc.set(gaussian(Vc * Nm, gen));
      gmg::check(gmg_agg_promote(ag, GMG_F64, GMG_F64, 1, vc.f.data, pf.f.data, nullptr));
      FineOp.Op(pf.f, dpf.f);
      gmg::check(gmg_agg_project(ag, GMG_F64, GMG_F64, 1, dpf.f.data, rc.f.data, nullptr));
      gmg::check(gmg_coarse_apply(op, GMG_OP_M, 8, GMG_F64, GMG_F64, 1, vc.f.data, dc.f.data, nullptr, 0, nullptr));
      ok &= report("(R D P - D_c) v_c after refinementSetup", rel_dev(rc.get(), dc.get()), 1e-12);
    }
    // ------------------------------------------------------------ Rework surface
    {
      typedef gmg::Rework::WilsonTwoSpinPolicy<nb> Policy;
      const gmg::Coordinate rbdims{cdims[0] / 2, cdims[1], cdims[2], cdims[3]};
      // (11) undoChiralDoublingG5C of the Upstream subspace (Bo), copied into the two-spin aggregation
      std::vector<cplx> undone(nb * Vf * 12);
      for (int n = 0; n < nb; ++n)
        for (long k = 0; k < Vf * 12; ++k) undone[n * Vf * 12 + k] = Bo[n * Vf * 12 + k] + Bo[(n + nb) * Vf * 12 + k];
      gmg::Rework::Aggregation<Policy> TwoSpinAggs(cdims, fdims, 0, 1);
      TwoSpinAggs.SetSubspace(reinterpret_cast<const double*>(undone.data()), false);
      std::vector<cplx> back2(nb * Vf * 12);
      TwoSpinAggs.GetSubspace(reinterpret_cast<double*>(back2.data()), false);
      ok &= report("two-spin Subspace() round trip", rel_dev(undone, back2), 1e-16);
      ok &= report("two-spin CheckOrthogonal", TwoSpinAggs.CheckOrthogonal(), 1e-13);

      // (12) two-spin CoarsenOperator (speed level 1) against the Upstream links
      gmg::Rework::CoarsenedMatrix<Policy> TwoSpinCMat(cdims, rbdims, 1, 0);
      TwoSpinCMat.CoarsenOperator(fdims, FineOp, TwoSpinAggs);
      std::vector<cplx> A(9 * Vc * N * N), Y(Vc * N * N);
      Dc.GetLinks(reinterpret_cast<double*>(A.data()), false);
      double worst = 0;
      for (int p = 0; p < 9; ++p) {
        TwoSpinCMat.GetLinks(p, reinterpret_cast<double*>(Y.data()), false);
        // convertLayout: Y(s1, s2)(c1, c2) = A(s1 nb + c1, s2 nb + c2)
        std::vector<cplx> flat(Vc * N * N);
        for (long st = 0; st < Vc; ++st)
          for (int s1 = 0; s1 < 2; ++s1)
            for (int s2 = 0; s2 < 2; ++s2)
              for (int c1 = 0; c1 < nb; ++c1)
                for (int c2 = 0; c2 < nb; ++c2)
                  flat[(st * N + s1 * nb + c1) * N + s2 * nb + c2] =
                      Y[(((st * 2 + s1) * 2 + s2) * nb + c1) * nb + c2];
        std::vector<cplx> ref(A.begin() + (long)p * Vc * N * N, A.begin() + (long)(p + 1) * Vc * N * N);
        worst = std::max(worst, rel_dev(ref, flat));
      }
      ok &= report("two-spin Y_[p] vs Upstream A[p], all points", worst, 1e-14);

      // (13) the operators on the same coarse fields
      DevField y1(Vc, 1, N), y2(Vc, 1, N);
      TwoSpinCMat.M(c.f, y1.f);
      Dc.M(c.f, y2.f);
      ok &= report("two-spin M vs Upstream M", rel_dev(y2.get(), y1.get()), 1e-14);
      TwoSpinCMat.Mdag(c.f, y1.f);
      Dc.Mdag(c.f, y2.f);
      ok &= report("two-spin Mdag vs Upstream Mdag", rel_dev(y2.get(), y1.get()), 1e-14);
      DevField e1(Vc / 2, 1, N), e2(Vc / 2, 1, N), o1(Vc / 2, 1, N);
      he.f.checkerboard = 0;
      TwoSpinCMat.Meooe(he.f, o1.f);  // even -> odd
      Dc.Meooe(he.f, t1.f, 0);
      ok &= report("two-spin Meooe (Even in) vs Upstream", rel_dev(t1.get(), o1.get()), 1e-14);
      if (o1.f.checkerboard != 1) ok &= report("two-spin Meooe sets the output checkerboard", 1.0, 0.5);
      TwoSpinCMat.Mooee(he.f, e1.f);
      TwoSpinCMat.MooeeInv(e1.f, e2.f);
      ok &= report("two-spin (1 - MooeeInv Mooee) v_e", rel_dev(he.get(), e2.get()), 1e-13);

      // (14) Create(MGBasisVectors): copy in and orthogonalise (two passes)
      gmg::Rework::Aggregation<Policy> Created(cdims, fdims);
      const double err = Created.Create(reinterpret_cast<const double*>(h.data()), false);
      ok &= report("two-spin Create: CheckOrthogonal", err, 1e-13);
    }
  } catch (const gmg::Error& e) {
    std::printf("gmg error %d: %s\n", (int)e.status, e.what());
    return 2;
  }
  std::printf("%s\n", ok ? "all checks passed" : "some checks FAILED");
  return ok ? 0 : 1;
}

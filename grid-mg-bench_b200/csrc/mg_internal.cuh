// mg_internal.cuh -- vectors and per-RHS kernels shared by the multigrid solvers.
#pragma once

#include "gmg_internal.cuh"

namespace gmg {

// A device field [V][R][dof] complex of precision prec (GMG_F64 / GMG_F32; GMG_BF16
// for the fine smoother's residual fields: one 32-bit word per complex number,
// real part in the low 16 bits).
struct Vec {
  void* p = nullptr;
  int64_t V = 0;
  int R = 0;
  int dof = 0;
  int prec = GMG_F64;
  int64_t elems() const { return V * (int64_t)R * dof; }
  size_t esize() const { return prec == GMG_F64 ? 16 : prec == GMG_BF16 ? 4 : 8; }
  size_t bytes() const { return (size_t)elems() * esize(); }
  // the first R' right-hand sides of a buffer laid out for R' RHS (compacted batches)
  Vec with_rhs(int r) const {
    Vec v = *this;
    v.R = r;
    return v;
  }
};

// Owned device field.
struct VecBuf : Vec {
  DevBuf buf;
  gmg_status alloc(int64_t V_, int R_, int dof_, int prec_) {
    V = V_;
    R = R_;
    dof = dof_;
    prec = prec_;
    GMG_TRY(buf.alloc(bytes()));
    p = buf.p;
    return GMG_OK;
  }
};

// out[j*R + r] = <X_j(r), Y(r)> for j < nx, X_j = X0 + j * xstride_elems (complex elements)
gmg_status vec_multidot(const Vec& X0, int nx, int64_t xstride_elems, const Vec& Y, double2* out_dev, const int* mask,
                        cudaStream_t s);
// Y(r) += sum_j a[j*R + r] X_j(r)
gmg_status vec_multiaxpy(const double2* a_dev, const Vec& X0, int nx, int64_t xstride_elems, Vec& Y, cudaStream_t s,
                         double sgn = 1.0);
// Y += sgn * sum_j a[j*R + r] X_j, then out = <X_j, Y> per (j, r) (mode 1) or
// <Y, Y> per r (mode 2) over the updated Y, in one sweep where possible
gmg_status vec_multiaxpy_dot(const double2* a_dev, const Vec& X0, int nx, int64_t xstride_elems, Vec& Y,
                             cudaStream_t s, double sgn, double2* out_dev, int mode);
// Y(r) = a[r] X(r) + b[r] Y(r)
gmg_status vec_axpby(const double2* a_dev, const Vec& X, const double2* b_dev, Vec& Y, cudaStream_t s);
// Y = X with a precision conversion
gmg_status vec_convert(const Vec& X, Vec& Y, cudaStream_t s);
// basis [2R][V][dof] (FP64) from X [V][R][dof] by chiral doubling
// basis [2 R][V][dof] FP64 = factor (1 +- G5) X from the R vectors of X
gmg_status vec_chiral_double(const Vec& X, double* basis_dev, cudaStream_t s, double factor = 0.5);
// dst(r') = src(idx[r']) (gather) / dst(idx[r']) = src(r') (scatter), idx on the device
gmg_status vec_gather(const Vec& src, const int* idx, Vec& dst, cudaStream_t s);
gmg_status vec_scatter(const Vec& src, const int* idx, Vec& dst, cudaStream_t s);
// seeded unit-Gaussian field (re, im ~ N(0, 1/2))
gmg_status vec_gaussian(Vec& X, uint64_t seed, cudaStream_t s);
// Y(r) = X(r) / sqrt(n[r].x), n from a device multidot
gmg_status vec_scale_inv_norm(const double2* n_dev, const Vec& X, Vec& Y, cudaStream_t s);
// MR step with alpha = d1 / d2 (device): x += alpha r, r -= alpha Ar
// x += a r, and r -= a Ar unless update_r is false, a = <Ar, r> / <Ar, Ar> per RHS
// (r, Ar BF16 with x FP32: the products in FP32, r rounded back to BF16)
// (conj_d1: d1 holds <r, Ar>, the conjugate)
gmg_status vec_mr_update(const double2* d1, const double2* d2, Vec& x, Vec& r, const Vec& Ar, cudaStream_t s,
                         bool update_r = true, bool conj_d1 = false);
// Y = X - Y
gmg_status vec_xmy(const Vec& X, Vec& Y, cudaStream_t s);
// Delayed-reorthogonalisation Gram-Schmidt sweeps (FP64, V0 [nv + 2] vectors at
// vstride elements): pass 1 forms <V_k, V_nv>, <V_k, B> (k < nv), <V_nv, V_nv>,
// <V_nv, B>, <B, B> per RHS (2 nv + 3 values at out[k * R + r]); pass 2 sets
// V_nv <- (V_nv - sum c_k V_k) / alpha and V_{nv+1} <- (B - sum g_k V_k - d V_nv) / beta
// with coef[k * R + r] = c (nv), g (nv), 1/alpha, d, 1/beta
bool vec_dcgs_supported(const Vec& B, int nv);
gmg_status vec_dcgs_dots(const Vec& V0, int64_t vstride, int nv, const Vec& B, double2* out_dev, cudaStream_t s);
gmg_status vec_dcgs_update(const double2* coef_dev, Vec& V0, int64_t vstride, int nv, const Vec& B, cudaStream_t s);
// Z (BF16) = X - Y (FP32), rounded to nearest even
gmg_status vec_xmy_bf16(const Vec& X, const Vec& Y, Vec& Z, cudaStream_t s);
// Z (BF16, site-blocked [V][3][R][4] words: the 16-byte quarters of one
// site's records back to back) = X - Y (FP32 spin-colour fields)
gmg_status vec_xmy_bf16_blocked(const Vec& X, const Vec& Y, Vec& Z, cudaStream_t s);
// MR on stored BF16 residuals, for a sweep that keeps every step's residual:
// rn = bf16(r - a Ar) with a = d1 / d2 (device) per RHS; `blocked`: the
// fields are site-blocked
gmg_status vec_mr_resid_bf16(const double2* d1, const double2* d2, const Vec& r, const Vec& Ar, Vec& rn, cudaStream_t s,
                             bool blocked = false);
// x (FP32) += sum_{j < K} a_j r_j with r_j = r0 + j * rstride words and
// a_j = d[j * dstride + k] / d[j * dstride + R + k].x for RHS k (K <= kMrMaxSteps)
constexpr int kMrMaxSteps = 16;
gmg_status vec_mr_xsum_bf16(const double2* d, int dstride, int K, const Vec& r0, int64_t rstride, Vec& x,
                            cudaStream_t s, bool blocked = false);
// G[a][b] = <X(a), X(b)> over the whole lattice (R <= 32 columns), FP64
gmg_status vec_gram(const Vec& X, double2* G_dev, cudaStream_t s);
// X(a) <- sum_{b <= a} T[a][b] X(b)   (lower-triangular recombination of the columns)
gmg_status vec_tri_apply(const double2* T_dev, Vec& X, cudaStream_t s);
// BiCGStab steps with per-RHS device scalars sc[4R] = (rho, alpha, omega, beta):
// bicg_scalar 0: beta / rho from rho_new = a; 1: alpha = rho / a; 2: omega = a / b
gmg_status bicg_scalar(int which, const double2* a, const double2* b, double2* sc, int R, cudaStream_t s);
// bicg_vec 0: a(p) = b(r) + beta (a - omega c(v)); 1: a(s) = b(r) - alpha c(v);
//          2: a(x) += alpha c(p) + omega d(s), b(r) = d(s) - omega e(t)
gmg_status bicg_vec(int which, Vec& a, const Vec& b, const Vec& c, const Vec& d, const Vec& e, const double2* sc,
                    cudaStream_t s);

}  // namespace gmg

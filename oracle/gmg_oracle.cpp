// gmg_oracle.cpp -- CPU FP64 restatement of the grid-mg-bench multigrid hot path.
//
// TEST INFRASTRUCTURE ONLY: the checker for the CUDA library, never linked by it.
// Parity: pinned by the reference's identity / known-answer checks (see header);
// absolute values of Grid's fine operator are parity unpinned (Grid is absent).
//
// Build: oracle/Makefile (g++ -O3 -march=native -fopenmp -shared).
#include "gmg_oracle.h"

#include <algorithm>
#include <cassert>
#include <cmath>
#include <complex>
#include <cstring>
#include <vector>

#include <omp.h>

typedef std::complex<double> cplx;
static const int NPOINT = 9;

// ----------------------------------------------------------------------------
// lexicographic helpers (Grid Lexicographic::CoorFromIndex / IndexFromCoor, x fastest)
// ----------------------------------------------------------------------------
static inline void coor_from_index(int64_t idx, const int* dims, int* c) {
  for (int d = 0; d < 4; ++d) { c[d] = (int)(idx % dims[d]); idx /= dims[d]; }
}
static inline int64_t index_from_coor(const int* c, const int* dims) {
  int64_t idx = 0;
  for (int d = 3; d >= 0; --d) idx = idx * dims[d] + c[d];
  return idx;
}
static inline int64_t volume(const int* dims) {
  return (int64_t)dims[0] * dims[1] * dims[2] * dims[3];
}
static inline int64_t shift_site(int64_t s, const int* dims, int dir, int disp) {
  int c[4];
  coor_from_index(s, dims, c);
  c[dir] = (c[dir] + disp + dims[dir]) % dims[dir];
  return index_from_coor(c, dims);
}
static inline cplx* C(double* p) { return reinterpret_cast<cplx*>(p); }
static inline const cplx* C(const double* p) { return reinterpret_cast<const cplx*>(p); }

// ----------------------------------------------------------------------------
// a1: geometry.  GeometryRework.h:54-125 (PointFromDirDisp, fill); the 4-d
// coarse stencil of CoarsenedMatrixUpstream.h:71-124.
// ----------------------------------------------------------------------------
extern "C" int orc_point_from_dir_disp(int ndim, int dirs_faster, int dir, int disp) {
  const int acts = ndim >= 5 ? 4 : ndim;
  const int base = ndim == 5 ? 1 : 0;
  if (dir == 0 && disp == 0) return 2 * acts;
  if (dirs_faster) return (1 - disp) / 2 * acts + dir - base;
  return 2 * (dir - base) + (1 - disp) / 2;
}

extern "C" void orc_geometry(int ndim, int dirs_faster, int* dirs, int* disps) {
  const int acts = ndim >= 5 ? 4 : ndim;
  const int base = ndim == 5 ? 1 : 0;
  const int npoint = 2 * acts + 1;
  for (int d = 0; d < acts; ++d) {
    if (dirs_faster) {
      dirs[d] = d + base; disps[d] = +1;
      dirs[d + acts] = d + base; disps[d + acts] = -1;
    } else {
      dirs[2 * d] = d + base; disps[2 * d] = +1;
      dirs[2 * d + 1] = d + base; disps[2 * d + 1] = -1;
    }
  }
  dirs[npoint - 1] = 0;
  disps[npoint - 1] = 0;
}

// a2: coarse neighbour table nbr[p][s] = lex(x + disp_p e_dir_p mod L) (Grid
// CartesianStencil with periodic wrap; used at CoarsenedMatrixUpstream.h:583-589).
extern "C" void orc_coarse_neighbors(const int* dims, int32_t* nbr) {
  const int64_t V = volume(dims);
  for (int p = 0; p < NPOINT; ++p) {
    const int dir = p < 8 ? (p % 4) : 0;
    const int disp = p < 4 ? +1 : (p < 8 ? -1 : 0);
    for (int64_t s = 0; s < V; ++s)
      nbr[p * V + s] = (int32_t)(disp ? shift_site(s, dims, dir, disp) : s);
  }
}

// ----------------------------------------------------------------------------
// a3: coarsening LUT.  CoarseningLookupTableRework.h:114-179: for every coarse
// site, the fine sites of its block in lexicographic in-block order, filtered
// by mask != 0; reverse[f] = coarse site of f (never has holes).
// ----------------------------------------------------------------------------
static void block_dims(const int* fdims, const int* cdims, int* b) {
  for (int d = 0; d < 4; ++d) {
    b[d] = fdims[d] / cdims[d];
    assert(b[d] * cdims[d] == fdims[d]);
  }
}

extern "C" int orc_lut_populate(const int* fdims, const int* cdims, const int8_t* mask,
                                int32_t* lut, int32_t* sizes, int32_t* reverse) {
  int b[4];
  block_dims(fdims, cdims, b);
  const int64_t Vc = volume(cdims);
  const int bv = b[0] * b[1] * b[2] * b[3];
#pragma omp parallel for
  for (int64_t sc = 0; sc < Vc; ++sc) {
    int cc[4], cb[4], cf[4];
    coor_from_index(sc, cdims, cc);
    int count = 0;
    for (int sb = 0; sb < bv; ++sb) {
      coor_from_index(sb, b, cb);
      for (int d = 0; d < 4; ++d) cf[d] = cc[d] * b[d] + cb[d];
      const int64_t sf = index_from_coor(cf, fdims);
      if (!mask || mask[sf] != 0) lut[sc * bv + count++] = (int32_t)sf;
      if (reverse) reverse[sf] = (int32_t)sc;
    }
    sizes[sc] = count;
    for (int k = count; k < bv; ++k) lut[sc * bv + k] = -1;
  }
  return bv;
}

// Outer masks of CoarsenOperator (CoarsenedMatrixUpstream.h:797-833):
// disp=+1 -> x_dir mod b == b-1; disp=-1 -> x_dir mod b == 0; self -> all zero.
extern "C" void orc_outer_mask(const int* fdims, const int* cdims, int point, int8_t* mask) {
  int b[4];
  block_dims(fdims, cdims, b);
  const int64_t Vf = volume(fdims);
  const int dir = point < 8 ? point % 4 : 0;
  const int disp = point < 4 ? +1 : (point < 8 ? -1 : 0);
  for (int64_t s = 0; s < Vf; ++s) {
    int c[4];
    coor_from_index(s, fdims, c);
    const int r = c[dir] % b[dir];
    mask[s] = disp == 0 ? 0 : (disp == 1 ? (r == b[dir] - 1) : (r == 0));
  }
}

// Block parity masks: bcb = sum_mu floor(x_mu / b_mu); even = bcb mod 2 == 0
// (CoarsenedMatrixUpstream.h:811-813, 826-827).
extern "C" void orc_block_parity_mask(const int* fdims, const int* cdims, int parity, int8_t* mask) {
  int b[4];
  block_dims(fdims, cdims, b);
  const int64_t Vf = volume(fdims);
  for (int64_t s = 0; s < Vf; ++s) {
    int c[4];
    coor_from_index(s, fdims, c);
    int bcb = 0;
    for (int d = 0; d < 4; ++d) bcb += c[d] / b[d];
    mask[s] = ((bcb % 2) == parity) ? 1 : 0;
  }
}

// ----------------------------------------------------------------------------
// a8-a11: coarse stencil.  CoarsenedMatrixUpstream.h:546-607 (M), 609-621
// (Mdag = G5C M G5C unless hermitian), 642-742 (MdirCalc / Mdir / Mdiag);
// multi-RHS form ...LutMRHS.h:767-794 (links shared across the RHS).
//   op: 0 = M, 1 = Mdag, 2 = Mdiag, 3 = single point `point`
// ----------------------------------------------------------------------------
extern "C" void orc_coarse_g5(int64_t V, int N, int R, double* v) {
  cplx* z = C(v);
#pragma omp parallel for
  for (int64_t s = 0; s < V; ++s)
    for (int r = 0; r < R; ++r)
      for (int b = N / 2; b < N; ++b) z[(s * R + r) * N + b] = -z[(s * R + r) * N + b];
}

extern "C" void orc_coarse_apply_range(const int* dims, int N, int R, const double* links,
                                       const double* in, double* out, int op, int point, int hermitian,
                                       int64_t s0, int64_t s1);

// number of OpenMP threads the oracle's parallel loops use (n <= 0: the
// runtime default); returns the previous setting (timing samples at 1 thread)
extern "C" int orc_set_threads(int n) {
  const int prev = omp_get_max_threads();
  omp_set_num_threads(n > 0 ? n : omp_get_num_procs());
  return prev;
}

extern "C" void orc_coarse_apply(const int* dims, int N, int R, const double* links,
                                 const double* in, double* out, int op, int point, int hermitian) {
  orc_coarse_apply_range(dims, N, R, links, in, out, op, point, hermitian, 0, volume(dims));
}

// Same as orc_coarse_apply restricted to output sites [s0, s1) (bounded CPU
// timing samples); other output sites are left untouched.
extern "C" void orc_coarse_apply_range(const int* dims, int N, int R, const double* links,
                                       const double* in, double* out, int op, int point, int hermitian,
                                       int64_t s0, int64_t s1) {
  const int64_t V = volume(dims);
  const cplx* A = C(links);
  const cplx* x = C(in);
  cplx* y = C(out);
  std::vector<int32_t> nbr(NPOINT * V);
  orc_coarse_neighbors(dims, nbr.data());
  std::vector<cplx> xin;
  const bool g5 = (op == 1 && !hermitian);
  if (g5) {  // G5C(tmp, in)
    xin.assign(x, x + V * R * N);
    orc_coarse_g5(V, N, R, reinterpret_cast<double*>(xin.data()));
    x = xin.data();
  }
  int p0 = 0, p1 = NPOINT;
  if (op == 2) { p0 = 8; p1 = 9; }
  if (op == 3) { p0 = point; p1 = point + 1; }
  // Per site and point the N x N link times the R x N input block, in real
  // arithmetic on split (re, im) copies so that the inner loop runs over the
  // output row b with unit stride and vectorises: for each (r, bb) the column
  // A[.][bb] is scaled by in[r][bb] and added to the accumulators of row r.
  // The sums over bb and p are taken in the same order for every output.
#pragma omp parallel
  {
    std::vector<double> atr((size_t)N * N), ati((size_t)N * N), accr((size_t)R * N), acci((size_t)R * N);
#pragma omp for schedule(static)
    for (int64_t s = s0; s < s1; ++s) {
      std::fill(accr.begin(), accr.end(), 0.0);
      std::fill(acci.begin(), acci.end(), 0.0);
      for (int p = p0; p < p1; ++p) {
        const cplx* Ap = A + ((int64_t)p * V + s) * N * N;
        for (int b = 0; b < N; ++b)
          for (int bb = 0; bb < N; ++bb) {
            atr[(size_t)bb * N + b] = Ap[(int64_t)b * N + bb].real();
            ati[(size_t)bb * N + b] = Ap[(int64_t)b * N + bb].imag();
          }
        const cplx* xs = x + (int64_t)nbr[p * V + s] * R * N;
        for (int r = 0; r < R; ++r) {
          double* __restrict__ yr = accr.data() + (size_t)r * N;
          double* __restrict__ yi = acci.data() + (size_t)r * N;
          for (int bb = 0; bb < N; ++bb) {
            const double xr = xs[(int64_t)r * N + bb].real(), xi = xs[(int64_t)r * N + bb].imag();
            const double* __restrict__ cr = atr.data() + (size_t)bb * N;
            const double* __restrict__ ci = ati.data() + (size_t)bb * N;
#pragma omp simd
            for (int b = 0; b < N; ++b) {
              yr[b] += cr[b] * xr - ci[b] * xi;
              yi[b] += cr[b] * xi + ci[b] * xr;
            }
          }
        }
      }
      for (int r = 0; r < R; ++r)
        for (int b = 0; b < N; ++b) y[(s * R + r) * N + b] = cplx(accr[(size_t)r * N + b], acci[(size_t)r * N + b]);
    }
  }
  if (g5) {  // G5C(out, out) on the computed sites
    cplx* z = C(out);
    for (int64_t s = s0; s < s1; ++s)
      for (int r = 0; r < R; ++r)
        for (int b = N / 2; b < N; ++b) z[(s * R + r) * N + b] = -z[(s * R + r) * N + b];
  }
}

// ----------------------------------------------------------------------------
// a4/a5/a6: block projection, promotion and orthonormalisation with LUTs.
//   project:  ...Lut.h:70-121   coarse_i(c) = sum_{x in lut[c]} <v_i(x), f(x)>
//   promote:  ...Lut.h:122-170  f(x) = sum_i c_i(c(x)) v_i(x), i ascending
//   ortho:    ...Lut.h:172-240  per-block modified Gram-Schmidt
// <a,b> = sum conj(a) b (Grid innerProduct).
// ----------------------------------------------------------------------------
struct Lut {
  std::vector<int32_t> lut, sizes, reverse;
  int bv;
  Lut(const int* fdims, const int* cdims, const int8_t* mask) {
    int b[4];
    block_dims(fdims, cdims, b);
    bv = b[0] * b[1] * b[2] * b[3];
    const int64_t Vc = volume(cdims), Vf = volume(fdims);
    lut.resize(Vc * bv);
    sizes.resize(Vc);
    reverse.resize(Vf);
    orc_lut_populate(fdims, cdims, mask, lut.data(), sizes.data(), reverse.data());
  }
};

extern "C" void orc_block_project(const int* fdims, const int* cdims, int dof, int N, int R,
                                  const double* basis, const double* fine, double* coarse,
                                  const int8_t* mask) {
  Lut L(fdims, cdims, mask);
  const int64_t Vc = volume(cdims), Vf = volume(fdims);
  const cplx* B = C(basis);
  const cplx* f = C(fine);
  cplx* c = C(coarse);
#pragma omp parallel for collapse(2)
  for (int64_t sc = 0; sc < Vc; ++sc)
    for (int r = 0; r < R; ++r)
      for (int i = 0; i < N; ++i) {
        cplx acc = 0.0;
        for (int j = 0; j < L.sizes[sc]; ++j) {
          const int64_t sf = L.lut[sc * L.bv + j];
          const cplx* v = B + ((int64_t)i * Vf + sf) * dof;
          const cplx* w = f + (sf * R + r) * dof;
          for (int a = 0; a < dof; ++a) acc += std::conj(v[a]) * w[a];
        }
        c[(sc * R + r) * N + i] = acc;
      }
}

extern "C" void orc_block_promote(const int* fdims, const int* cdims, int dof, int N, int R,
                                  const double* basis, const double* coarse, double* fine) {
  Lut L(fdims, cdims, nullptr);
  const int64_t Vf = volume(fdims);
  const cplx* B = C(basis);
  const cplx* c = C(coarse);
  cplx* f = C(fine);
#pragma omp parallel for
  for (int64_t sf = 0; sf < Vf; ++sf) {
    const int64_t sc = L.reverse[sf];
    for (int r = 0; r < R; ++r)
      for (int a = 0; a < dof; ++a) {
        cplx acc = 0.0;
        for (int i = 0; i < N; ++i)
          acc += c[(sc * R + r) * N + i] * B[((int64_t)i * Vf + sf) * dof + a];
        f[(sf * R + r) * dof + a] = acc;
      }
  }
}

extern "C" void orc_block_orthonormalise(const int* fdims, const int* cdims, int dof, int N,
                                         double* basis, int passes) {
  Lut L(fdims, cdims, nullptr);
  const int64_t Vc = volume(cdims), Vf = volume(fdims);
  cplx* B = C(basis);
  for (int pass = 0; pass < passes; ++pass) {
#pragma omp parallel for
    for (int64_t sc = 0; sc < Vc; ++sc) {
      const int n = L.sizes[sc];
      const int32_t* l = &L.lut[sc * L.bv];
      for (int v = 0; v < N; ++v) {
        cplx* bv = B + (int64_t)v * Vf * dof;
        for (int u = 0; u < v; ++u) {
          const cplx* bu = B + (int64_t)u * Vf * dof;
          cplx alpha = 0.0;
          for (int j = 0; j < n; ++j)
            for (int a = 0; a < dof; ++a) alpha += std::conj(bu[l[j] * dof + a]) * bv[l[j] * dof + a];
          for (int j = 0; j < n; ++j)
            for (int a = 0; a < dof; ++a) bv[l[j] * dof + a] -= alpha * bu[l[j] * dof + a];
        }
        double nrm = 0.0;
        for (int j = 0; j < n; ++j)
          for (int a = 0; a < dof; ++a) nrm += std::norm(bv[l[j] * dof + a]);
        const double s = 1.0 / std::sqrt(nrm);
        for (int j = 0; j < n; ++j)
          for (int a = 0; a < dof; ++a) bv[l[j] * dof + a] *= s;
      }
    }
  }
}

// ----------------------------------------------------------------------------
// a7: chiral doubling (Benchmark_helpers.h:156-181 with factor 1/2 = G5C;
// :130-154 with factor 1 = G5R5, equal to gamma5 in 4-d).  gamma5 is
// diag(+1,+1,-1,-1) on spin for dof=12 (spin-major, colour fastest), and
// diag(+1 x dof/2, -1 x dof/2) on a coarse vector (G5C).
//   v_n <- f (v + g5 v),   v_{n+nb} <- f (v - g5 v)
// ----------------------------------------------------------------------------
static inline double g5_sign(int dof, int a) { return (a < dof / 2) ? 1.0 : -1.0; }

extern "C" void orc_chiral_double(int64_t V, int dof, int nb, double* basis, double factor) {
  cplx* B = C(basis);
  for (int n = 0; n < nb; ++n) {
    cplx* lo = B + (int64_t)n * V * dof;
    cplx* hi = B + (int64_t)(n + nb) * V * dof;
#pragma omp parallel for
    for (int64_t s = 0; s < V; ++s)
      for (int a = 0; a < dof; ++a) {
        const cplx v = lo[s * dof + a];
        const cplx g = g5_sign(dof, a) * v;
        lo[s * dof + a] = factor * (v + g);
        hi[s * dof + a] = factor * (v - g);
      }
  }
}

// undoChiralDoublingG5C (Benchmark_helpers.h:193-213): v_n = v_n + v_{n+nb}
extern "C" void orc_undo_chiral_double(int64_t V, int dof, int nb, double* basis) {
  cplx* B = C(basis);
  for (int n = 0; n < nb; ++n) {
    cplx* lo = B + (int64_t)n * V * dof;
    const cplx* hi = B + (int64_t)(n + nb) * V * dof;
    for (int64_t k = 0; k < V * dof; ++k) lo[k] += hi[k];
  }
}

// ----------------------------------------------------------------------------
// a15: fine Wilson-clover operator (Grid WilsonCloverFermion semantics restated
// from the textbook definition; absolute parity with Grid unpinned).
//   D psi(x) = Mdiag psi(x) + sum_{mu, disp} Mdir_{mu,disp} psi(x)
//   Mdir_{mu,+1} psi(x) = -1/2 (1 - gamma_mu) U_mu(x)        psi(x+mu)
//   Mdir_{mu,-1} psi(x) = -1/2 (1 + gamma_mu) U_mu(x-mu)^dag psi(x-mu)
//   Mdiag psi(x)        = (4 + m) psi(x) + Cl(x) psi(x),
//   Cl(x) = -(c_sw/2) sum_{mu<nu} sigma_{mu nu} F_{mu nu}(x),
//   sigma_{mu nu} = (i/2)[gamma_mu, gamma_nu],  F = (Q - Q^dag)/(8i),
//   Q = sum of the four plaquette leaves in the (mu,nu) plane at x.
// Antiperiodic time: hops across the t boundary pick up a factor -1.
// Gamma matrices: DeGrand-Rossi chiral basis, gamma5 = diag(1,1,-1,-1).
// Layouts: U[site][mu][3][3], clover[site][2][6][6] (chiral blocks, index
// 3*s_local + c), spinor [site][rhs][spin 4][colour 3].
// ----------------------------------------------------------------------------
static void gamma_mat(int mu, cplx g[4][4]) {
  const cplx I(0, 1);
  for (int a = 0; a < 4; ++a)
    for (int b = 0; b < 4; ++b) g[a][b] = 0.0;
  switch (mu) {
    case 0: g[0][3] = I; g[1][2] = I; g[2][1] = -I; g[3][0] = -I; break;
    case 1: g[0][3] = -1.0; g[1][2] = 1.0; g[2][1] = 1.0; g[3][0] = -1.0; break;
    case 2: g[0][2] = I; g[1][3] = -I; g[2][0] = -I; g[3][1] = I; break;
    case 3: g[0][2] = 1.0; g[1][3] = 1.0; g[2][0] = 1.0; g[3][1] = 1.0; break;
    default: for (int a = 0; a < 4; ++a) g[a][a] = a < 2 ? 1.0 : -1.0;  // gamma5
  }
}

extern "C" void orc_gamma(int mu, double* g) {
  cplx m[4][4];
  gamma_mat(mu, m);
  for (int a = 0; a < 4; ++a)
    for (int b = 0; b < 4; ++b) C(g)[a * 4 + b] = m[a][b];
}

typedef cplx Mat3[3][3];
static inline void mat_load(const cplx* p, Mat3 m) {
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) m[a][b] = p[a * 3 + b];
}
static inline void mat_mul(const Mat3 a, const Mat3 b, Mat3 c) {
  Mat3 t;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      cplx s = 0.0;
      for (int k = 0; k < 3; ++k) s += a[i][k] * b[k][j];
      t[i][j] = s;
    }
  std::memcpy(c, t, sizeof(Mat3));
}
static inline void mat_dag(const Mat3 a, Mat3 c) {
  Mat3 t;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) t[i][j] = std::conj(a[j][i]);
  std::memcpy(c, t, sizeof(Mat3));
}

extern "C" void orc_clover_build(const int* dims, const double* Ud, double csw, double* clover) {
  const int64_t V = volume(dims);
  const cplx* U = C(Ud);
  cplx* Cl = C(clover);
  cplx G[4][4][4];
  for (int mu = 0; mu < 4; ++mu) gamma_mat(mu, G[mu]);
#pragma omp parallel for
  for (int64_t s = 0; s < V; ++s) {
    cplx full[12][12];
    for (int a = 0; a < 12; ++a)
      for (int b = 0; b < 12; ++b) full[a][b] = 0.0;
    for (int mu = 0; mu < 4; ++mu)
      for (int nu = mu + 1; nu < 4; ++nu) {
        auto link = [&](int64_t site, int d, Mat3 m) { mat_load(U + (site * 4 + d) * 9, m); };
        const int64_t xpm = shift_site(s, dims, mu, +1), xpn = shift_site(s, dims, nu, +1);
        const int64_t xmm = shift_site(s, dims, mu, -1), xmn = shift_site(s, dims, nu, -1);
        const int64_t xmm_pn = shift_site(xmm, dims, nu, +1);
        const int64_t xmm_mn = shift_site(xmm, dims, nu, -1);
        const int64_t xmn_pm = shift_site(xmn, dims, mu, +1);
        Mat3 Q, t, a, b;
        for (int i = 0; i < 3; ++i)
          for (int j = 0; j < 3; ++j) Q[i][j] = 0.0;
        auto acc = [&](const Mat3 m) {
          for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) Q[i][j] += m[i][j];
        };
        // leaf 1: U_mu(x) U_nu(x+mu) U_mu(x+nu)^+ U_nu(x)^+
        link(s, mu, a); link(xpm, nu, b); mat_mul(a, b, t);
        link(xpn, mu, a); mat_dag(a, a); mat_mul(t, a, t);
        link(s, nu, a); mat_dag(a, a); mat_mul(t, a, t); acc(t);
        // leaf 2: U_nu(x) U_mu(x-mu+nu)^+ U_nu(x-mu)^+ U_mu(x-mu)
        link(s, nu, a); link(xmm_pn, mu, b); mat_dag(b, b); mat_mul(a, b, t);
        link(xmm, nu, a); mat_dag(a, a); mat_mul(t, a, t);
        link(xmm, mu, a); mat_mul(t, a, t); acc(t);
        // leaf 3: U_mu(x-mu)^+ U_nu(x-mu-nu)^+ U_mu(x-mu-nu) U_nu(x-nu)
        link(xmm, mu, a); mat_dag(a, a); link(xmm_mn, nu, b); mat_dag(b, b); mat_mul(a, b, t);
        link(xmm_mn, mu, a); mat_mul(t, a, t);
        link(xmn, nu, a); mat_mul(t, a, t); acc(t);
        // leaf 4: U_nu(x-nu)^+ U_mu(x-nu) U_nu(x-nu+mu) U_mu(x)^+
        link(xmn, nu, a); mat_dag(a, a); link(xmn, mu, b); mat_mul(a, b, t);
        link(xmn_pm, nu, a); mat_mul(t, a, t);
        link(s, mu, a); mat_dag(a, a); mat_mul(t, a, t); acc(t);
        // F = (Q - Q^+)/(8i)
        Mat3 F;
        for (int i = 0; i < 3; ++i)
          for (int j = 0; j < 3; ++j) F[i][j] = (Q[i][j] - std::conj(Q[j][i])) / cplx(0, 8);
        // sigma = (i/2)[g_mu, g_nu]
        cplx sig[4][4];
        for (int i = 0; i < 4; ++i)
          for (int j = 0; j < 4; ++j) {
            cplx c1 = 0.0;
            for (int k = 0; k < 4; ++k) c1 += G[mu][i][k] * G[nu][k][j] - G[nu][i][k] * G[mu][k][j];
            sig[i][j] = cplx(0, 0.5) * c1;
          }
        for (int si = 0; si < 4; ++si)
          for (int sj = 0; sj < 4; ++sj)
            for (int ci = 0; ci < 3; ++ci)
              for (int cj = 0; cj < 3; ++cj)
                full[si * 3 + ci][sj * 3 + cj] += -0.5 * csw * sig[si][sj] * F[ci][cj];
      }
    // store the two chiral 6x6 blocks (off-diagonal blocks vanish: sigma commutes with gamma5)
    for (int blk = 0; blk < 2; ++blk)
      for (int a = 0; a < 6; ++a)
        for (int b = 0; b < 6; ++b) Cl[((s * 2 + blk) * 6 + a) * 6 + b] = full[blk * 6 + a][blk * 6 + b];
  }
}

// Mdir apply for one (mu, disp) added into out with coefficient `coef`
static void wilson_hop(const int* dims, const cplx* U, int antiperiodic_t, int R, const cplx* in,
                       cplx* out, int mu, int disp, bool accumulate) {
  const int64_t V = volume(dims);
  cplx G[4][4];
  gamma_mat(mu, G);
  const double sg = disp > 0 ? -1.0 : 1.0;  // (1 - g) for +1, (1 + g) for -1
#pragma omp parallel for
  for (int64_t s = 0; s < V; ++s) {
    int c[4];
    coor_from_index(s, dims, c);
    const int64_t nb = shift_site(s, dims, mu, disp);
    double phase = 1.0;
    if (antiperiodic_t && mu == 3) {
      if (disp > 0 && c[3] == dims[3] - 1) phase = -1.0;
      if (disp < 0 && c[3] == 0) phase = -1.0;
    }
    Mat3 Um;
    if (disp > 0) mat_load(U + (s * 4 + mu) * 9, Um);
    else { mat_load(U + (nb * 4 + mu) * 9, Um); mat_dag(Um, Um); }
    for (int r = 0; r < R; ++r) {
      const cplx* psi = in + (nb * R + r) * 12;
      cplx upsi[4][3];
      for (int sp = 0; sp < 4; ++sp)
        for (int a = 0; a < 3; ++a) {
          cplx t = 0.0;
          for (int b = 0; b < 3; ++b) t += Um[a][b] * psi[sp * 3 + b];
          upsi[sp][a] = t;
        }
      cplx* o = out + (s * R + r) * 12;
      for (int sp = 0; sp < 4; ++sp)
        for (int a = 0; a < 3; ++a) {
          cplx t = upsi[sp][a];
          for (int k = 0; k < 4; ++k) t += sg * G[sp][k] * upsi[k][a];
          t *= -0.5 * phase;
          if (accumulate) o[sp * 3 + a] += t; else o[sp * 3 + a] = t;
        }
    }
  }
}

static void wilson_diag(const int* dims, const cplx* Cl, double mass, int R, const cplx* in,
                        cplx* out, bool accumulate) {
  const int64_t V = volume(dims);
#pragma omp parallel for
  for (int64_t s = 0; s < V; ++s)
    for (int r = 0; r < R; ++r) {
      const cplx* psi = in + (s * R + r) * 12;
      cplx* o = out + (s * R + r) * 12;
      for (int blk = 0; blk < 2; ++blk)
        for (int a = 0; a < 6; ++a) {
          cplx t = (4.0 + mass) * psi[blk * 6 + a];
          if (Cl)
            for (int b = 0; b < 6; ++b) t += Cl[((s * 2 + blk) * 6 + a) * 6 + b] * psi[blk * 6 + b];
          if (accumulate) o[blk * 6 + a] += t; else o[blk * 6 + a] = t;
        }
    }
}

static void g5_fine(int64_t V, int R, cplx* v) {
#pragma omp parallel for
  for (int64_t k = 0; k < V * R; ++k)
    for (int a = 6; a < 12; ++a) v[k * 12 + a] = -v[k * 12 + a];
}

// op: 0 = M, 1 = Mdag (= g5 M g5), 2 = Mdiag, 3 = Mdir(dir, disp)
extern "C" void orc_wilson_clover_apply(const int* dims, const double* U, const double* clover,
                                        double mass, int antiperiodic_t, int R, const double* in,
                                        double* out, int op, int dir, int disp) {
  const int64_t V = volume(dims);
  const cplx* x = C(in);
  cplx* y = C(out);
  const cplx* Cl = clover ? C(clover) : nullptr;
  std::vector<cplx> tmp;
  if (op == 1) {
    tmp.assign(x, x + V * R * 12);
    g5_fine(V, R, tmp.data());
    x = tmp.data();
  }
  if (op == 3) {
    wilson_hop(dims, C(U), antiperiodic_t, R, x, y, dir, disp, false);
    return;
  }
  wilson_diag(dims, Cl, mass, R, x, y, false);
  if (op == 2) return;
  for (int mu = 0; mu < 4; ++mu)
    for (int d : {+1, -1}) wilson_hop(dims, C(U), antiperiodic_t, R, x, y, mu, d, true);
  if (op == 1) g5_fine(V, R, y);
}

// ----------------------------------------------------------------------------
// a12/a13: Galerkin coarse-operator construction over a generic fine operator.
//   variant 0 = Upstream (CoarsenedMatrixUpstream.h:755-931): project all 8
//               directional applies over their outer masks, self term by the
//               even/odd block trick, ForceHermitian if hermitian.
//   variant 1 = Dirsave/Lut (...DirsaveLut.h:927-1097): project only the
//               disp=-1 directions, then ConstructRemainingLinks (:1164-1196)
//               or ForceHermitian.
// ----------------------------------------------------------------------------
struct FineOpOracle {
  int dims[4];
  int dof;
  virtual void mdir(const cplx* in, cplx* out, int point) const = 0;  // point < 8
  virtual void mdiag(const cplx* in, cplx* out) const = 0;
  void m(const cplx* in, cplx* out) const {
    const int64_t n = volume(dims) * dof;
    std::vector<cplx> t(n);
    mdiag(in, out);
    for (int p = 0; p < 8; ++p) {
      mdir(in, t.data(), p);
      for (int64_t k = 0; k < n; ++k) out[k] += t[k];
    }
  }
  virtual ~FineOpOracle() {}
};

struct WilsonOracle : FineOpOracle {
  const cplx *U, *Cl;
  double mass;
  int apbc;
  void mdir(const cplx* in, cplx* out, int p) const override {
    wilson_hop(dims, U, apbc, 1, in, out, p % 4, p < 4 ? +1 : -1, false);
  }
  void mdiag(const cplx* in, cplx* out) const override { wilson_diag(dims, Cl, mass, 1, in, out, false); }
};

struct CoarseOracle : FineOpOracle {
  const double* links;
  int hermitian;
  void mdir(const cplx* in, cplx* out, int p) const override {
    orc_coarse_apply(dims, dof, 1, links, reinterpret_cast<const double*>(in),
                     reinterpret_cast<double*>(out), 3, p, hermitian);
  }
  void mdiag(const cplx* in, cplx* out) const override {
    orc_coarse_apply(dims, dof, 1, links, reinterpret_cast<const double*>(in),
                     reinterpret_cast<double*>(out), 2, 8, hermitian);
  }
};

extern "C" void orc_construct_remaining_links(const int* dims, int N, double* links, int hermitian) {
  const int64_t V = volume(dims);
  cplx* A = C(links);
  const int64_t NN = (int64_t)N * N;
  for (int p = 4; p < 8; ++p) {
    const int dir = p - 4;
    std::vector<cplx> tmp(V * NN);
    for (int64_t s = 0; s < V; ++s)
      for (int n1 = 0; n1 < N; ++n1)
        for (int n2 = 0; n2 < N; ++n2) {
          double f = 1.0;
          if (!hermitian) {
            const int k = n1 / (N / 2), l = n2 / (N / 2);
            f = ((k + l) % 2 == 1) ? -1.0 : 1.0;
          }
          tmp[s * NN + n1 * N + n2] = f * std::conj(A[((int64_t)p * V + s) * NN + n2 * N + n1]);
        }
    // A[p-4] = Cshift(tmp, dir, +1): A(x) = tmp(x + dir)
    for (int64_t s = 0; s < V; ++s) {
      const int64_t sp = shift_site(s, dims, dir, +1);
      std::memcpy(&A[((int64_t)dir * V + s) * NN], &tmp[sp * NN], NN * sizeof(cplx));
    }
  }
}

static void coarsen_generic(const FineOpOracle& op, const int* cdims, int N, const cplx* basis,
                            int hermitian, int variant, cplx* A) {
  const int* fdims = op.dims;
  const int dof = op.dof;
  const int64_t Vf = volume(fdims), Vc = volume(cdims);
  const int64_t NN = (int64_t)N * N;
  std::memset((void*)A, 0, sizeof(cplx) * NPOINT * Vc * NN);
  std::vector<int8_t> even(Vf), odd(Vf), mask(Vf);
  orc_block_parity_mask(fdims, cdims, 0, even.data());
  orc_block_parity_mask(fdims, cdims, 1, odd.data());
  std::vector<cplx> Mphi(Vf * dof), tmp(Vf * dof), Me(Vf * dof), Mo(Vf * dof), proj(Vc * N);
  for (int i = 0; i < N; ++i) {
    const cplx* phi = basis + (int64_t)i * Vf * dof;
    for (int p = 0; p < 8; ++p) {
      const int disp = p < 4 ? +1 : -1;
      if (variant == 1 && disp != -1) continue;
      if (variant == 0 && hermitian && disp != -1) continue;
      op.mdir(phi, Mphi.data(), p);
      orc_outer_mask(fdims, cdims, p, mask.data());
      orc_block_project(fdims, cdims, dof, N, 1, reinterpret_cast<const double*>(basis),
                        reinterpret_cast<const double*>(Mphi.data()),
                        reinterpret_cast<double*>(proj.data()), mask.data());
      for (int64_t sc = 0; sc < Vc; ++sc)
        for (int j = 0; j < N; ++j) A[((int64_t)p * Vc + sc) * NN + j * N + i] = proj[sc * N + j];
    }
    // self term: tmp = e*M(e phi) + o*M(o phi)
    for (int64_t s = 0; s < Vf; ++s)
      for (int a = 0; a < dof; ++a) tmp[s * dof + a] = even[s] ? phi[s * dof + a] : 0.0;
    op.m(tmp.data(), Me.data());
    for (int64_t s = 0; s < Vf; ++s)
      for (int a = 0; a < dof; ++a) tmp[s * dof + a] = odd[s] ? phi[s * dof + a] : 0.0;
    op.m(tmp.data(), Mo.data());
    for (int64_t s = 0; s < Vf; ++s)
      for (int a = 0; a < dof; ++a) tmp[s * dof + a] = even[s] ? Me[s * dof + a] : Mo[s * dof + a];
    orc_block_project(fdims, cdims, dof, N, 1, reinterpret_cast<const double*>(basis),
                      reinterpret_cast<const double*>(tmp.data()), reinterpret_cast<double*>(proj.data()),
                      nullptr);
    for (int64_t sc = 0; sc < Vc; ++sc)
      for (int j = 0; j < N; ++j) A[((int64_t)8 * Vc + sc) * NN + j * N + i] = proj[sc * N + j];
  }
  if (hermitian || variant == 1)
    orc_construct_remaining_links(cdims, N, reinterpret_cast<double*>(A), hermitian);
}

extern "C" void orc_coarsen_wilson(const int* fdims, const int* cdims, int N, const double* basis,
                                   const double* U, const double* clover, double mass,
                                   int antiperiodic_t, int hermitian, int variant, double* links) {
  WilsonOracle op;
  std::memcpy(op.dims, fdims, sizeof(op.dims));
  op.dof = 12;
  op.U = C(U);
  op.Cl = clover ? C(clover) : nullptr;
  op.mass = mass;
  op.apbc = antiperiodic_t;
  coarsen_generic(op, cdims, N, C(basis), hermitian, variant, C(links));
}

extern "C" void orc_coarsen_coarse(const int* fdims, const int* cdims, int Nf, int N,
                                   const double* basis, const double* flinks, int fhermitian,
                                   int hermitian, int variant, double* links) {
  CoarseOracle op;
  std::memcpy(op.dims, fdims, sizeof(op.dims));
  op.dof = Nf;
  op.links = flinks;
  op.hermitian = fhermitian;
  coarsen_generic(op, cdims, N, C(basis), hermitian, variant, C(links));
}

// ----------------------------------------------------------------------------
// a14: Rework layout maps (Layout_converters.h:49-56, 107-110): flat index
// n = s*Nc_c + c.  Vectors keep their memory order; links go from
// [n1][n2] to [s1][s2][c1][c2].
// ----------------------------------------------------------------------------
extern "C" void orc_layout_vec_flat_to_spin(int64_t V, int N, int ncs, const double* in, double* out) {
  const int ncc = N / ncs;
  for (int64_t s = 0; s < V; ++s)
    for (int n = 0; n < N; ++n) {
      const int sp = n / ncc, c = n % ncc;
      C(out)[s * N + sp * ncc + c] = C(in)[s * N + n];
    }
}

extern "C" void orc_layout_link_flat_to_spin(int64_t V, int N, int ncs, const double* in, double* out) {
  const int ncc = N / ncs;
  const int64_t NN = (int64_t)N * N;
  for (int64_t s = 0; s < V; ++s)
    for (int n1 = 0; n1 < N; ++n1)
      for (int n2 = 0; n2 < N; ++n2) {
        const int s1 = n1 / ncc, c1 = n1 % ncc, s2 = n2 / ncc, c2 = n2 % ncc;
        C(out)[s * NN + ((s1 * ncs + s2) * ncc + c1) * ncc + c2] = C(in)[s * NN + n1 * N + n2];
      }
}

// ----------------------------------------------------------------------------
// Red-black (checkerboarded) coarse operator, Rework::CoarsenedMatrix
// (CoarsenedMatrixRework.h:178-245 Meooe/Mooee/Dhop, 288-394 DhopInternal,
// 617-640 MooeeInternal, 642-668 InvertSelfStencilPoint, 670-679 FillHalfCbs).
//
// Half fields follow Grid's red-black grid, checkerboarded in x: a site of
// parity q = (x+y+z+t) % 2 has half index h = x/2 + (Lx/2)*(y + Ly*(z + Lz*t)).
// ----------------------------------------------------------------------------
static inline int site_parity(int64_t s, const int* dims) {
  int c[4];
  coor_from_index(s, dims, c);
  return (c[0] + c[1] + c[2] + c[3]) & 1;
}

static inline int64_t half_index(int64_t s, const int* dims) {
  int c[4];
  coor_from_index(s, dims, c);
  return c[0] / 2 + (int64_t)(dims[0] / 2) * (c[1] + (int64_t)dims[1] * (c[2] + (int64_t)dims[2] * c[3]));
}

// pickCheckerboard / setCheckerboard on [site][per_site complex] fields
extern "C" void orc_pick_checkerboard(const int* dims, int cb, int64_t per_site, const double* full, double* half) {
  const int64_t V = volume(dims);
  for (int64_t s = 0; s < V; ++s)
    if (site_parity(s, dims) == cb)
      for (int64_t k = 0; k < per_site; ++k) C(half)[half_index(s, dims) * per_site + k] = C(full)[s * per_site + k];
}

extern "C" void orc_set_checkerboard(const int* dims, int cb, int64_t per_site, const double* half, double* full) {
  const int64_t V = volume(dims);
  for (int64_t s = 0; s < V; ++s)
    if (site_parity(s, dims) == cb)
      for (int64_t k = 0; k < per_site; ++k) C(full)[s * per_site + k] = C(half)[half_index(s, dims) * per_site + k];
}

// Inverse of each site's N x N self-stencil link (InvertSelfStencilPoint,
// Eigen's inverse() in the reference): Gauss-Jordan with partial pivoting.
// A8 and Ainv are [V][N][N] row-major.  Returns the number of singular sites.
extern "C" int orc_invert_self_links(int64_t V, int N, const double* A8, double* Ainv) {
  int singular = 0;
#pragma omp parallel for schedule(static) reduction(+ : singular)
  for (int64_t s = 0; s < V; ++s) {
    std::vector<cplx> a(C(A8) + s * N * N, C(A8) + (s + 1) * N * N);
    std::vector<cplx> inv((size_t)N * N, 0.0);
    for (int i = 0; i < N; ++i) inv[(size_t)i * N + i] = 1.0;
    for (int col = 0; col < N; ++col) {
      int piv = col;
      for (int r = col + 1; r < N; ++r)
        if (std::abs(a[(size_t)r * N + col]) > std::abs(a[(size_t)piv * N + col])) piv = r;
      if (std::abs(a[(size_t)piv * N + col]) == 0.0) {
        ++singular;
        break;
      }
      if (piv != col)
        for (int k = 0; k < N; ++k) {
          std::swap(a[(size_t)piv * N + k], a[(size_t)col * N + k]);
          std::swap(inv[(size_t)piv * N + k], inv[(size_t)col * N + k]);
        }
      const cplx d = 1.0 / a[(size_t)col * N + col];
      for (int k = 0; k < N; ++k) {
        a[(size_t)col * N + k] *= d;
        inv[(size_t)col * N + k] *= d;
      }
      for (int r = 0; r < N; ++r) {
        if (r == col) continue;
        const cplx f = a[(size_t)r * N + col];
        if (f == 0.0) continue;
        for (int k = 0; k < N; ++k) {
          a[(size_t)r * N + k] -= f * a[(size_t)col * N + k];
          inv[(size_t)r * N + k] -= f * inv[(size_t)col * N + k];
        }
      }
    }
    for (int64_t k = 0; k < (int64_t)N * N; ++k) C(Ainv)[s * N * N + k] = inv[k];
  }
  return singular;
}

// Red-black ops on half fields [Vh][R][N].  cb = parity of `in`.
//   op 0 Meooe       (DhopOE / DhopEO): out (parity 1-cb) = sum_{p<8} A_p in(nbr_p)
//   op 1 MeooeDag    G5C Meooe G5C (DhopInternal with dag, Galerkin form, :289-346)
//   op 2 Mooee       out (parity cb) = A_8 in
//   op 3 MooeeDag    adj(A_8) in          (MooeeInternal, :617-640)
//   op 4 MooeeInv    A_8^-1 in
//   op 5 MooeeInvDag adj(A_8^-1) in
// links [9][V][N][N] (exchange layout), self_inv [V][N][N] (ops 4, 5 only).
extern "C" void orc_coarse_rb_apply(const int* dims, int N, int R, const double* links, const double* self_inv,
                                    int op, int cb, const double* in_half, double* out_half) {
  const int64_t V = volume(dims), NN = (int64_t)N * N;
  const cplx* A = C(links);
  const cplx* x = C(in_half);
  cplx* y = C(out_half);
  std::vector<int32_t> nbr(NPOINT * V);
  orc_coarse_neighbors(dims, nbr.data());
  const bool hop = op <= 1;
  const int out_par = hop ? 1 - cb : cb;
  const bool g5 = op == 1;
  const int half = N / 2;
#pragma omp parallel for schedule(static)
  for (int64_t s = 0; s < V; ++s) {
    if (site_parity(s, dims) != out_par) continue;
    const int64_t ho = half_index(s, dims);
    for (int r = 0; r < R; ++r)
      for (int b = 0; b < N; ++b) {
        cplx res = 0.0;
        if (hop) {
          for (int p = 0; p < 8; ++p) {
            const cplx* Ap = A + ((int64_t)p * V + s) * NN + (int64_t)b * N;
            const cplx* nb = x + (half_index(nbr[p * V + s], dims) * R + r) * N;
            for (int bb = 0; bb < N; ++bb) res += Ap[bb] * (g5 && bb >= half ? -nb[bb] : nb[bb]);
          }
          if (g5 && b >= half) res = -res;
        } else {
          const cplx* M = (op >= 4) ? C(self_inv) + s * NN : A + ((int64_t)8 * V + s) * NN;
          const bool dag = (op == 3 || op == 5);
          const cplx* xi = x + (ho * R + r) * N;
          for (int bb = 0; bb < N; ++bb) res += (dag ? std::conj(M[(int64_t)bb * N + b]) : M[(int64_t)b * N + bb]) * xi[bb];
        }
        y[(ho * R + r) * N + b] = res;
      }
  }
}

// Full-grid Dhop (CoarsenedMatrixRework.h:210-217): the 8 hopping points,
// dag = G5C Dhop G5C regardless of the hermitian flag (DhopInternal, :289-346).
extern "C" void orc_coarse_dhop(const int* dims, int N, int R, const double* links, int dag, const double* in,
                                double* out) {
  const int64_t V = volume(dims), NN = (int64_t)N * N;
  const cplx* A = C(links);
  const cplx* x = C(in);
  cplx* y = C(out);
  std::vector<int32_t> nbr(NPOINT * V);
  orc_coarse_neighbors(dims, nbr.data());
  const int half = N / 2;
#pragma omp parallel for schedule(static)
  for (int64_t s = 0; s < V; ++s)
    for (int r = 0; r < R; ++r)
      for (int b = 0; b < N; ++b) {
        cplx res = 0.0;
        for (int p = 0; p < 8; ++p) {
          const cplx* Ap = A + ((int64_t)p * V + s) * NN + (int64_t)b * N;
          const cplx* nb = x + ((int64_t)nbr[p * V + s] * R + r) * N;
          for (int bb = 0; bb < N; ++bb) res += Ap[bb] * (dag && bb >= half ? -nb[bb] : nb[bb]);
        }
        y[(s * R + r) * N + b] = (dag && b >= half) ? -res : res;
      }
}

// Full-grid Mooee family (MooeeInternal on the full grid): op 2..5 as above.
extern "C" void orc_coarse_mooee(const int* dims, int N, int R, const double* links, const double* self_inv, int op,
                                 const double* in, double* out) {
  const int64_t V = volume(dims), NN = (int64_t)N * N;
#pragma omp parallel for schedule(static)
  for (int64_t s = 0; s < V; ++s) {
    const cplx* M = (op >= 4) ? C(self_inv) + s * NN : C(links) + ((int64_t)8 * V + s) * NN;
    const bool dag = (op == 3 || op == 5);
    for (int r = 0; r < R; ++r)
      for (int b = 0; b < N; ++b) {
        cplx res = 0.0;
        const cplx* xi = C(in) + (s * R + r) * N;
        for (int bb = 0; bb < N; ++bb) res += (dag ? std::conj(M[(int64_t)bb * N + b]) : M[(int64_t)b * N + bb]) * xi[bb];
        C(out)[(s * R + r) * N + b] = res;
      }
  }
}

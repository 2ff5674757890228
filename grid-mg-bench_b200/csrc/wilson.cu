// wilson.cu -- fine Wilson-clover operator on the GPU (FP64 / FP32, multi-RHS).
//
// The operator the reference coarsens and solves with is Grid's
// WilsonCloverFermionR reached through MdagMLinearOperator::{Op, AdjOp,
// OpDiag, OpDir} (src/Test_wilsonclover_mg.cc:103-113; identity checked at
// include/MultigridPreconditioner.h:317-350).  Grid is not part of the
// reference, so its textbook form is restated here (DeGrand-Rossi chiral
// gamma basis, gamma5 = diag(1,1,-1,-1)):
//
//   Mdir_{mu,+1} psi(x) = -1/2 (1 - gamma_mu) U_mu(x)        psi(x+mu)
//   Mdir_{mu,-1} psi(x) = -1/2 (1 + gamma_mu) U_mu(x-mu)^dag psi(x-mu)
//   Mdiag psi(x)        = (4 + m) psi(x) + Cl(x) psi(x)
//   Cl = -(c_sw/2) sum_{mu<nu} sigma_{mu nu} F_{mu nu}, F = (Q - Q^dag)/(8i)
//   M = Mdiag + sum Mdir,  Mdag = gamma5 M gamma5
//
// Hops across the time boundary pick up -1 for antiperiodic time.  One thread
// per (site, rhs); the (1 -+ gamma) projection halves the colour-matrix work
// (rank-2 projector: lower spins are a phase times the upper ones).
#include <algorithm>

#include "gmg_internal.cuh"

namespace gmg {

template <class T> struct wt;
template <> struct wt<double> { typedef double2 C; };
template <> struct wt<float> { typedef float2 C; };

template <class C> __device__ __forceinline__ C cmul(C a, C b) {
  C r;
  r.x = a.x * b.x - a.y * b.y;
  r.y = a.x * b.y + a.y * b.x;
  return r;
}
template <class C> __device__ __forceinline__ C cmulc(C a, C b) {  // conj(a) b
  C r;
  r.x = a.x * b.x + a.y * b.y;
  r.y = a.x * b.y - a.y * b.x;
  return r;
}
template <class C> __device__ __forceinline__ C cadd(C a, C b) { a.x += b.x; a.y += b.y; return a; }
// multiply by a unit phase code: 0 -> 1, 1 -> i, 2 -> -1, 3 -> -i
template <class C> __device__ __forceinline__ C cphase(C a, int code) {
  C r;
  switch (code & 3) {
    case 0: r = a; break;
    case 1: r.x = -a.y; r.y = a.x; break;
    case 2: r.x = -a.x; r.y = -a.y; break;
    default: r.x = a.y; r.y = -a.x; break;
  }
  return r;
}

// gamma_mu row s has one non-zero entry at column perm, value phase code
__constant__ int c_gperm[4][4] = {{3, 2, 1, 0}, {3, 2, 1, 0}, {2, 3, 0, 1}, {2, 3, 0, 1}};
__constant__ int c_gphase[4][4] = {{1, 1, 3, 3}, {2, 0, 0, 2}, {1, 3, 3, 1}, {0, 0, 0, 0}};
// the same tables as constexpr functions: with mu and s known at compile time
// (unrolled loops) the spinor indices fold and the spinors stay in registers
__host__ __device__ constexpr int gperm(int mu, int s) { return mu < 2 ? 3 - s : (s ^ 2); }
__host__ __device__ constexpr int gphase(int mu, int s) {
  return mu == 0 ? (s < 2 ? 1 : 3) : mu == 1 ? ((s == 0 || s == 3) ? 2 : 0) : mu == 2 ? ((s == 0 || s == 3) ? 1 : 3) : 0;
}

// accumulate one hop into out[4][3]
template <class T>
__device__ __forceinline__ void wilson_hop(typename wt<T>::C out[4][3],
                                           const typename wt<T>::C* __restrict__ U,  // 3x3 row-major
                                           bool dagger, const typename wt<T>::C* __restrict__ psi,
                                           int mu, int disp, T coef) {
  typedef typename wt<T>::C C;
  // projector P = 1 + sg gamma_mu, sg = -1 for disp +1, +1 for disp -1
  const int sgc = disp > 0 ? 2 : 0;  // phase code of sg
  C h[2][3];
#pragma unroll
  for (int s = 0; s < 2; ++s) {
    const int ps = gperm(mu, s);
    const int code = (gphase(mu, s) + sgc) & 3;
#pragma unroll
    for (int c = 0; c < 3; ++c) h[s][c] = cadd(psi[s * 3 + c], cphase(psi[ps * 3 + c], code));
  }
  C uh[2][3];
#pragma unroll
  for (int s = 0; s < 2; ++s)
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      C acc{0, 0};
#pragma unroll
      for (int b = 0; b < 3; ++b) {
        if (!dagger) acc = cadd(acc, cmul(U[a * 3 + b], h[s][b]));
        else acc = cadd(acc, cmulc(U[b * 3 + a], h[s][b]));
      }
      uh[s][a] = acc;
    }
#pragma unroll
  for (int s = 0; s < 2; ++s)
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      out[s][a].x += coef * uh[s][a].x;
      out[s][a].y += coef * uh[s][a].y;
    }
#pragma unroll
  for (int s = 2; s < 4; ++s) {
    const int ps = gperm(mu, s);
    const int code = (gphase(mu, s) + sgc) & 3;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const C v = cphase(uh[ps][a], code);
      out[s][a].x += coef * v.x;
      out[s][a].y += coef * v.y;
    }
  }
}

// One output spinor (site, rhs).  links(p) returns the 3x3 link of hop p
// (p < 4: U_mu(x), p >= 4: U_mu(x - mu), applied daggered); cl: the site's
// two 6x6 clover blocks.
template <class T, class LinkFn>
__device__ __forceinline__ void wilson_site(const typename wt<T>::C* __restrict__ cl, LinkFn links,
                                            const int32_t* __restrict__ nbr, const typename wt<T>::C* __restrict__ in,
                                            typename wt<T>::C* __restrict__ out, int V, int nrhs, int site, int r,
                                            T diag, int op, int dir, int disp, int apbc, int tvol, int Lt) {
  typedef typename wt<T>::C C;
  const bool g5 = (op == GMG_OP_MDAG);
  const int tc = site / tvol;
  C acc[4][3];
#pragma unroll
  for (int s = 0; s < 4; ++s)
#pragma unroll
    for (int c = 0; c < 3; ++c) acc[s][c] = C{0, 0};
  if (op != GMG_OP_MDIR) {
    // diagonal: (4 + m) psi + Cl psi, two chiral 6x6 blocks
    C psi[12];
    const C* src = in + ((int64_t)site * nrhs + r) * 12;
#pragma unroll
    for (int k = 0; k < 12; ++k) {
      psi[k] = src[k];
      if (g5 && k >= 6) { psi[k].x = -psi[k].x; psi[k].y = -psi[k].y; }
    }
#pragma unroll
    for (int blk = 0; blk < 2; ++blk)
#pragma unroll
      for (int a = 0; a < 6; ++a) {
        C v;
        v.x = diag * psi[blk * 6 + a].x;
        v.y = diag * psi[blk * 6 + a].y;
#pragma unroll
        for (int b = 0; b < 6; ++b) v = cadd(v, cmul(cl[(blk * 6 + a) * 6 + b], psi[blk * 6 + b]));
        acc[(blk * 6 + a) / 3][(blk * 6 + a) % 3] = v;
      }
  }
  if (op != GMG_OP_MDIAG) {
#pragma unroll
    for (int p = 0; p < 8; ++p) {
      const int mu = p & 3;
      const int dsp = p < 4 ? 1 : -1;
      if (op == GMG_OP_MDIR && (mu != dir || dsp != disp)) continue;
      const int nb = nbr[(int64_t)p * V + site];
      T coef = (T)-0.5;
      if (apbc && mu == 3 && ((dsp > 0 && tc == Lt - 1) || (dsp < 0 && tc == 0))) coef = (T)0.5;
      C psi[12];
      const C* src = in + ((int64_t)nb * nrhs + r) * 12;
#pragma unroll
      for (int k = 0; k < 12; ++k) {
        psi[k] = src[k];
        if (g5 && k >= 6) { psi[k].x = -psi[k].x; psi[k].y = -psi[k].y; }
      }
      wilson_hop<T>(acc, links(p, nb), dsp < 0, psi, mu, dsp, coef);
    }
  }
  C* dst = out + ((int64_t)site * nrhs + r) * 12;
#pragma unroll
  for (int s = 0; s < 4; ++s)
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      C v = acc[s][c];
      if (g5 && s >= 2) { v.x = -v.x; v.y = -v.y; }
      dst[s * 3 + c] = v;
    }
}

// thread per (site, rhs); links and clover read from global memory (few RHS)
template <class T>
__global__ void __launch_bounds__(256) wilson_kernel(
    const typename wt<T>::C* __restrict__ gauge, const typename wt<T>::C* __restrict__ clover,
    const int32_t* __restrict__ nbr, const typename wt<T>::C* __restrict__ in,
    typename wt<T>::C* __restrict__ out, int V, int nrhs, T diag, int op, int dir, int disp,
    int apbc, int tvol, int Lt) {
  typedef typename wt<T>::C C;
  const int64_t total = (int64_t)V * nrhs;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int site = (int)(e / nrhs);
    const int r = (int)(e % nrhs);
    auto links = [&](int p, int nb) -> const C* {
      return gauge + ((int64_t)(p < 4 ? site : nb) * 4 + (p & 3)) * 9;
    };
    wilson_site<T>(clover + (int64_t)site * 72, links, nbr, in, out, V, nrhs, site, r, diag, op, dir, disp, apbc, tvol,
                   Lt);
  }
}

// Multi-RHS tile: a CTA takes kTileSites consecutive sites and all right-hand
// sides (rt threads per site, each looping over its RHS); the sites' 8 hop
// links and clover blocks are staged in shared memory once and read by every
// RHS of the tile instead of once per RHS from global memory.
constexpr int kTileSites = 16;

template <class T>
__global__ void __launch_bounds__(256) wilson_tile_kernel(
    const typename wt<T>::C* __restrict__ gauge, const typename wt<T>::C* __restrict__ clover,
    const int32_t* __restrict__ nbr, const typename wt<T>::C* __restrict__ in,
    typename wt<T>::C* __restrict__ out, int V, int nrhs, int rt, T diag, int op, int dir, int disp,
    int apbc, int tvol, int Lt) {
  typedef typename wt<T>::C C;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* Ls = reinterpret_cast<C*>(smem_raw);  // [kTileSites][8][9]: p < 4 U_mu(x), p >= 4 U_mu(x - mu)
  C* Cs = Ls + kTileSites * 72;            // [kTileSites][72]
  const int nt = (V + kTileSites - 1) / kTileSites;
  const int sl = threadIdx.x / rt, rl = threadIdx.x % rt;
  for (int tile = blockIdx.x; tile < nt; tile += gridDim.x) {
    const int s0 = tile * kTileSites;
    const int ns = min(kTileSites, V - s0);
    __syncthreads();
    for (int k = threadIdx.x; k < ns * 72; k += blockDim.x) {
      const int j = k / 72, e = k % 72, p = e / 9, m = e % 9;
      const int site = s0 + j;
      const int ls = p < 4 ? site : nbr[(int64_t)p * V + site];
      Ls[k] = gauge[((int64_t)ls * 4 + (p & 3)) * 9 + m];
      Cs[k] = clover[(int64_t)s0 * 72 + k];
    }
    __syncthreads();
    if (sl < ns) {
      const int site = s0 + sl;
      const C* lsite = Ls + sl * 72;
      auto links = [&](int p, int) -> const C* { return lsite + p * 9; };
      for (int r = rl; r < nrhs; r += rt)
        wilson_site<T>(Cs + sl * 72, links, nbr, in, out, V, nrhs, site, r, diag, op, dir, disp, apbc, tvol, Lt);
    }
  }
}

// Multi-RHS quad kernel: four lanes per (site, rhs), lane q owning spin q.
// A quad reads its 12-component record as one contiguous run and consecutive
// quads hold consecutive right-hand sides, so a warp's loads cover 8 records
// back to back.  The spin projection (1 -+ gamma_mu) couples spin q with spin
// perm(q) of the same record: a quad-local shuffle.  Lanes 0 and 1 form the
// two projected half-spinors and multiply them by the link; lanes 2 and 3
// take the reconstructed lower spins from lanes perm(q).  The clover couples
// the two spins of a chiral block: one more shuffle.  Links and clover of the
// tile's kTileSites sites are staged in shared memory once per tile.
template <class C>
__device__ __forceinline__ C shfl_c(C v, int src_lane) {
  v.x = __shfl_sync(0xffffffffu, v.x, src_lane);
  v.y = __shfl_sync(0xffffffffu, v.y, src_lane);
  return v;
}

template <class T, int MU, bool DAG>
__device__ __forceinline__ void quad_hop(typename wt<T>::C acc[3], const typename wt<T>::C* __restrict__ U,
                                         const typename wt<T>::C psi[3], int q, int qbase, T coef) {
  typedef typename wt<T>::C C;
  const int sgc = DAG ? 0 : 2;  // projector 1 + sg gamma_mu: sg = -1 forward (code 2), +1 backward
  // upper half-spinor h[q] = psi_q + phase * psi_perm(q), formed on lanes 0, 1
  const int pq = gperm(MU, q & 1);
  C other[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) other[c] = shfl_c(psi[c], qbase + (q < 2 ? gperm(MU, q) : pq));
  C uh[3];
  if (q < 2) {
    const int code = (gphase(MU, q) + sgc) & 3;
    C h[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) h[c] = cadd(psi[c], cphase(other[c], code));
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      C v{0, 0};
#pragma unroll
      for (int b = 0; b < 3; ++b) v = cadd(v, DAG ? cmulc(U[b * 3 + a], h[b]) : cmul(U[a * 3 + b], h[b]));
      uh[a] = v;
    }
  } else {
#pragma unroll
    for (int a = 0; a < 3; ++a) uh[a] = C{0, 0};
  }
  // lower spins: phase * uh[perm(q)] from lane perm(q) (an upper lane)
  C low[3];
  const int src = q < 2 ? q : gperm(MU, q);
#pragma unroll
  for (int a = 0; a < 3; ++a) low[a] = shfl_c(uh[a], qbase + src);
  if (q < 2) {
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      acc[a].x += coef * uh[a].x;
      acc[a].y += coef * uh[a].y;
    }
  } else {
    const int code = (gphase(MU, q) + sgc) & 3;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const C v = cphase(low[a], code);
      acc[a].x += coef * v.x;
      acc[a].y += coef * v.y;
    }
  }
}

//
// DOTS (op M or MDAG only): also accumulate, per RHS r, d1[r] += <out, in> and
// d2[r].x += <out, out> over all sites -- the two inner products of the
// minimal-residual step -- so the smoother reads neither vector again.  A quad
// folds its lanes with shuffles, the CTA its sites in shared memory, and the
// CTA adds its totals to d1 / d2 (zeroed by the caller) once at the end.
template <class T, bool DOTS>
__global__ void __launch_bounds__(512) wilson_quad_kernel(
    const typename wt<T>::C* __restrict__ gauge, const typename wt<T>::C* __restrict__ clover,
    const int32_t* __restrict__ nbr, const typename wt<T>::C* __restrict__ in,
    typename wt<T>::C* __restrict__ out, int V, int nrhs, int rt, T diag, int op, int dir, int disp,
    int apbc, int tvol, int Lt, double2* __restrict__ d1, double2* __restrict__ d2) {
  typedef typename wt<T>::C C;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* Ls = reinterpret_cast<C*>(smem_raw);  // [kTileSites][8][9]: p < 4 U_mu(x), p >= 4 U_mu(x - mu)
  C* Cs = Ls + kTileSites * 72;            // [kTileSites][72]
  double* Ds = reinterpret_cast<double*>(Cs + kTileSites * 72);  // DOTS: [nrhs][3]
  if (DOTS) {
    for (int k = threadIdx.x; k < 3 * nrhs; k += blockDim.x) Ds[k] = 0.0;
  }
  const bool g5 = (op == GMG_OP_MDAG);
  const int q = threadIdx.x & 3, qbase = threadIdx.x & 31 & ~3;
  const int grp = threadIdx.x >> 2;
  const int sl = grp / rt, rl = grp % rt;
  const int nt = (V + kTileSites - 1) / kTileSites;
  const T sg5 = (g5 && q >= 2) ? (T)-1 : (T)1;
  for (int tile = blockIdx.x; tile < nt; tile += gridDim.x) {
    const int s0 = tile * kTileSites;
    const int ns = min(kTileSites, V - s0);
    __syncthreads();
    for (int k = threadIdx.x; k < ns * 72; k += blockDim.x) {
      const int j = k / 72, e = k % 72, p = e / 9, m = e % 9;
      const int st = s0 + j;
      const int ls = p < 4 ? st : nbr[(int64_t)p * V + st];
      Ls[k] = gauge[((int64_t)ls * 4 + (p & 3)) * 9 + m];
      Cs[k] = clover[(int64_t)s0 * 72 + k];
    }
    __syncthreads();
    // a quad with sl >= ns has no site; it still joins the shuffles (all lanes of
    // a quad agree), reading site s0 harmlessly, and stores nothing
    const bool active = sl < ns;
    const int site = s0 + (active ? sl : 0);
    const int tc = site / tvol;
    const C* Lsite = Ls + (active ? sl : 0) * 72;
    for (int r = rl; r < nrhs; r += rt) {
      C acc[3], cin[3];
#pragma unroll
      for (int c = 0; c < 3; ++c) acc[c] = C{0, 0};
      if (op != GMG_OP_MDIR) {
        const C* src = in + ((int64_t)site * nrhs + r) * 12 + q * 3;
        C psi[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          cin[c] = src[c];
          psi[c] = cin[c];
          psi[c].x *= sg5;
          psi[c].y *= sg5;
        }
        // clover block of this spin's chirality: rows a = (q & 1) * 3 + c, columns over both spins
        C partner[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) partner[c] = shfl_c(psi[c], qbase + (q ^ 1));
        const C* cl = Cs + (active ? sl : 0) * 72 + (q >> 1) * 36;
        const int a0 = (q & 1) * 3;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          C v;
          v.x = diag * psi[c].x;
          v.y = diag * psi[c].y;
#pragma unroll
          for (int b = 0; b < 3; ++b) {
            // block columns 0..2 belong to the even spin of the block, 3..5 to the odd one
            const C lo = (q & 1) ? partner[b] : psi[b];
            const C hi = (q & 1) ? psi[b] : partner[b];
            v = cadd(v, cmul(cl[(a0 + c) * 6 + b], lo));
            v = cadd(v, cmul(cl[(a0 + c) * 6 + 3 + b], hi));
          }
          acc[c] = v;
        }
      }
      if (op != GMG_OP_MDIAG) {
#pragma unroll
        for (int p = 0; p < 8; ++p) {
          const int mu = p & 3, dsp = p < 4 ? 1 : -1;
          if (op == GMG_OP_MDIR && (mu != dir || dsp != disp)) continue;
          const int nb = nbr[(int64_t)p * V + site];
          T coef = (T)-0.5;
          if (apbc && mu == 3 && ((dsp > 0 && tc == Lt - 1) || (dsp < 0 && tc == 0))) coef = (T)0.5;
          const C* src = in + ((int64_t)nb * nrhs + r) * 12 + q * 3;
          C psi[3];
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            psi[c] = src[c];
            psi[c].x *= sg5;
            psi[c].y *= sg5;
          }
          const C* U = Lsite + p * 9;
          switch (p) {
            case 0: quad_hop<T, 0, false>(acc, U, psi, q, qbase, coef); break;
            case 1: quad_hop<T, 1, false>(acc, U, psi, q, qbase, coef); break;
            case 2: quad_hop<T, 2, false>(acc, U, psi, q, qbase, coef); break;
            case 3: quad_hop<T, 3, false>(acc, U, psi, q, qbase, coef); break;
            case 4: quad_hop<T, 0, true>(acc, U, psi, q, qbase, coef); break;
            case 5: quad_hop<T, 1, true>(acc, U, psi, q, qbase, coef); break;
            case 6: quad_hop<T, 2, true>(acc, U, psi, q, qbase, coef); break;
            default: quad_hop<T, 3, true>(acc, U, psi, q, qbase, coef); break;
          }
        }
      }
      double pr = 0.0, pi = 0.0, pn = 0.0;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        acc[c].x *= sg5;
        acc[c].y *= sg5;
        if (DOTS) {
          const double vx = acc[c].x, vy = acc[c].y, ix = cin[c].x, iy = cin[c].y;
          pr += vx * ix + vy * iy;
          pi += vx * iy - vy * ix;
          pn += vx * vx + vy * vy;
        }
      }
      if (active) {
        C* dst = out + ((int64_t)site * nrhs + r) * 12 + q * 3;
#pragma unroll
        for (int c = 0; c < 3; ++c) dst[c] = acc[c];
      }
      if (DOTS) {
#pragma unroll
        for (int m = 1; m <= 2; m <<= 1) {
          pr += __shfl_xor_sync(0xffffffffu, pr, m);
          pi += __shfl_xor_sync(0xffffffffu, pi, m);
          pn += __shfl_xor_sync(0xffffffffu, pn, m);
        }
        if (active && q == 0) {
          atomicAdd(&Ds[3 * r], pr);
          atomicAdd(&Ds[3 * r + 1], pi);
          atomicAdd(&Ds[3 * r + 2], pn);
        }
      }
    }
  }
  if (DOTS) {
    __syncthreads();
    for (int k = threadIdx.x; k < nrhs; k += blockDim.x) {
      atomicAdd(&d1[k].x, Ds[3 * k]);
      atomicAdd(&d1[k].y, Ds[3 * k + 1]);
      atomicAdd(&d2[k].x, Ds[3 * k + 2]);
    }
  }
}

// ---------------------------------------------------------------------------
// clover term from the gauge field (thread per site)
// ---------------------------------------------------------------------------
struct M3 { double2 m[3][3]; };

__device__ __forceinline__ M3 m3_load(const double2* p) {
  M3 r;
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b) r.m[a][b] = p[a * 3 + b];
  return r;
}
__device__ __forceinline__ M3 m3_dag(const M3& a) {
  M3 r;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) r.m[i][j] = make_double2(a.m[j][i].x, -a.m[j][i].y);
  return r;
}
__device__ __forceinline__ M3 m3_mul(const M3& a, const M3& b) {
  M3 r;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      double2 s = make_double2(0, 0);
#pragma unroll
      for (int k = 0; k < 3; ++k) s = cadd(s, cmul(a.m[i][k], b.m[k][j]));
      r.m[i][j] = s;
    }
  return r;
}

__device__ __forceinline__ int shift(int site, const int* L, int d, int disp) {
  int c[4];
  int t = site;
#pragma unroll
  for (int k = 0; k < 4; ++k) { c[k] = t % L[k]; t /= L[k]; }
  c[d] = (c[d] + disp + L[d]) % L[d];
  return c[0] + L[0] * (c[1] + L[1] * (c[2] + L[2] * c[3]));
}

__global__ void clover_kernel(const double2* __restrict__ U, double2* __restrict__ Cl, int V, int L0,
                              int L1, int L2, int L3, double csw) {
  const int L[4] = {L0, L1, L2, L3};
  // gamma matrices as dense 4x4 from the perm/phase tables
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < V; s += gridDim.x * blockDim.x) {
    double2 full[12][12];
#pragma unroll
    for (int a = 0; a < 12; ++a)
#pragma unroll
      for (int b = 0; b < 12; ++b) full[a][b] = make_double2(0, 0);
    for (int mu = 0; mu < 4; ++mu)
      for (int nu = mu + 1; nu < 4; ++nu) {
        const int xpm = shift(s, L, mu, 1), xpn = shift(s, L, nu, 1);
        const int xmm = shift(s, L, mu, -1), xmn = shift(s, L, nu, -1);
        const int xmm_pn = shift(xmm, L, nu, 1), xmm_mn = shift(xmm, L, nu, -1);
        const int xmn_pm = shift(xmn, L, mu, 1);
        auto lk = [&](int site, int d) { return m3_load(U + ((int64_t)site * 4 + d) * 9); };
        M3 q1 = m3_mul(m3_mul(m3_mul(lk(s, mu), lk(xpm, nu)), m3_dag(lk(xpn, mu))), m3_dag(lk(s, nu)));
        M3 q2 = m3_mul(m3_mul(m3_mul(lk(s, nu), m3_dag(lk(xmm_pn, mu))), m3_dag(lk(xmm, nu))), lk(xmm, mu));
        M3 q3 = m3_mul(m3_mul(m3_mul(m3_dag(lk(xmm, mu)), m3_dag(lk(xmm_mn, nu))), lk(xmm_mn, mu)), lk(xmn, nu));
        M3 q4 = m3_mul(m3_mul(m3_mul(m3_dag(lk(xmn, nu)), lk(xmn, mu)), lk(xmn_pm, nu)), m3_dag(lk(s, mu)));
        double2 F[3][3];
        for (int i = 0; i < 3; ++i)
          for (int j = 0; j < 3; ++j) {
            double2 q = cadd(cadd(q1.m[i][j], q2.m[i][j]), cadd(q3.m[i][j], q4.m[i][j]));
            double2 qd = cadd(cadd(q1.m[j][i], q2.m[j][i]), cadd(q3.m[j][i], q4.m[j][i]));
            // (q - conj(qd)) / (8i) = -i/8 (q - conj(qd))
            const double2 d = make_double2(q.x - qd.x, q.y + qd.y);
            F[i][j] = make_double2(d.y / 8.0, -d.x / 8.0);
          }
        // sigma_{mu nu} = (i/2)[g_mu, g_nu]; coefficient -(csw/2)
        for (int si = 0; si < 4; ++si)
          for (int sj = 0; sj < 4; ++sj) {
            // [g_mu g_nu](si,sj) = g_mu(si, perm_mu(si)) g_nu(perm_mu(si), sj)
            double2 com = make_double2(0, 0);
            {
              const int k = c_gperm[mu][si];
              if (c_gperm[nu][k] == sj) com = cadd(com, cphase(make_double2(1, 0), c_gphase[mu][si] + c_gphase[nu][k]));
              const int k2 = c_gperm[nu][si];
              if (c_gperm[mu][k2] == sj) com = cadd(com, cphase(make_double2(-1, 0), c_gphase[nu][si] + c_gphase[mu][k2]));
            }
            if (com.x == 0 && com.y == 0) continue;
            // sig = (i/2) com; factor = -(csw/2) sig = -(i csw/4) com
            const double2 f = cphase(make_double2(-csw * 0.25 * com.x, -csw * 0.25 * com.y), 1);
            for (int ci = 0; ci < 3; ++ci)
              for (int cj = 0; cj < 3; ++cj)
                full[si * 3 + ci][sj * 3 + cj] = cadd(full[si * 3 + ci][sj * 3 + cj], cmul(f, F[ci][cj]));
          }
      }
    for (int blk = 0; blk < 2; ++blk)
      for (int a = 0; a < 6; ++a)
        for (int b = 0; b < 6; ++b)
          Cl[(((int64_t)s * 2 + blk) * 6 + a) * 6 + b] = full[blk * 6 + a][blk * 6 + b];
  }
}

__global__ void d2f_wilson(const double2* __restrict__ a, float2* __restrict__ b, int64_t n) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n;
       e += (int64_t)gridDim.x * blockDim.x)
    b[e] = make_float2((float)a[e].x, (float)a[e].y);
}

gmg_status wilson_build_clover(gmg_wilson* h, cudaStream_t s) {
  const int V = (int)h->dims.vol();
  GMG_TRY(h->clover.alloc(sizeof(double2) * 72 * (size_t)V));
  GMG_TRY(h->clover_f.alloc(sizeof(float2) * 72 * (size_t)V));
  GMG_TRY(h->gauge_f.alloc(sizeof(float2) * 36 * (size_t)V));
  clover_kernel<<<std::min((V + 127) / 128, 148 * 16), 128, 0, s>>>(
      h->gauge.as<double2>(), h->clover.as<double2>(), V, h->dims.d[0], h->dims.d[1], h->dims.d[2],
      h->dims.d[3], h->csw);
  GMG_CUDA(cudaGetLastError());
  d2f_wilson<<<std::min((V * 72 + 255) / 256, 148 * 64), 256, 0, s>>>(h->clover.as<double2>(),
                                                                       h->clover_f.as<float2>(), (int64_t)V * 72);
  d2f_wilson<<<std::min((V * 36 + 255) / 256, 148 * 64), 256, 0, s>>>(h->gauge.as<double2>(),
                                                                       h->gauge_f.as<float2>(), (int64_t)V * 36);
  GMG_CUDA(cudaGetLastError());
  return GMG_OK;
}

// quad kernel launch: kTileSites sites x rt RHS x 4 spin lanes per CTA, rt the
// largest divisor of nrhs up to 8 (at most 512 threads)
template <bool DOTS>
static gmg_status launch_quad(gmg_wilson* h, int op, int dir, int disp, int vec_prec, int nrhs, const void* in,
                              void* out, double2* d1, double2* d2, cudaStream_t s) {
  const int V = (int)h->dims.vol();
  const int tvol = h->dims.d[0] * h->dims.d[1] * h->dims.d[2];
  int rt = 1;
  for (int c = std::min(nrhs, 8); c >= 1; --c)
    if (nrhs % c == 0) {
      rt = c;
      break;
    }
  const int threads = kTileSites * rt * 4;
  const int tiles = (V + kTileSites - 1) / kTileSites;
  // about 2048 resident threads per SM
  const int g = std::min(tiles, 148 * std::max(1, 2048 / threads));
  const size_t dots = DOTS ? sizeof(double) * 3 * (size_t)nrhs : 0;
  if (vec_prec == GMG_F64) {
    const size_t smem = sizeof(double2) * 2 * kTileSites * 72 + dots;
    if (smem > 48 * 1024)
      GMG_CUDA(cudaFuncSetAttribute(wilson_quad_kernel<double, DOTS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)smem));
    wilson_quad_kernel<double, DOTS><<<g, threads, smem, s>>>(
        h->gauge.as<double2>(), h->clover.as<double2>(), h->nbr.as<int32_t>(), (const double2*)in, (double2*)out, V,
        nrhs, rt, 4.0 + h->mass, op, dir, disp, h->apbc, tvol, h->dims.d[3], d1, d2);
  } else if (vec_prec == GMG_F32) {
    const size_t smem = sizeof(float2) * 2 * kTileSites * 72 + dots;
    if (smem > 48 * 1024)
      GMG_CUDA(cudaFuncSetAttribute(wilson_quad_kernel<float, DOTS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)smem));
    wilson_quad_kernel<float, DOTS><<<g, threads, smem, s>>>(
        h->gauge_f.as<float2>(), h->clover_f.as<float2>(), h->nbr.as<int32_t>(), (const float2*)in, (float2*)out, V,
        nrhs, rt, (float)(4.0 + h->mass), op, dir, disp, h->apbc, tvol, h->dims.d[3], d1, d2);
  } else {
    return fail(GMG_ERR_UNSUPPORTED, "wilson apply: vectors must be F64 or F32");
  }
  GMG_CUDA(cudaGetLastError());
  return GMG_OK;
}

gmg_status wilson_apply(gmg_wilson* h, int op, int dir, int disp, int vec_prec, int nrhs,
                        const void* in, void* out, cudaStream_t s) {
  const int V = (int)h->dims.vol();
  const int tvol = h->dims.d[0] * h->dims.d[1] * h->dims.d[2];
  const int64_t total = (int64_t)V * nrhs;
  const int grid = (int)std::min<int64_t>((total + 127) / 128, 148 * 32);
  KernelTimer kt("wilson", s);
  if (nrhs >= 4) return launch_quad<false>(h, op, dir, disp, vec_prec, nrhs, in, out, nullptr, nullptr, s);
  if (vec_prec == GMG_F64) {
    wilson_kernel<double><<<grid, 128, 0, s>>>(h->gauge.as<double2>(), h->clover.as<double2>(),
                                                h->nbr.as<int32_t>(), (const double2*)in, (double2*)out, V,
                                                nrhs, 4.0 + h->mass, op, dir, disp, h->apbc, tvol,
                                                h->dims.d[3]);
  } else if (vec_prec == GMG_F32) {
    wilson_kernel<float><<<grid, 128, 0, s>>>(h->gauge_f.as<float2>(), h->clover_f.as<float2>(),
                                               h->nbr.as<int32_t>(), (const float2*)in, (float2*)out, V,
                                               nrhs, (float)(4.0 + h->mass), op, dir, disp, h->apbc, tvol,
                                               h->dims.d[3]);
  } else {
    return fail(GMG_ERR_UNSUPPORTED, "wilson apply: vectors must be F64 or F32");
  }
  GMG_CUDA(cudaGetLastError());
  return GMG_OK;
}

// out = M in, and the minimal-residual inner products d1[r] = <out, in>,
// d2[r].x = <out, out> (d1, d2: nrhs entries each, zeroed here)
gmg_status wilson_apply_mr(gmg_wilson* h, int vec_prec, int nrhs, const void* in, void* out, double2* d1,
                           double2* d2, cudaStream_t s) {
  KernelTimer kt("wilson", s);
  GMG_CUDA(cudaMemsetAsync(d1, 0, sizeof(double2) * nrhs, s));
  GMG_CUDA(cudaMemsetAsync(d2, 0, sizeof(double2) * nrhs, s));
  return launch_quad<true>(h, GMG_OP_M, 0, 0, vec_prec, nrhs, in, out, d1, d2, s);
}

}  // namespace gmg

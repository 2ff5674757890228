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
#include <type_traits>

#include <cuda_bf16.h>
#include <vector>

#include "async_copy.cuh"
#include "gmg_internal.cuh"

namespace gmg {

template <class T> struct wt;
template <> struct wt<double> { typedef double2 C; };
template <> struct wt<float> { typedef float2 C; };
// BF16 storage of a complex number: one 32-bit word, real part in the low
// 16 bits (the fine smoother's residual fields; arithmetic in FP32)
struct bf16s {};
template <> struct wt<bf16s> { typedef uint32_t C; };

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
// acc + a b and acc + conj(a) b as four fused multiply-adds (written out so that
// no product is rounded separately and no add is left over)
template <class C> __device__ __forceinline__ C cfma(C a, C b, C acc) {
  acc.x = fma(a.x, b.x, acc.x);
  acc.x = fma(-a.y, b.y, acc.x);
  acc.y = fma(a.x, b.y, acc.y);
  acc.y = fma(a.y, b.x, acc.y);
  return acc;
}
template <class C> __device__ __forceinline__ C cfmac(C a, C b, C acc) {
  acc.x = fma(a.x, b.x, acc.x);
  acc.x = fma(a.y, b.y, acc.x);
  acc.y = fma(a.x, b.y, acc.y);
  acc.y = fma(-a.y, b.x, acc.y);
  return acc;
}
// FP64: the product and the add as written (the fused form measured slower in
// the FP64 kernels: more registers live, 7.39 -> 7.80 ms at 32^4 x 24 RHS)
template <> __device__ __forceinline__ double2 cfma<double2>(double2 a, double2 b, double2 acc) {
  return cadd(acc, cmul(a, b));
}
template <> __device__ __forceinline__ double2 cfmac<double2>(double2 a, double2 b, double2 acc) {
  return cadd(acc, cmulc(a, b));
}
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
        if (!dagger) acc = cfma(U[a * 3 + b], h[s][b], acc);
        else acc = cfmac(U[b * 3 + a], h[s][b], acc);
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
// (p < 4: U_mu(x), p >= 4: U_mu(x - mu), applied daggered unless LDAG says the
// links come daggered already); cl: the site's
// two 6x6 clover blocks.
// 12 complex numbers of one (site, RHS) record.  VEC 2: 32-byte accesses
// (ld/st .v8.f32 / .v4.f64; the record start is 32-byte aligned), so that
// every access covers one whole 32-byte sector; VEC 1: 16-byte accesses (the
// record start is 16-byte aligned); VEC 0: one access per complex number.
template <class T, int VEC>
__device__ __forceinline__ void ld12(typename wt<T>::C v[12], const typename wt<T>::C* __restrict__ p) {
  if (VEC == 2 && sizeof(T) == 4) {
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      float r[8];
      asm volatile("ld.global.nc.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                   : "=f"(r[0]), "=f"(r[1]), "=f"(r[2]), "=f"(r[3]), "=f"(r[4]), "=f"(r[5]), "=f"(r[6]), "=f"(r[7])
                   : "l"(reinterpret_cast<const float*>(p) + 8 * k));
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        v[4 * k + i].x = (T)r[2 * i];
        v[4 * k + i].y = (T)r[2 * i + 1];
      }
    }
  } else if (VEC == 2) {
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      double r[4];
      asm volatile("ld.global.nc.v4.f64 {%0,%1,%2,%3}, [%4];"
                   : "=d"(r[0]), "=d"(r[1]), "=d"(r[2]), "=d"(r[3])
                   : "l"(reinterpret_cast<const double*>(p) + 4 * k));
      v[2 * k].x = (T)r[0];
      v[2 * k].y = (T)r[1];
      v[2 * k + 1].x = (T)r[2];
      v[2 * k + 1].y = (T)r[3];
    }
  } else if (VEC == 1 && sizeof(T) == 4) {
    const float4* q = reinterpret_cast<const float4*>(p);
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      const float4 a = q[k];
      v[2 * k].x = a.x;
      v[2 * k].y = a.y;
      v[2 * k + 1].x = a.z;
      v[2 * k + 1].y = a.w;
    }
  } else {
#pragma unroll
    for (int k = 0; k < 12; ++k) v[k] = p[k];
  }
}
template <class T, int VEC>
__device__ __forceinline__ void st12(typename wt<T>::C* __restrict__ p, const typename wt<T>::C v[12]) {
  if (VEC == 2 && sizeof(T) == 4) {
#pragma unroll
    for (int k = 0; k < 3; ++k)
      asm volatile("st.global.v8.f32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};" ::"l"(reinterpret_cast<float*>(p) + 8 * k),
                   "f"((float)v[4 * k].x), "f"((float)v[4 * k].y), "f"((float)v[4 * k + 1].x),
                   "f"((float)v[4 * k + 1].y), "f"((float)v[4 * k + 2].x), "f"((float)v[4 * k + 2].y),
                   "f"((float)v[4 * k + 3].x), "f"((float)v[4 * k + 3].y)
                   : "memory");
  } else if (VEC == 2) {
#pragma unroll
    for (int k = 0; k < 6; ++k)
      asm volatile("st.global.v4.f64 [%0], {%1,%2,%3,%4};" ::"l"(reinterpret_cast<double*>(p) + 4 * k),
                   "d"((double)v[2 * k].x), "d"((double)v[2 * k].y), "d"((double)v[2 * k + 1].x),
                   "d"((double)v[2 * k + 1].y)
                   : "memory");
  } else if (VEC == 1 && sizeof(T) == 4) {
    float4* q = reinterpret_cast<float4*>(p);
#pragma unroll
    for (int k = 0; k < 6; ++k) q[k] = make_float4(v[2 * k].x, v[2 * k].y, v[2 * k + 1].x, v[2 * k + 1].y);
  } else {
#pragma unroll
    for (int k = 0; k < 12; ++k) p[k] = v[k];
  }
}

// Record (site, r) of a field: [V][nrhs][12] complex numbers, or for BF16
// fields with VEC 3 the site-blocked layout [V][3][nrhs][4] words, in which
// the 16-byte quarter g of the records of one site's right-hand sides lie
// back to back, so that the lanes of a warp that hold consecutive RHS of a
// site read one contiguous run (three 16-byte loads of a record at a stride
// of 4 nrhs words).
template <int VEC, class P>
__device__ __forceinline__ P* recp(P* base, int64_t site, int r, int nrhs) {
  return VEC == 3 ? base + site * 12 * nrhs + 4 * r : base + (site * nrhs + r) * 12;
}

// a record of input type TI read as T: FP32 records promoted exactly to FP64
// on load (the FP64 operator applied to FP32 vectors), BF16 records (48 bytes,
// three 16-byte loads) widened to FP32
// A record as loaded, before widening: BF16 records stay packed (12 words), so
// that a record prefetched one hop ahead holds 12 registers instead of 24.
template <class T, class TI> struct RawRec { typedef typename wt<T>::C type; };
template <class T> struct RawRec<T, bf16s> { typedef uint32_t type; };

template <class T, class TI, int VEC>
__device__ __forceinline__ void ld12x(typename wt<T>::C v[12], const typename wt<TI>::C* __restrict__ base,
                                      int64_t site, int r, int nrhs);

template <class T, class TI, int VEC>
__device__ __forceinline__ void ld12raw(typename RawRec<T, TI>::type w[12],
                                        const typename wt<TI>::C* __restrict__ base, int64_t site, int r, int nrhs) {
  if constexpr (std::is_same<TI, bf16s>::value) {
    // VEC 3: 32-bit index arithmetic in 16-byte units (the caller keeps the
    // field below 2^31 of them)
    const uint4* q = VEC == 3 ? reinterpret_cast<const uint4*>(base) + ((int)site * 3 * nrhs + r)
                              : reinterpret_cast<const uint4*>(recp<VEC>(base, site, r, nrhs));
    const int gs = VEC == 3 ? nrhs : 1;  // uint4 stride of the three quarters
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const uint4 u = __ldg(q + k * gs);
      w[4 * k] = u.x;
      w[4 * k + 1] = u.y;
      w[4 * k + 2] = u.z;
      w[4 * k + 3] = u.w;
    }
  } else {
    ld12x<T, TI, VEC>(w, base, site, r, nrhs);
  }
}

template <class T, class TI>
__device__ __forceinline__ void unraw12(typename wt<T>::C v[12], const typename RawRec<T, TI>::type w[12]) {
#pragma unroll
  for (int i = 0; i < 12; ++i) {
    if constexpr (std::is_same<TI, bf16s>::value)
      v[i] = typename wt<T>::C{(T)__uint_as_float(w[i] << 16), (T)__uint_as_float(w[i] & 0xffff0000u)};
    else
      v[i] = w[i];
  }
}

template <class T, class TI, int VEC>
__device__ __forceinline__ void ld12x(typename wt<T>::C v[12], const typename wt<TI>::C* __restrict__ base,
                                      int64_t site, int r, int nrhs) {
  const typename wt<TI>::C* p = recp<VEC>(base, site, r, nrhs);
  if constexpr (std::is_same<TI, bf16s>::value) {
    uint32_t w[12];
    ld12raw<T, TI, VEC>(w, base, site, r, nrhs);
    unraw12<T, TI>(v, w);
  } else if (sizeof(TI) == sizeof(T)) {
    ld12<T, VEC>(v, reinterpret_cast<const typename wt<T>::C*>(p));
  } else {
    float2 f[12];
    ld12<float, VEC>(f, reinterpret_cast<const float2*>(p));
#pragma unroll
    for (int k = 0; k < 12; ++k) v[k] = typename wt<T>::C{(T)f[k].x, (T)f[k].y};
  }
}

// a record of T written as TO (BF16: rounded to nearest even, three 16-byte stores)
template <class T, class TO, int VEC>
__device__ __forceinline__ void st12x(typename wt<TO>::C* __restrict__ base, int64_t site, int r, int nrhs,
                                      const typename wt<T>::C v[12]) {
  typename wt<TO>::C* p = recp<VEC>(base, site, r, nrhs);
  if (std::is_same<TO, bf16s>::value) {
    uint4* q = reinterpret_cast<uint4*>(p);
    const int gs = VEC == 3 ? nrhs : 1;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      uint32_t w[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const __nv_bfloat162 b = __floats2bfloat162_rn((float)v[4 * k + i].x, (float)v[4 * k + i].y);
        w[i] = *reinterpret_cast<const uint32_t*>(&b);
      }
      q[k * gs] = make_uint4(w[0], w[1], w[2], w[3]);
    }
  } else {
    st12<T, VEC>(reinterpret_cast<typename wt<T>::C*>(p), v);
  }
}

// DOTS (op M or MDAG): also add <out, in> and <out, out> of this (site, r) to
// dsum[0..1] and dsum[2].  VEC: 16-byte spinor accesses.  skip: hops p with
// bit p set are left out (0 for the plain operator); with the bits of the
// hops to blocks of the other parity this gives e D e + o D o of the
// coarsening's self term in one pass.
// VOUT: the output record layout (VEC by default); SUB: write bsub - M in
// (bsub laid out and typed as the input) instead of M in.
// NBS: nbr is a tile's staged neighbour table, entry p of this site at
// nbr[p * nbs_stride + nbs_i] (instead of nbr[p * V + site]).
template <class T, class LinkFn, bool DOTS = false, int VEC = 0, bool LDAG = false, bool PF = false, class TI = T,
          class TO = T, int VOUT = VEC, bool SUB = false, bool NBS = false>
__device__ __forceinline__ void wilson_site(const typename wt<T>::C* __restrict__ cl, LinkFn links,
                                            const int32_t* __restrict__ nbr, const typename wt<TI>::C* __restrict__ in,
                                            typename wt<TO>::C* __restrict__ out, int V, int nrhs, int site, int r,
                                            T diag, int op, int dir, int disp, int apbc, int tvol, int Lt,
                                            double* dsum = nullptr, int skip = 0,
                                            const typename wt<TI>::C* __restrict__ bsub = nullptr, int nbs_stride = 0,
                                            int nbs_i = 0) {
  typedef typename wt<T>::C C;
  auto nbidx = [&](int p) -> int {
    if constexpr (NBS)
      return nbr[p * nbs_stride + nbs_i];
    else
      return nbr[(int64_t)p * V + site];
  };
  const bool g5 = (op == GMG_OP_MDAG);
  const int tc = site / tvol;
  C acc[4][3];
  C cin[12];
#pragma unroll
  for (int s = 0; s < 4; ++s)
#pragma unroll
    for (int c = 0; c < 3; ++c) acc[s][c] = C{0, 0};
  if (PF && (op == GMG_OP_M || op == GMG_OP_MDAG)) {
    // the full operator with the neighbour records software-pipelined: the
    // eight neighbour indices first, then each hop's record is requested one
    // hop ahead (the first one before the clover term), so that a record's
    // latency overlaps the previous hop's arithmetic
    int nbs[8];
#pragma unroll
    for (int p = 0; p < 8; ++p) nbs[p] = nbidx(p);
    C psi[12];
    typename RawRec<T, TI>::type nxt[12];
    ld12x<T, TI, VEC>(psi, in, site, r, nrhs);
    ld12raw<T, TI, VEC>(nxt, in, nbs[0], r, nrhs);
#pragma unroll
    for (int k = 6; k < 12; ++k)
      if (g5) psi[k] = C{-psi[k].x, -psi[k].y};
#pragma unroll
    for (int blk = 0; blk < 2; ++blk)
#pragma unroll
      for (int a = 0; a < 6; ++a) {
        C v;
        v.x = diag * psi[blk * 6 + a].x;
        v.y = diag * psi[blk * 6 + a].y;
#pragma unroll
        for (int b = 0; b < 6; ++b) v = cfma(cl[(blk * 6 + a) * 6 + b], psi[blk * 6 + b], v);
        acc[(blk * 6 + a) / 3][(blk * 6 + a) % 3] = v;
      }
#pragma unroll
    for (int p = 0; p < 8; ++p) {
      const int mu = p & 3;
      const int dsp = p < 4 ? 1 : -1;
      C cur[12];
      unraw12<T, TI>(cur, nxt);
      if (p < 7) ld12raw<T, TI, VEC>(nxt, in, nbs[p < 7 ? p + 1 : 7], r, nrhs);
      if (skip & (1 << p)) continue;
      T coef = (T)-0.5;
      if (apbc && mu == 3 && ((dsp > 0 && tc == Lt - 1) || (dsp < 0 && tc == 0))) coef = (T)0.5;
      if (g5) {
#pragma unroll
        for (int k = 6; k < 12; ++k) cur[k] = C{-cur[k].x, -cur[k].y};
      }
      wilson_hop<T>(acc, links(p, nbs[p]), dsp < 0 && !LDAG, cur, mu, dsp, coef);
    }
  } else {
  if (op != GMG_OP_MDIR) {
    // diagonal: (4 + m) psi + Cl psi, two chiral 6x6 blocks
    C psi[12];
    ld12x<T, TI, VEC>(psi, in, site, r, nrhs);
#pragma unroll
    for (int k = 0; k < 12; ++k) {
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
        for (int b = 0; b < 6; ++b) v = cfma(cl[(blk * 6 + a) * 6 + b], psi[blk * 6 + b], v);
        acc[(blk * 6 + a) / 3][(blk * 6 + a) % 3] = v;
      }
  }
  if (op != GMG_OP_MDIAG) {
#pragma unroll
    for (int p = 0; p < 8; ++p) {
      const int mu = p & 3;
      const int dsp = p < 4 ? 1 : -1;
      if (op == GMG_OP_MDIR && (mu != dir || dsp != disp)) continue;
      if (skip & (1 << p)) continue;
      const int nb = nbidx(p);
      T coef = (T)-0.5;
      if (apbc && mu == 3 && ((dsp > 0 && tc == Lt - 1) || (dsp < 0 && tc == 0))) coef = (T)0.5;
      C psi[12];
      ld12x<T, TI, VEC>(psi, in, nb, r, nrhs);
      if (g5) {
#pragma unroll
        for (int k = 6; k < 12; ++k) { psi[k].x = -psi[k].x; psi[k].y = -psi[k].y; }
      }
      wilson_hop<T>(acc, links(p, nb), dsp < 0 && !LDAG, psi, mu, dsp, coef);
    }
  }
  }
  // per-record partial products in T (12 terms), accumulated in FP64 by the caller
  T pr = 0, pi = 0, pn = 0;
  C ov[12];
  // the input record again for the products (re-read rather than kept live
  // through the hops: registers decide the occupancy of this kernel)
  if (DOTS) ld12x<T, TI, VEC>(cin, in, site, r, nrhs);
  if (SUB) ld12x<T, TI, VEC>(ov, bsub, site, r, nrhs);
#pragma unroll
  for (int s = 0; s < 4; ++s)
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      C v = acc[s][c];
      if (g5 && s >= 2) { v.x = -v.x; v.y = -v.y; }
      if (SUB) {
        v.x = ov[s * 3 + c].x - v.x;
        v.y = ov[s * 3 + c].y - v.y;
      }
      ov[s * 3 + c] = v;
      if (DOTS) {
        const T ix = cin[s * 3 + c].x, iy = cin[s * 3 + c].y;
        pr += v.x * ix + v.y * iy;
        pi += v.x * iy - v.y * ix;
        pn += v.x * v.x + v.y * v.y;
      }
    }
  st12x<T, TO, VOUT>(out, site, r, nrhs, ov);
  if (DOTS) {
    dsum[0] += pr;
    dsum[1] += pi;
    dsum[2] += pn;
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

constexpr int kTileSites = 16;

// bytes of one staging buffer of the tile kernel for link / clover entries of
// csize bytes: the tile's hop links and clover blocks and, without SEL, its
// neighbour table
__host__ __device__ constexpr int tile_stage_bytes(int csize, bool sel) {
  return csize * 2 * kTileSites * 72 + (sel ? 0 : 4 * 8 * kTileSites);
}
// shared memory of a tile kernel launch (dots: the DOTS products' bytes)
constexpr size_t tile_smem(int csize, bool sel, size_t dots) {
  return (size_t)(sel ? 1 : 2) * tile_stage_bytes(csize, sel) + dots;
}

// Multi-RHS tile kernel: a CTA takes kTileSites consecutive sites and all
// right-hand sides (rt threads per site, each looping over its RHS); the
// sites' 8 hop links, clover blocks and neighbour indices are staged in
// shared memory once and read by every RHS of the tile, the next tile's copied
// (cp.async) into a second buffer while this one computes.  Thread per (site,
// RHS) otherwise, spinors read from global memory.
// SEL (the coarsening's self term, compiled separately): the tiles run over
// the nsel sites of the list `sel` (all V sites when null) and only those are
// written; hskip (per site, bit p: leave hop p out) restricts the hops to
// neighbours of the same block parity (see wilson_site).
// PF: the neighbour records are software-pipelined (see wilson_site).  (A
// z-blocked tile order, as the staged kernel uses, measured no different here:
// 2.73-2.79 ms at 32^4 x 24 RHS FP32 for z blocks of 1 to 32 planes.)
// TI: the input vectors' precision (float with T = double: the FP64 operator
// on FP32 vectors, promoted on load).
// VOUT, SUB: the output layout and bsub - M in (see wilson_site).
template <class T, bool DOTS, int MINB, bool SEL = false, int VEC = 1, bool PF = false, class TI = T, class TO = T,
          int VOUT = VEC, bool SUB = false>
__global__ void __launch_bounds__(256, MINB) wilson_tile_kernel(
    const typename wt<T>::C* __restrict__ hop, const typename wt<T>::C* __restrict__ clover,
    const int32_t* __restrict__ nbr, const typename wt<TI>::C* __restrict__ in,
    typename wt<TO>::C* __restrict__ out, int V, int nrhs, int rt, T diag, int op, int dir, int disp,
    int apbc, int tvol, int Lt, double2* __restrict__ d1, double2* __restrict__ d2,
    const int32_t* __restrict__ sel = nullptr, int nsel = 0, const uint8_t* __restrict__ hskip = nullptr,
    const typename wt<TI>::C* __restrict__ bsub = nullptr) {
  typedef typename wt<T>::C C;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  // staging buffers (tile_stage_bytes each; two without SEL, the next tile's
  // filled while this one is computed): [kTileSites][8][9] hop links (p < 4
  // U_mu(x), p >= 4 U_mu(x - mu)^dagger), [kTileSites][72] clover and, without
  // SEL, the [8][kTileSites] neighbour table; then DOTS: [nrhs][3] products
  constexpr int kBuf = tile_stage_bytes(sizeof(C), SEL);
  double* Ds = reinterpret_cast<double*>(smem_raw + (SEL ? 1 : 2) * kBuf);
  if (DOTS)
    for (int k = threadIdx.x; k < 3 * nrhs; k += blockDim.x) Ds[k] = 0.0;
  const int nsites = (SEL && sel) ? nsel : V;
  const int nt = (nsites + kTileSites - 1) / kTileSites;
  const int sl = threadIdx.x / rt, rl = threadIdx.x % rt;
  const bool two = nrhs <= 2 * rt;
  double da[3] = {0.0, 0.0, 0.0}, db[3] = {0.0, 0.0, 0.0};
  // the tile's sites from buffer buf (links Ls, clover Cs, neighbour table Ns or nullptr)
  auto compute = [&](int tile, const C* Ls, const C* Cs, const int32_t* Ns) {
    const int s0 = tile * kTileSites;
    const int ns = min(kTileSites, nsites - s0);
    if (sl < ns) {
      const int site = (SEL && sel) ? sel[s0 + sl] : s0 + sl;
      const int skip = (SEL && hskip) ? hskip[site] : 0;
      const C* lsite = Ls + sl * 72;
      auto links = [&](int p, int) -> const C* { return lsite + p * 9; };
      // with two RHS or fewer per thread (rl, rl + rt) the thread owns them for
      // the whole launch and its products stay in registers until the end
      int k = 0;
      for (int r = rl; r < nrhs; r += rt, ++k) {
        double dt[3] = {0.0, 0.0, 0.0};
        wilson_site<T, decltype(links), DOTS, VEC, true, PF, TI, TO, VOUT, SUB, !SEL>(
            Cs + sl * 72, links, SEL ? nbr : Ns, in, out, V, nrhs, site, r, diag, op, dir, disp, apbc, tvol, Lt, dt,
            skip, bsub, kTileSites, sl);
        if (DOTS) {
          if (two) {
#pragma unroll
            for (int c = 0; c < 3; ++c) {
              if (k == 0)
                da[c] += dt[c];
              else
                db[c] += dt[c];
            }
          } else {
            atomicAdd(&Ds[3 * r], dt[0]);
            atomicAdd(&Ds[3 * r + 1], dt[1]);
            atomicAdd(&Ds[3 * r + 2], dt[2]);
          }
        }
      }
    }
  };
  if constexpr (SEL) {
    C* Ls = reinterpret_cast<C*>(smem_raw);
    C* Cs = Ls + kTileSites * 72;
    for (int tile = blockIdx.x; tile < nt; tile += gridDim.x) {
      const int s0 = tile * kTileSites;
      const int ns = min(kTileSites, nsites - s0);
      __syncthreads();
      for (int k = threadIdx.x; k < ns * 72; k += blockDim.x) {
        const int64_t st = sel ? sel[s0 + k / 72] : s0 + k / 72;
        Ls[k] = hop[st * 72 + k % 72];
        Cs[k] = clover[st * 72 + k % 72];
      }
      __syncthreads();
      compute(tile, Ls, Cs, nullptr);
    }
  } else {
    // cp.async copies of a tile's links, clover (16-byte pieces: a site's 72
    // entries are a multiple of 16 bytes, the arrays 16-byte aligned) and
    // neighbour indices (4-byte pieces) into buffer b; one copy group per call,
    // empty past the last tile
    auto stage = [&](int tile, int b) {
      if (tile < nt) {
        const int s0 = tile * kTileSites;
        const int ns = min(kTileSites, nsites - s0);
        unsigned char* base = smem_raw + b * kBuf;
        const int n16 = ns * 72 * (int)sizeof(C) / 16;
        const unsigned char* hs = reinterpret_cast<const unsigned char*>(hop + (int64_t)s0 * 72);
        const unsigned char* cs = reinterpret_cast<const unsigned char*>(clover + (int64_t)s0 * 72);
        unsigned char* cd = base + kTileSites * 72 * sizeof(C);
        for (int k = threadIdx.x; k < n16; k += blockDim.x) {
          ac::cpa16(base + 16 * k, hs + 16 * k);
          ac::cpa16(cd + 16 * k, cs + 16 * k);
        }
        int32_t* nd = reinterpret_cast<int32_t*>(base + 2 * kTileSites * 72 * sizeof(C));
        for (int k = threadIdx.x; k < 8 * ns; k += blockDim.x) {
          const int p = k / ns, j = k - p * ns;
          ac::cpa4(nd + p * kTileSites + j, nbr + (int64_t)p * V + s0 + j);
        }
      }
      ac::cpa_commit();
    };
    int b = 0;
    stage(blockIdx.x, 0);
    for (int tile = blockIdx.x; tile < nt; tile += gridDim.x, b ^= 1) {
      stage(tile + gridDim.x, b ^ 1);  // buffer b ^ 1 was last read before the previous iteration's final barrier
      ac::cpa_wait<1>();               // this thread's copies of this tile have landed
      __syncthreads();                 // everyone's have
      const unsigned char* base = smem_raw + b * kBuf;
      const C* Ls = reinterpret_cast<const C*>(base);
      compute(tile, Ls, Ls + kTileSites * 72, reinterpret_cast<const int32_t*>(base + 2 * kTileSites * 72 * sizeof(C)));
      __syncthreads();  // buffer b is read: the next iteration's staging may overwrite it
    }
    ac::cpa_wait<0>();
  }
  if (DOTS) {
    if (two) {
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        if (rl < nrhs) atomicAdd(&Ds[3 * rl + c], da[c]);
        if (rl + rt < nrhs) atomicAdd(&Ds[3 * (rl + rt) + c], db[c]);
      }
    }
    __syncthreads();
    for (int k = threadIdx.x; k < nrhs; k += blockDim.x) {
      atomicAdd(&d1[k].x, Ds[3 * k]);
      atomicAdd(&d1[k].y, Ds[3 * k + 1]);
      atomicAdd(&d2[k].x, Ds[3 * k + 2]);
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
      for (int b = 0; b < 3; ++b) v = DAG ? cfmac(U[b * 3 + a], h[b], v) : cfma(U[a * 3 + b], h[b], v);
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
            v = cfma(cl[(a0 + c) * 6 + b], lo, v);
            v = cfma(cl[(a0 + c) * 6 + 3 + b], hi, v);
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
// Pipelined staged multi-RHS kernel (variant GMG_WILSON_STAGED).
//
// A work item is a tile of kPipeTS = 4 consecutive sites and a chunk of up to
// CMAX consecutive right-hand sides.  Every distinct neighbour record of the
// tile -- (site, chunk) is chunk x 12 complex numbers, contiguous in the
// [V][nrhs][12] layout -- is brought into its own shared-memory slot by one
// bulk copy (cp.async.bulk), together with the tile's hop links, clover
// blocks and plan entry.  One producer warp fills a ring of stages, each
// tracked by an mbarrier transaction count (full[s]); the consumer warps
// compute from a full stage and release it (empty[s]), so the copies of the
// next stages overlap the arithmetic of this one.  CTAs are persistent (one
// per SM) and walk the items in plan order: tiles sorted by (z block, t, z,
// y, x), so that a record shared with the t and z neighbours of its site is
// still in L2 when they are processed.
//
// Consumer lanes: lane bit 4 is the role h.  h = 0 applies the four forward
// hops and the upper chiral clover block, h = 1 the four backward hops and
// the lower block.  Both roles run one instruction stream (the backward hop
// links are stored daggered, and the projector's sign is a factor), and the
// two halves of an output record meet through one shuffle exchange.  The
// other lane bits pick (site, RHS) so that the 16-byte shared-memory reads of
// a quarter warp fall on distinct banks: 2 sites x 4 RHS (FP32) or 4 sites x
// 2 RHS (FP64), with the slots padded to an odd number of 16-byte units.
constexpr int kPipeTS = 4;
constexpr int kPipeSMax = 7 * kPipeTS + 4;
constexpr int kPipeMaxStages = 4;
constexpr int kPipeHead = 256;  // mbarriers at the start of the dynamic shared memory

// plan entry of one tile (48 bytes, copied into the stage with the records)
struct PipeTile {
  int32_t s0, ns, nss, pad;
  uint8_t slot[kPipeTS * 8];  // slot of the record of hop p of tile site j: slot[j * 8 + p]
};
static_assert(sizeof(PipeTile) == 48, "plan entry size");

// CMAX: RHS per chunk; WARPS: consumer warps of one group (16 (site, RHS)
// items per warp); GMAX: most consumer groups, each computing its own stage
template <class T> struct PipeCfg;
// (several groups measured slower: the stages' bulk copies, not the
// arithmetic, bound this kernel, and more groups leave fewer stages to fill)
template <> struct PipeCfg<float> { static constexpr int CMAX = 24, WARPS = 6, GMAX = 1; };
template <> struct PipeCfg<double> { static constexpr int CMAX = 16, WARPS = 4, GMAX = 1; };

template <class T>
struct PipeGeo {
  typedef typename wt<T>::C C;
  static constexpr int LREC = 72 * (int)sizeof(C) + 16;  // links / clover stride per site
  static constexpr int OFF_LINKS = 48;
  static constexpr int OFF_CLOV = OFF_LINKS + kPipeTS * LREC;
  static constexpr int OFF_SLOTS = OFF_CLOV + kPipeTS * LREC;
  static constexpr int MAX_THREADS = (PipeCfg<T>::WARPS * PipeCfg<T>::GMAX + 1) * 32;
  static_assert((LREC / 16) % 2 == 1, "odd 16-byte stride");
  static_assert(PipeCfg<T>::WARPS * 16 == kPipeTS * PipeCfg<T>::CMAX, "16 (site, RHS) items per warp");
  // slot stride for a chunk of ch RHS: an odd number of 16-byte units
  __host__ __device__ static int srec(int ch) { return ch * 12 * (int)sizeof(C) + 16; }
  __host__ __device__ static int stage_bytes(int ch, int smax) { return OFF_SLOTS + smax * srec(ch); }
};

// One hop with a compile-time direction for either role: the projected
// half spinor (1 + sgn gamma_MU) psi, times the link U (already daggered for
// backward hops), accumulated with coef into the upper spins and, through the
// projector's rank-2 structure, into the lower ones.  sgn = -1 for the
// forward hop (disp +1), +1 for the backward hop.
template <class T, int MU>
__device__ __forceinline__ void pipe_hop(typename wt<T>::C acc[4][3], const typename wt<T>::C* __restrict__ U,
                                         const typename wt<T>::C psi[12], T sgn, T coef) {
  typedef typename wt<T>::C C;
  C hh[2][3];
#pragma unroll
  for (int s = 0; s < 2; ++s) {
    const int ps = gperm(MU, s), code = gphase(MU, s) & 3;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const C v = cphase(psi[ps * 3 + c], code);
      hh[s][c] = C{psi[s * 3 + c].x + sgn * v.x, psi[s * 3 + c].y + sgn * v.y};
    }
  }
  C uh[2][3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const C u0 = U[a * 3], u1 = U[a * 3 + 1], u2 = U[a * 3 + 2];
#pragma unroll
    for (int s = 0; s < 2; ++s) uh[s][a] = cfma(u2, hh[s][2], cfma(u1, hh[s][1], cfma(u0, hh[s][0], C{0, 0})));
  }
#pragma unroll
  for (int s = 0; s < 2; ++s)
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      acc[s][a].x += coef * uh[s][a].x;
      acc[s][a].y += coef * uh[s][a].y;
    }
  const T cl = coef * sgn;
#pragma unroll
  for (int s = 2; s < 4; ++s) {
    const int ps = gperm(MU, s), code = gphase(MU, s) & 3;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const C v = cphase(uh[ps][a], code);
      acc[s][a].x += cl * v.x;
      acc[s][a].y += cl * v.y;
    }
  }
}

template <class T>
__device__ __forceinline__ void load_spinor(typename wt<T>::C* psi, const unsigned char* p, int n) {
  typedef typename wt<T>::C C;
  if (sizeof(T) == 4) {
    const float4* q = reinterpret_cast<const float4*>(p);
#pragma unroll
    for (int k = 0; k < n / 2; ++k) {
      const float4 v = q[k];
      psi[2 * k] = C{(T)v.x, (T)v.y};
      psi[2 * k + 1] = C{(T)v.z, (T)v.w};
    }
  } else {
    const C* q = reinterpret_cast<const C*>(p);
#pragma unroll
    for (int k = 0; k < n; ++k) psi[k] = q[k];
  }
}

// the hop of direction MU of role h (p = 4 h + MU), unless left out
template <class T, int MU, bool SKIP>
__device__ __forceinline__ void pipe_role_hop(typename wt<T>::C acc[4][3], const unsigned char* slots, int srec,
                                              const uint8_t* tab, const typename wt<T>::C* Ls, int rr, int h,
                                              T sgn, bool g5, int op, int dir, int disp, int skipb, bool tedge,
                                              int apbc) {
  typedef typename wt<T>::C C;
  if (op == GMG_OP_MDIR && (MU != dir || disp != (h ? -1 : 1))) return;
  if (SKIP && ((skipb >> (4 * h + MU)) & 1)) return;
  C psi[12];
  load_spinor<T>(psi, slots + tab[MU] * srec + rr * 12 * (int)sizeof(C), 12);
  if (g5) {
#pragma unroll
    for (int k = 6; k < 12; ++k) psi[k] = C{-psi[k].x, -psi[k].y};
  }
  const T coef = (apbc && MU == 3 && tedge) ? (T)0.5 : (T)-0.5;
  pipe_hop<T, MU>(acc, Ls + (4 * h + MU) * 9, psi, sgn, coef);
}

template <class T, bool DOTS, bool SKIP>
__global__ void __launch_bounds__(PipeGeo<T>::MAX_THREADS, 1) wilson_pipe_kernel(
    const typename wt<T>::C* __restrict__ hop, const typename wt<T>::C* __restrict__ clover,
    const PipeTile* __restrict__ tiles, const int32_t* __restrict__ tsites, const typename wt<T>::C* __restrict__ in,
    typename wt<T>::C* __restrict__ out, int nrhs, int ch, int nch, int ntiles, int nst, int ngrp, int sbytes, int soff,
    T diag, int op, int dir, int disp, int apbc, int tvol, int Lt, const uint8_t* __restrict__ hskip,
    double2* __restrict__ d1, double2* __restrict__ d2, int* __restrict__ err) {
  typedef typename wt<T>::C C;
  typedef PipeGeo<T> G;
  constexpr int W = PipeCfg<T>::WARPS;
  extern __shared__ __align__(128) unsigned char sm[];
  uint64_t* full = reinterpret_cast<uint64_t*>(sm);
  uint64_t* empty = full + kPipeMaxStages;
  double* Ds = reinterpret_cast<double*>(sm + kPipeHead);
  unsigned char* stages = sm + soff;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t items = (int64_t)ntiles * nch;
  const int srec = G::srec(ch);

  if (threadIdx.x == 0) {
    for (int k = 0; k < nst; ++k) {
      ac::mbar_init(&full[k], 1);
      ac::mbar_init(&empty[k], W);  // one group consumes each fill of a stage
    }
  }
  if (DOTS)
    for (int k = threadIdx.x; k < 3 * nrhs; k += blockDim.x) Ds[k] = 0.0;
  __syncthreads();

  if (warp == W * ngrp) {
    // ---- producer: one stage per item, in the order the consumers take them
    uint32_t n = 0;
    for (int64_t it = blockIdx.x; it < items; it += gridDim.x, ++n) {
      const int st = (int)(n % (uint32_t)nst);
      const uint32_t use = n / (uint32_t)nst;
      if (use > 0 && !ac::mbar_wait(&empty[st], (use - 1) & 1)) {
        if (lane == 0) atomicCAS(err, 0, 2);
        break;
      }
      const int tile = (int)(it / nch), chunk = (int)(it - (int64_t)tile * nch);
      const int r0 = chunk * ch, rc = min(ch, nrhs - r0);
      const PipeTile* tp = tiles + tile;
      const int ns = tp->ns, nss = tp->nss, s0 = tp->s0;
      unsigned char* sb = stages + (size_t)st * sbytes;
      const uint32_t rbytes = (uint32_t)rc * 12u * (uint32_t)sizeof(C);
      if (lane == 0)
        ac::mbar_expect_tx(&full[st], 48u + 2u * (uint32_t)nss * 72u * (uint32_t)sizeof(C) + (uint32_t)ns * rbytes);
      __syncwarp();
      if (lane < ns)
        ac::bulk_g2s(sb + G::OFF_SLOTS + lane * srec, in + ((int64_t)tsites[(int64_t)tile * kPipeSMax + lane] * nrhs + r0) * 12,
                     rbytes, &full[st]);
      if (lane < nss) {
        ac::bulk_g2s(sb + G::OFF_LINKS + lane * G::LREC, hop + (int64_t)(s0 + lane) * 72, 72 * sizeof(C), &full[st]);
        ac::bulk_g2s(sb + G::OFF_CLOV + lane * G::LREC, clover + (int64_t)(s0 + lane) * 72, 72 * sizeof(C),
                     &full[st]);
      }
      if (lane == 31) ac::bulk_g2s(sb, tp, 48, &full[st]);
    }
    // every stage this warp filled has landed before it exits (normally the
    // consumers have waited for all of them already)
    if (lane == 0) {
      const uint32_t last = n < (uint32_t)nst ? n : (uint32_t)nst;
      for (uint32_t k = 1; k <= last; ++k) {
        const uint32_t m = n - k;
        if (!ac::mbar_wait(&full[m % (uint32_t)nst], (m / (uint32_t)nst) & 1)) atomicCAS(err, 0, 2);
      }
    }
    return;
  }

  // ---- consumers: group g takes the items n = g, g + ngrp, ... (stage n mod nst)
  const int grp = warp / W, cw = warp - grp * W, h = lane >> 4, qtr = (lane >> 3) & 1, in8 = lane & 7;
  const int j = sizeof(T) == 4 ? 2 * qtr + (in8 >> 2) : in8 >> 1;
  const int rr = sizeof(T) == 4 ? 4 * cw + (in8 & 3) : 4 * cw + 2 * qtr + (in8 & 1);
  const bool g5 = (op == GMG_OP_MDAG);
  const T sgn = h ? (T)1 : (T)-1;
  uint32_t n = (uint32_t)grp;
  for (int64_t it = blockIdx.x + (int64_t)grp * gridDim.x; it < items;
       it += (int64_t)ngrp * gridDim.x, n += (uint32_t)ngrp) {
    const int st = (int)(n % (uint32_t)nst);
    const uint32_t use = n / (uint32_t)nst;
    if (!ac::mbar_wait(&full[st], use & 1)) {
      if (lane == 0) atomicCAS(err, 0, 3);
      break;
    }
    const unsigned char* sb = stages + (size_t)st * sbytes;
    const int chunk = (int)(it % nch);
    const int r0 = chunk * ch, rc = min(ch, nrhs - r0);
    if (4 * cw < rc) {
      const PipeTile* tp = reinterpret_cast<const PipeTile*>(sb);
      const int nss = tp->nss, site = tp->s0 + j;
      const bool valid = j < nss && rr < rc;
      const unsigned char* slots = sb + G::OFF_SLOTS;
      C acc[4][3];
#pragma unroll
      for (int s = 0; s < 4; ++s)
#pragma unroll
        for (int c = 0; c < 3; ++c) acc[s][c] = C{0, 0};
      C c6[6], cin[6];
#pragma unroll
      for (int k = 0; k < 6; ++k) c6[k] = cin[k] = C{0, 0};
      if (valid) {
        const int tc = site / tvol;
        const bool tedge = h ? tc == 0 : tc == Lt - 1;
        const int skipb = SKIP ? (int)hskip[site] : 0;
        if (op != GMG_OP_MDIAG) {
          const uint8_t* tab = tp->slot + j * 8 + 4 * h;
          const C* Ls = reinterpret_cast<const C*>(sb + G::OFF_LINKS + j * G::LREC);
          pipe_role_hop<T, 0, SKIP>(acc, slots, srec, tab, Ls, rr, h, sgn, g5, op, dir, disp, skipb, tedge, apbc);
          pipe_role_hop<T, 1, SKIP>(acc, slots, srec, tab, Ls, rr, h, sgn, g5, op, dir, disp, skipb, tedge, apbc);
          pipe_role_hop<T, 2, SKIP>(acc, slots, srec, tab, Ls, rr, h, sgn, g5, op, dir, disp, skipb, tedge, apbc);
          pipe_role_hop<T, 3, SKIP>(acc, slots, srec, tab, Ls, rr, h, sgn, g5, op, dir, disp, skipb, tedge, apbc);
        }
        if (op != GMG_OP_MDIR || DOTS) {
          // this role's chiral half of the site's own record (spins 2h, 2h + 1)
          load_spinor<T>(cin, slots + j * srec + (rr * 12 + 6 * h) * (int)sizeof(C), 6);
        }
        if (op != GMG_OP_MDIR) {
          C pin[6];
#pragma unroll
          for (int k = 0; k < 6; ++k) pin[k] = (g5 && h) ? C{-cin[k].x, -cin[k].y} : cin[k];
          const C* cl = reinterpret_cast<const C*>(sb + G::OFF_CLOV + j * G::LREC) + h * 36;
#pragma unroll
          for (int a = 0; a < 6; ++a) {
            C v = C{diag * pin[a].x, diag * pin[a].y};
#pragma unroll
            for (int b = 0; b < 6; ++b) v = cfma(cl[a * 6 + b], pin[b], v);
            c6[a] = v;
          }
        }
      }
      // exchange: each role keeps its own two spins and hands the other two to its partner
      C o[6];
#pragma unroll
      for (int k = 0; k < 6; ++k) {
        const C keep = h ? acc[2 + k / 3][k % 3] : acc[k / 3][k % 3];
        const C give = h ? acc[k / 3][k % 3] : acc[2 + k / 3][k % 3];
        C got;
        got.x = __shfl_xor_sync(0xffffffffu, give.x, 16);
        got.y = __shfl_xor_sync(0xffffffffu, give.y, 16);
        o[k] = cadd(cadd(keep, got), c6[k]);
        if (g5 && h) o[k] = C{-o[k].x, -o[k].y};
      }
      if (valid) {
        C* dst = out + ((int64_t)site * nrhs + r0 + rr) * 12 + 6 * h;
        if (sizeof(T) == 4) {
          float4* q = reinterpret_cast<float4*>(dst);
#pragma unroll
          for (int k = 0; k < 3; ++k)
            q[k] = make_float4((float)o[2 * k].x, (float)o[2 * k].y, (float)o[2 * k + 1].x, (float)o[2 * k + 1].y);
        } else {
#pragma unroll
          for (int k = 0; k < 6; ++k) dst[k] = o[k];
        }
      }
      if (DOTS) {
        double pr = 0.0, pi = 0.0, pn = 0.0;
        if (valid) {
#pragma unroll
          for (int k = 0; k < 6; ++k) {
            const double vx = o[k].x, vy = o[k].y, ix = cin[k].x, iy = cin[k].y;
            pr += vx * ix + vy * iy;
            pi += vx * iy - vy * ix;
            pn += vx * vx + vy * vy;
          }
        }
        // fold the lanes of one RHS: the sites (and the quarter for FP32) and the roles
        const int m1 = sizeof(T) == 4 ? 4 : 2, m2 = sizeof(T) == 4 ? 8 : 4;
#pragma unroll
        for (int q = 0; q < 3; ++q) {
          const int m = q == 0 ? m1 : q == 1 ? m2 : 16;
          pr += __shfl_xor_sync(0xffffffffu, pr, m);
          pi += __shfl_xor_sync(0xffffffffu, pi, m);
          pn += __shfl_xor_sync(0xffffffffu, pn, m);
        }
        if ((lane & (m1 | m2 | 16)) == 0 && rr < rc) {
          atomicAdd(&Ds[3 * (r0 + rr)], pr);
          atomicAdd(&Ds[3 * (r0 + rr) + 1], pi);
          atomicAdd(&Ds[3 * (r0 + rr) + 2], pn);
        }
      }
    }
    __syncwarp();
    if (lane == 0) ac::mbar_arrive(&empty[st]);
  }
  if (DOTS) {
    asm volatile("bar.sync 1, %0;" ::"r"(W * ngrp * 32) : "memory");
    for (int k = threadIdx.x; k < nrhs; k += W * ngrp * 32) {
      atomicAdd(&d1[k].x, Ds[3 * k]);
      atomicAdd(&d1[k].y, Ds[3 * k + 1]);
      atomicAdd(&d2[k].x, Ds[3 * k + 2]);
    }
  }
}

// hop links: hop[x][p] = p < 4 ? U_p(x) : U_{p-4}(x - p)^dagger, so that
// every hop multiplies by its link as stored
template <class C>
__global__ void hop_links_kernel(const C* __restrict__ gauge, const int32_t* __restrict__ nbr, C* __restrict__ hop,
                                 int V) {
  const int64_t n = (int64_t)V * 72;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    const int site = (int)(e / 72), k = (int)(e % 72), p = k / 9, m = k % 9;
    if (p < 4) {
      hop[e] = gauge[((int64_t)site * 4 + p) * 9 + m];
    } else {
      const int src = nbr[(int64_t)p * V + site];
      const C u = gauge[((int64_t)src * 4 + (p & 3)) * 9 + (m % 3) * 3 + m / 3];
      hop[e] = C{u.x, -u.y};
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
  GMG_TRY(h->hop.alloc(sizeof(double2) * 72 * (size_t)V));
  GMG_TRY(h->hop_f.alloc(sizeof(float2) * 72 * (size_t)V));
  const int g = (int)std::min<int64_t>(((int64_t)V * 72 + 255) / 256, 148 * 64);
  hop_links_kernel<double2><<<g, 256, 0, s>>>(h->gauge.as<double2>(), h->nbr.as<int32_t>(), h->hop.as<double2>(), V);
  hop_links_kernel<float2><<<g, 256, 0, s>>>(h->gauge_f.as<float2>(), h->nbr.as<int32_t>(), h->hop_f.as<float2>(), V);
  GMG_CUDA(cudaGetLastError());
  return GMG_OK;
}

// Plan of the pipelined staged kernel, tiles in processing order: per tile a
// PipeTile entry (first site, slot count, site count, the slot of each hop's
// record) and the sites of its slots (the tile's own sites first, then every
// distinct out-of-tile neighbour).  Tiles are sorted by (z / bz, t, z mod bz,
// y, x): the records that neighbouring tiles in t share stay within a window
// of about 2 bz Lx Ly sites.  At most 7 TS + 4 slots per tile (TS own, 6 TS
// across y, z, t, at most 4 x halos where a tile starts or ends inside an x
// row); a lattice that needs more gets no plan.
static size_t align16(size_t x) { return (x + 15) & ~(size_t)15; }

static gmg_status build_pipe_plan(gmg_wilson* h, int bz, cudaStream_t s, const gmg_wilson::PipePlan** out) {
  auto found = h->pplans.find(bz);
  if (found != h->pplans.end()) {
    *out = &found->second;
    return GMG_OK;
  }
  gmg_wilson::PipePlan& plan = h->pplans[bz];
  *out = &plan;
  const int64_t V = h->dims.vol();
  const int L0 = h->dims.d[0], L1 = h->dims.d[1], L2 = h->dims.d[2], L3 = h->dims.d[3];
  const int ntiles = (int)((V + kPipeTS - 1) / kPipeTS);
  std::vector<int32_t> nbr(9 * V);
  host_neighbors(h->dims, nbr.data());
  std::vector<int64_t> key(ntiles);
  std::vector<int32_t> order(ntiles);
  for (int tile = 0; tile < ntiles; ++tile) {
    const int64_t s0 = (int64_t)tile * kPipeTS;
    const int64_t x = s0 % L0, y = (s0 / L0) % L1, z = (s0 / ((int64_t)L0 * L1)) % L2,
                  t = s0 / ((int64_t)L0 * L1 * L2);
    key[tile] = ((((z / bz) * L3 + t) * bz + z % bz) * L1 + y) * L0 + x;
    order[tile] = tile;
  }
  std::sort(order.begin(), order.end(), [&](int32_t a, int32_t b) { return key[a] < key[b]; });
  const size_t tbytes = sizeof(PipeTile) * (size_t)ntiles;
  std::vector<unsigned char> host(tbytes + sizeof(int32_t) * (size_t)ntiles * kPipeSMax, 0);
  PipeTile* tiles = reinterpret_cast<PipeTile*>(host.data());
  int32_t* sites = reinterpret_cast<int32_t*>(host.data() + tbytes);
  int smax = 0;
  for (int k = 0; k < ntiles; ++k) {
    const int64_t s0 = (int64_t)order[k] * kPipeTS;
    const int nss = (int)std::min<int64_t>(kPipeTS, V - s0);
    PipeTile& tp = tiles[k];
    int32_t* st = sites + (size_t)k * kPipeSMax;
    tp.s0 = (int32_t)s0;
    tp.nss = nss;
    int n = nss;
    for (int j = 0; j < nss; ++j) st[j] = (int32_t)(s0 + j);
    for (int p = 0; p < 8; ++p)
      for (int j = 0; j < nss; ++j) {
        const int32_t nb = nbr[(size_t)p * V + s0 + j];
        int slot = -1;
        for (int q = 0; q < n; ++q)
          if (st[q] == nb) {
            slot = q;
            break;
          }
        if (slot < 0) {
          if (n == kPipeSMax) return GMG_OK;  // no plan (smax 0): the staged kernel does not apply
          st[n] = nb;
          slot = n++;
        }
        tp.slot[j * 8 + p] = (uint8_t)slot;
      }
    tp.ns = n;
    smax = std::max(smax, n);
  }
  GMG_TRY(plan.buf.alloc(host.size()));
  GMG_CUDA(cudaMemcpyAsync(plan.buf.p, host.data(), host.size(), cudaMemcpyHostToDevice, s));
  GMG_CUDA(cudaStreamSynchronize(s));  // host goes out of scope
  plan.smax = smax;
  return GMG_OK;
}

// z block of the tile order: the largest divisor of Lz whose window of
// records, 2 bz Lx Ly sites of rec_bytes each, stays within budget (at least 1)
static int pipe_bz(const gmg_wilson* h, int64_t rec_bytes, double budget) {
  const int L2 = h->dims.d[2];
  const double plane = (double)h->dims.d[0] * h->dims.d[1] * (double)rec_bytes;
  int bz = 1;
  for (int b = 1; b <= L2; ++b)
    if (L2 % b == 0 && 2.0 * b * plane <= budget) bz = b;
  return bz;
}

// pipelined staged kernel launch; *launched = false when it does not apply
// (unaligned fields, no plan for this lattice, or too little shared memory for
// two stages).  hskip (per site, bit p: leave hop p out) is the coarsening's
// self-term restriction, or null.
template <bool DOTS>
static gmg_status launch_pipe(gmg_wilson* h, int op, int dir, int disp, int vec_prec, int nrhs, const void* in,
                              void* out, double2* d1, double2* d2, cudaStream_t s, bool* launched,
                              const uint8_t* hskip = nullptr) {
  *launched = false;
  if (((uintptr_t)in | (uintptr_t)out) & 15) return GMG_OK;
  const bool f32 = vec_prec == GMG_F32;
  if (!f32 && vec_prec != GMG_F64) return GMG_OK;
  const int cmax = f32 ? PipeCfg<float>::CMAX : PipeCfg<double>::CMAX;
  const int nch = (nrhs + cmax - 1) / cmax, ch = (nrhs + nch - 1) / nch;
  const int64_t rec = (int64_t)nrhs * 12 * (f32 ? sizeof(float2) : sizeof(double2));
  const int bz = pipe_bz(h, rec, 48.0 * 1024 * 1024);
  const gmg_wilson::PipePlan* plan = nullptr;
  GMG_TRY(build_pipe_plan(h, bz, s, &plan));
  if (plan->smax == 0) return GMG_OK;
  const int sbytes = f32 ? PipeGeo<float>::stage_bytes(ch, plan->smax) : PipeGeo<double>::stage_bytes(ch, plan->smax);
  const int soff = kPipeHead + (DOTS ? (int)align16(sizeof(double) * 3 * (size_t)nrhs) : 0);
  int dev = 0, nsm = 148, smem_optin = 0;
  GMG_CUDA(cudaGetDevice(&dev));
  GMG_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  GMG_CUDA(cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  const int nst = std::min(kPipeMaxStages, (smem_optin - soff) / sbytes);
  if (nst < 2) return GMG_OK;
  // consumer groups: all but one stage being computed, one being filled
  const int gmax = f32 ? PipeCfg<float>::GMAX : PipeCfg<double>::GMAX;
  const int ngrp = std::min(gmax, nst - 1);
  const size_t smem = (size_t)soff + (size_t)nst * sbytes;
  if (!h->dev_err.p) {
    GMG_TRY(h->dev_err.alloc(256));
    GMG_CUDA(cudaMemsetAsync(h->dev_err.p, 0, 256, s));
  }
  const int V = (int)h->dims.vol();
  const int tvol = h->dims.d[0] * h->dims.d[1] * h->dims.d[2];
  const int ntiles = (V + kPipeTS - 1) / kPipeTS;
  const int64_t items = (int64_t)ntiles * nch;
  const PipeTile* tiles = plan->buf.as<PipeTile>();
  const int32_t* tsites =
      reinterpret_cast<const int32_t*>(plan->buf.as<unsigned char>() + sizeof(PipeTile) * (size_t)ntiles);
  const int g = (int)std::min<int64_t>(items, nsm);
  auto go = [&](auto kern, int wpg, auto diag, const void* hp, const void* cp) -> gmg_status {
    const int threads = (wpg * ngrp + 1) * 32;
    typedef decltype(diag) T;
    typedef typename wt<T>::C C;
    GMG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    kern<<<g, threads, smem, s>>>(reinterpret_cast<const C*>(hp), reinterpret_cast<const C*>(cp), tiles, tsites,
                                  reinterpret_cast<const C*>(in), reinterpret_cast<C*>(out), nrhs, ch, nch, ntiles,
                                  nst, ngrp, sbytes, soff, diag, op, dir, disp, h->apbc, tvol, h->dims.d[3], hskip, d1, d2,
                                  h->dev_err.as<int>());
    GMG_CUDA(cudaGetLastError());
    return GMG_OK;
  };
  if (f32) {
    const float diag = (float)(4.0 + h->mass);
    if (hskip)
      GMG_TRY(go(wilson_pipe_kernel<float, DOTS, true>, PipeCfg<float>::WARPS, diag, h->hop_f.p, h->clover_f.p));
    else
      GMG_TRY(go(wilson_pipe_kernel<float, DOTS, false>, PipeCfg<float>::WARPS, diag, h->hop_f.p, h->clover_f.p));
  } else {
    const double diag = 4.0 + h->mass;
    if (hskip)
      GMG_TRY(go(wilson_pipe_kernel<double, DOTS, true>, PipeCfg<double>::WARPS, diag, h->hop.p, h->clover.p));
    else
      GMG_TRY(go(wilson_pipe_kernel<double, DOTS, false>, PipeCfg<double>::WARPS, diag, h->hop.p, h->clover.p));
  }
  *launched = true;
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

// thread per (site, RHS), links and clover from global memory
static gmg_status launch_site(gmg_wilson* h, int op, int dir, int disp, int vec_prec, int nrhs, const void* in,
                              void* out, cudaStream_t s) {
  const int V = (int)h->dims.vol();
  const int tvol = h->dims.d[0] * h->dims.d[1] * h->dims.d[2];
  const int64_t total = (int64_t)V * nrhs;
  const int grid = (int)std::min<int64_t>((total + 127) / 128, 148 * 32);
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

// Grid of the tile kernels: one resident wave (the CTAs loop over the tiles),
// so no CTA waits for a later wave and the MR products take one atomic per CTA
// and RHS.  (At 16^4 x 24 RHS the BF16 smoother form ran 162 -> 150 us against
// a grid of 16 CTAs per SM.)
template <class K>
static int wave_grid(K kern, int threads, size_t smem, int tiles) {
  int nb = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kern, threads, smem) != cudaSuccess || nb < 1) nb = 1;
  int dev = 0, nsm = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  return std::max(1, std::min(tiles, nsm * nb));
}

// tile kernel: kTileSites sites x rt threads per CTA (rt <= 16); MINB: CTAs
// per SM the register allocation must allow (FP32: 2 or 3)
template <bool DOTS, int MINB = 2, bool PF = (MINB == 2)>
static gmg_status launch_tile(gmg_wilson* h, int op, int dir, int disp, int vec_prec, int nrhs, const void* in,
                              void* out, double2* d1, double2* d2, cudaStream_t s) {
  const int V = (int)h->dims.vol();
  const int tvol = h->dims.d[0] * h->dims.d[1] * h->dims.d[2];
  // threads per site: the largest divisor of nrhs up to 16, so that every
  // thread of a site handles the same number of RHS (24 -> 12 x 2); nrhs
  // without a divisor of 8 or more above 16 uses 16 (the last round uneven)
  int rt = 1;
  for (int c = std::min(nrhs, 16); c >= 1; --c)
    if (nrhs % c == 0) {
      rt = c;
      break;
    }
  if (nrhs > 16 && rt < 8) rt = 16;
  const int tiles = (V + kTileSites - 1) / kTileSites;
  const size_t dots = DOTS ? sizeof(double) * 3 * (size_t)nrhs : 0;
  // 32-byte record accesses when both fields are 32-byte aligned
  const bool v32 = ((((uintptr_t)in | (uintptr_t)out) & 31) == 0);
  auto go = [&](auto kern, auto diag, const void* hp, const void* cp, size_t csize) -> gmg_status {
    typedef decltype(diag) T;
    typedef typename wt<T>::C C;
    const size_t smem = tile_smem((int)csize, false, dots);
    if (smem > 48 * 1024) GMG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const int g = wave_grid(kern, kTileSites * rt, smem, tiles);
    kern<<<g, kTileSites * rt, smem, s>>>(reinterpret_cast<const C*>(hp), reinterpret_cast<const C*>(cp),
                                          h->nbr.as<int32_t>(), reinterpret_cast<const C*>(in),
                                          reinterpret_cast<C*>(out), V, nrhs, rt, diag, op, dir, disp, h->apbc, tvol,
                                          h->dims.d[3], d1, d2, nullptr, 0, nullptr, nullptr);
    return GMG_OK;
  };
  if (vec_prec == GMG_F64) {
    const double diag = 4.0 + h->mass;
    if (v32)
      GMG_TRY(go(wilson_tile_kernel<double, DOTS, 2, false, 2, true>, diag, h->hop.p, h->clover.p, sizeof(double2)));
    else
      GMG_TRY(go(wilson_tile_kernel<double, DOTS, 2, false, 1>, diag, h->hop.p, h->clover.p, sizeof(double2)));
  } else if (vec_prec == GMG_F32) {
    const float diag = (float)(4.0 + h->mass);
    if (v32)
      GMG_TRY(go(wilson_tile_kernel<float, DOTS, MINB, false, 2, PF>, diag, h->hop_f.p, h->clover_f.p,
                 sizeof(float2)));
    else
      GMG_TRY(go(wilson_tile_kernel<float, DOTS, MINB, false, 1>, diag, h->hop_f.p, h->clover_f.p, sizeof(float2)));
  } else {
    return fail(GMG_ERR_UNSUPPORTED, "wilson apply: vectors must be F64 or F32");
  }
  GMG_CUDA(cudaGetLastError());
  return GMG_OK;
}

// internal variant id: a second register budget of the tile kernel, tuned
// alongside the public variants and reported as GMG_WILSON_TILE
constexpr int kTileOcc3 = 16;
// and the same with the neighbour records prefetched (FP32)
constexpr int kTileOcc3Pf = 17;

// One launch of kernel variant v; *launched = false when v does not apply.
static gmg_status run_variant(gmg_wilson* h, int v, bool dots, int op, int dir, int disp, int vec_prec, int nrhs,
                              const void* in, void* out, double2* d1, double2* d2, cudaStream_t s, bool* launched) {
  *launched = true;
  switch (v) {
    case GMG_WILSON_SITE:
      if (dots) break;
      return launch_site(h, op, dir, disp, vec_prec, nrhs, in, out, s);
    case GMG_WILSON_TILE:
      if (((uintptr_t)in | (uintptr_t)out) & 15) break;  // 16-byte spinor accesses
      return dots ? launch_tile<true>(h, op, dir, disp, vec_prec, nrhs, in, out, d1, d2, s)
                  : launch_tile<false>(h, op, dir, disp, vec_prec, nrhs, in, out, d1, d2, s);
    case kTileOcc3Pf:
      if ((((uintptr_t)in | (uintptr_t)out) & 31) || vec_prec != GMG_F32) break;
      return dots ? launch_tile<true, 3, true>(h, op, dir, disp, vec_prec, nrhs, in, out, d1, d2, s)
                  : launch_tile<false, 3, true>(h, op, dir, disp, vec_prec, nrhs, in, out, d1, d2, s);
    case kTileOcc3:  // the tile kernel with registers capped for 3 CTAs per SM (FP32)
      if ((((uintptr_t)in | (uintptr_t)out) & 15) || vec_prec != GMG_F32) break;
      return dots ? launch_tile<true, 3>(h, op, dir, disp, vec_prec, nrhs, in, out, d1, d2, s)
                  : launch_tile<false, 3>(h, op, dir, disp, vec_prec, nrhs, in, out, d1, d2, s);
    case GMG_WILSON_QUAD:
      return dots ? launch_quad<true>(h, op, dir, disp, vec_prec, nrhs, in, out, d1, d2, s)
                  : launch_quad<false>(h, op, dir, disp, vec_prec, nrhs, in, out, d1, d2, s);
    case GMG_WILSON_STAGED:
      return dots ? launch_pipe<true>(h, op, dir, disp, vec_prec, nrhs, in, out, d1, d2, s, launched)
                  : launch_pipe<false>(h, op, dir, disp, vec_prec, nrhs, in, out, d1, d2, s, launched);
    default:
      break;
  }
  *launched = false;
  return GMG_OK;
}

// Autotuned dispatch.  The kernel variant is chosen per (vector precision,
// fused products or not, single-hop op or not, nrhs class) by timing every
// applicable variant once on the call that first meets the key (CUDA events
// on the caller's stream; not while the stream is being captured) and is
// cached in the handle.  The nrhs classes (1-3, 4-7, 8-15, 16-31, 32+) keep a
// batch that shrinks as right-hand sides converge from re-tuning at every size.
static gmg_status wilson_dispatch(gmg_wilson* h, bool dots, int op, int dir, int disp, int vec_prec, int nrhs,
                                  const void* in, void* out, double2* d1, double2* d2, cudaStream_t s) {
  auto zero_dots = [&]() -> gmg_status {
    if (dots) {
      GMG_CUDA(cudaMemsetAsync(d1, 0, sizeof(double2) * nrhs, s));
      GMG_CUDA(cudaMemsetAsync(d2, 0, sizeof(double2) * nrhs, s));
    }
    return GMG_OK;
  };
  bool launched = false;
  if (h->wforce >= 0) {
    GMG_TRY(zero_dots());
    GMG_TRY(run_variant(h, h->wforce, dots, op, dir, disp, vec_prec, nrhs, in, out, d1, d2, s, &launched));
    if (launched) return GMG_OK;
    // a forced variant that does not apply falls through to the tuned choice
  }
  const int cls = nrhs < 4 ? 0 : nrhs < 8 ? 1 : nrhs < 16 ? 2 : nrhs < 32 ? 3 : 4;
  const uint64_t key = (uint64_t)vec_prec | ((uint64_t)dots << 4) | ((uint64_t)(op == GMG_OP_MDIR) << 5) |
                       ((uint64_t)cls << 8);
  auto it = h->wtune.find(key);
  if (it != h->wtune.end()) {
    GMG_TRY(zero_dots());
    GMG_TRY(run_variant(h, it->second, dots, op, dir, disp, vec_prec, nrhs, in, out, d1, d2, s, &launched));
    if (launched) return GMG_OK;
  }
  std::vector<int> cand;
  if (!dots && nrhs < 4) cand.push_back(GMG_WILSON_SITE);
  cand.push_back(GMG_WILSON_TILE);
  if (vec_prec == GMG_F32) {
    cand.push_back(kTileOcc3);
    cand.push_back(kTileOcc3Pf);
  }
  cand.push_back(GMG_WILSON_QUAD);
  if (nrhs >= 4) cand.push_back(GMG_WILSON_STAGED);
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  GMG_CUDA(cudaStreamIsCapturing(s, &cap));
  int best = nrhs >= 4 ? GMG_WILSON_TILE : (dots ? GMG_WILSON_QUAD : GMG_WILSON_SITE);
  if (cap == cudaStreamCaptureStatusNone) {
    cudaEvent_t e0, e1;
    GMG_CUDA(cudaEventCreate(&e0));
    GMG_CUDA(cudaEventCreate(&e1));
    float best_ms = 1e30f;
    gmg_status st = GMG_OK;
    for (int v : cand) {
      bool ok = false;
      st = run_variant(h, v, dots, op, dir, disp, vec_prec, nrhs, in, out, d1, d2, s, &ok);  // warm-up
      if (st != GMG_OK) break;
      if (!ok) continue;
      if (cudaEventRecord(e0, s) != cudaSuccess) break;
      for (int k = 0; k < 2 && st == GMG_OK; ++k)
        st = run_variant(h, v, dots, op, dir, disp, vec_prec, nrhs, in, out, d1, d2, s, &ok);
      if (st != GMG_OK || cudaEventRecord(e1, s) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess) break;
      float ms = 0.f;
      cudaEventElapsedTime(&ms, e0, e1);
      if (ms < best_ms) {
        best_ms = ms;
        best = v;
      }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    GMG_TRY(st);
    GMG_CUDA(cudaGetLastError());
    h->wtune[key] = best;
  }
  GMG_TRY(zero_dots());
  GMG_TRY(run_variant(h, best, dots, op, dir, disp, vec_prec, nrhs, in, out, d1, d2, s, &launched));
  if (!launched) return fail(GMG_ERR_UNSUPPORTED, "wilson apply: no kernel variant applies");
  return GMG_OK;
}

// Single-hop operator (Mdir of stencil point p) on a list of sites, FP64, for
// the coarsening's face terms.  A CTA takes S = blockDim / nrhs sites: their
// neighbour records (all RHS, 12 components each, contiguous in memory) come
// into shared memory with coalesced loads, one thread per (site, RHS) applies
// the hop from there into its own slot, and the results leave through the
// same buffer with coalesced stores.  Slots are padded to 13 complex numbers so
// that the 16-byte reads of consecutive RHS fall on different banks.  The
// arithmetic is wilson_hop's, as in wilson_site with op GMG_OP_MDIR.
constexpr int kFacePad = 13;

template <int MU>
__device__ __forceinline__ void face_hop(double2 acc[4][3], const double2* __restrict__ U, const double2* psi,
                                         int disp, double coef) {
  wilson_hop<double>(acc, U, false, psi, MU, disp, coef);  // backward links stored daggered
}

__global__ void __launch_bounds__(256, 3) wilson_face_hop_kernel(
    const double2* __restrict__ hop, const int32_t* __restrict__ nbr, const double2* __restrict__ in,
    double2* __restrict__ out, int V, int nrhs, const int32_t* __restrict__ sel, int nsel, int p, int apbc,
    int tvol, int Lt) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int R = nrhs, W = nrhs * 12;
  const int S = blockDim.x / R;
  double2* rec = reinterpret_cast<double2*>(smem_raw);  // [S][R][kFacePad]
  int* sidx = reinterpret_cast<int*>(rec + (size_t)S * R * kFacePad);
  int* nidx = sidx + S;
  const int mu = p & 3, disp = p < 4 ? 1 : -1;
  const int t = threadIdx.x, q = t / R, r = t % R;
  const int ntl = (nsel + S - 1) / S;
  for (int tile = blockIdx.x; tile < ntl; tile += gridDim.x) {
    const int s0 = tile * S, ns = min(S, nsel - s0);
    __syncthreads();  // the previous tile's stores have read rec, sidx
    if (t < ns) {
      const int st = sel[s0 + t];
      sidx[t] = st;
      nidx[t] = nbr[(int64_t)p * V + st];
    }
    __syncthreads();
    // one flat loop over the tile's records: its loads are independent and
    // issue back to back (12 per thread for 40 RHS)
#pragma unroll 12
    for (int k = t; k < ns * W; k += blockDim.x) {
      const int qq = k / W, e = k - qq * W;
      rec[qq * R * kFacePad + (e / 12) * kFacePad + e % 12] = in[(int64_t)nidx[qq] * W + e];
    }
    __syncthreads();
    if (q < ns) {
      const int site = sidx[q];
      double2* my = rec + (q * R + r) * kFacePad;
      double2 psi[12];
#pragma unroll
      for (int a = 0; a < 12; ++a) psi[a] = my[a];
      double2 acc[4][3];
#pragma unroll
      for (int s2 = 0; s2 < 4; ++s2)
#pragma unroll
        for (int c = 0; c < 3; ++c) acc[s2][c] = make_double2(0.0, 0.0);
      const int tc = site / tvol;
      double coef = -0.5;
      if (apbc && mu == 3 && ((disp > 0 && tc == Lt - 1) || (disp < 0 && tc == 0))) coef = 0.5;
      const double2* U = hop + (int64_t)site * 72 + p * 9;
      switch (mu) {
        case 0: face_hop<0>(acc, U, psi, disp, coef); break;
        case 1: face_hop<1>(acc, U, psi, disp, coef); break;
        case 2: face_hop<2>(acc, U, psi, disp, coef); break;
        default: face_hop<3>(acc, U, psi, disp, coef); break;
      }
#pragma unroll
      for (int s2 = 0; s2 < 4; ++s2)
#pragma unroll
        for (int c = 0; c < 3; ++c) my[s2 * 3 + c] = acc[s2][c];
    }
    __syncthreads();
#pragma unroll 12
    for (int k = t; k < ns * W; k += blockDim.x) {
      const int qq = k / W, e = k - qq * W;
      out[(int64_t)sidx[qq] * W + e] = rec[qq * R * kFacePad + (e / 12) * kFacePad + e % 12];
    }
  }
}

// out = Mdir_p in on the nsel sites of `sel` (FP64, nrhs <= 64); the other
// sites of `out` are not written
gmg_status wilson_apply_face(gmg_wilson* h, int p, int nrhs, const double* in, double* out, const int32_t* sel,
                             int nsel, cudaStream_t s) {
  GMG_CHECK(nrhs >= 1 && nrhs <= 64, GMG_ERR_UNSUPPORTED, "wilson face hop: nrhs must be in [1, 64]");
  GMG_CHECK(p >= 0 && p < 8, GMG_ERR_ARGUMENT, "wilson face hop: bad stencil point");
  if (nsel == 0) return GMG_OK;
  const int V = (int)h->dims.vol();
  const int tvol = h->dims.d[0] * h->dims.d[1] * h->dims.d[2];
  const int S = std::max(1, 256 / nrhs);
  const int threads = S * nrhs;
  const size_t smem = sizeof(double2) * (size_t)S * nrhs * kFacePad + sizeof(int) * 2 * S;
  if (smem > 48 * 1024)
    GMG_CUDA(cudaFuncSetAttribute(wilson_face_hop_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  // all of the unified L1 / shared array as shared memory: three CTAs of
  // 50 KB per SM, as many as the register bound allows (two with the default
  // split)
  GMG_CUDA(cudaFuncSetAttribute(wilson_face_hop_kernel, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
  // one resident wave of CTAs looping over the tiles
  int occ = 1, dev = 0, nsm = 148;
  GMG_CUDA(cudaGetDevice(&dev));
  GMG_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  GMG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, wilson_face_hop_kernel, threads, smem));
  const int tiles = (nsel + S - 1) / S;
  const int g = std::min(tiles, nsm * std::max(occ, 1));
  KernelTimer kt("wilson", s);
  wilson_face_hop_kernel<<<g, threads, smem, s>>>(h->hop.as<double2>(), h->nbr.as<int32_t>(),
                                                   reinterpret_cast<const double2*>(in),
                                                   reinterpret_cast<double2*>(out), V, nrhs, sel, nsel, p, h->apbc,
                                                   tvol, h->dims.d[3]);
  GMG_CUDA(cudaGetLastError());
  return GMG_OK;
}

// the tile kernel's SEL instance (FP64): op on the nsel sites of `sel` (all
// sites when null), hops restricted by hskip; with all sites and 32-byte
// aligned fields, 32-byte record accesses (the prefetching form spills here)
static gmg_status launch_tile_sel(gmg_wilson* h, int op, int dir, int disp, int nrhs, const double* in, double* out,
                                  const int32_t* sel, int nsel, const uint8_t* hskip, cudaStream_t s) {
  const int V = (int)h->dims.vol();
  const int tvol = h->dims.d[0] * h->dims.d[1] * h->dims.d[2];
  int rt = 1;
  for (int c = std::min(nrhs, 16); c >= 1; --c)
    if (nrhs % c == 0) {
      rt = c;
      break;
    }
  if (nrhs > 16 && rt < 8) rt = 16;
  const int nsites = sel ? nsel : V;
  const int tiles = (nsites + kTileSites - 1) / kTileSites;
  const int g = std::min(tiles, 148 * 16);
  const size_t smem = tile_smem(sizeof(double2), true, 0);
  const bool fast = !sel && ((((uintptr_t)in | (uintptr_t)out) & 31) == 0);
  auto k = fast ? wilson_tile_kernel<double, false, 2, true, 2> : wilson_tile_kernel<double, false, 2, true>;
  if (smem > 48 * 1024) GMG_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  k<<<g, kTileSites * rt, smem, s>>>(h->hop.as<double2>(), h->clover.as<double2>(), h->nbr.as<int32_t>(),
                                     (const double2*)in, (double2*)out, V, nrhs, rt, 4.0 + h->mass, op, dir, disp,
                                     h->apbc, tvol, h->dims.d[3], nullptr, nullptr, sel, nsel, hskip, nullptr);
  GMG_CUDA(cudaGetLastError());
  return GMG_OK;
}

// The coarsening's forms of the FP64 operator: op on the nsel sites of `sel`
// only (all sites when null; the other sites of `out` are not written), and
// with hskip (per site, bit p set: leave hop p out) the hops restricted to
// neighbours of the same block parity.  With all sites, the pipelined staged
// kernel and the tile kernel are timed once per nrhs (not while the stream is
// being captured) and the faster one is kept.
gmg_status wilson_apply_sel(gmg_wilson* h, int op, int dir, int disp, int nrhs, const double* in, double* out,
                            const int32_t* sel, int nsel, const uint8_t* hskip, cudaStream_t s) {
  const int nsites = sel ? nsel : (int)h->dims.vol();
  if (nsites == 0) return GMG_OK;
  if (sel) {
    KernelTimer kt("wilson", s);
    return launch_tile_sel(h, op, dir, disp, nrhs, in, out, sel, nsel, hskip, s);
  }
  auto run = [&](int which, bool* launched) -> gmg_status {
    if (which == 0)
      return launch_pipe<false>(h, op, dir, disp, GMG_F64, nrhs, in, out, nullptr, nullptr, s, launched, hskip);
    *launched = true;
    return launch_tile_sel(h, op, dir, disp, nrhs, in, out, nullptr, 0, hskip, s);
  };
  int pick = 1;
  auto it = h->sel_pick.find(nrhs);
  if (it != h->sel_pick.end()) {
    pick = it->second;
  } else {
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    GMG_CUDA(cudaStreamIsCapturing(s, &cap));
    if (cap == cudaStreamCaptureStatusNone) {
      cudaEvent_t e0, e1;
      GMG_CUDA(cudaEventCreate(&e0));
      GMG_CUDA(cudaEventCreate(&e1));
      float best = 1e30f;
      gmg_status st = GMG_OK;
      for (int which = 0; which < 2 && st == GMG_OK; ++which) {
        bool launched = false;
        st = run(which, &launched);  // warm-up
        if (st != GMG_OK || !launched) continue;
        if (cudaEventRecord(e0, s) != cudaSuccess) break;
        for (int k = 0; k < 2 && st == GMG_OK; ++k) st = run(which, &launched);
        float ms = 0.f;
        if (st != GMG_OK || cudaEventRecord(e1, s) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
            cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess)
          break;
        if (ms < best) {
          best = ms;
          pick = which;
        }
      }
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
      GMG_TRY(st);
      if (best < 1e30f) h->sel_pick[nrhs] = pick;
    }
  }
  KernelTimer kt("wilson", s);
  bool launched = false;
  GMG_TRY(run(pick, &launched));
  if (!launched) GMG_TRY(run(1, &launched));
  return GMG_OK;
}

// out (FP64) = op in (FP32), op M or MDAG, in FP64 arithmetic on the FP32
// records promoted exactly on load: the same result as converting `in` to FP64
// and applying the FP64 operator, without the converted copy (the outer
// Arnoldi step's apply to a preconditioned direction).  The tile kernel at 2
// CTAs per SM with the records prefetched.
gmg_status wilson_apply_f32_in(gmg_wilson* h, int op, int nrhs, const float* in, double* out, cudaStream_t s) {
  GMG_CHECK(op == GMG_OP_M || op == GMG_OP_MDAG, GMG_ERR_UNSUPPORTED,
            "wilson apply (FP32 in, FP64 out): op must be M or Mdag");
  GMG_CHECK(nrhs >= 1, GMG_ERR_ARGUMENT, "wilson apply (FP32 in, FP64 out): nrhs must be positive");
  const int V = (int)h->dims.vol();
  const int tvol = h->dims.d[0] * h->dims.d[1] * h->dims.d[2];
  int rt = 1;
  for (int c = std::min(nrhs, 16); c >= 1; --c)
    if (nrhs % c == 0) {
      rt = c;
      break;
    }
  if (nrhs > 16 && rt < 8) rt = 16;
  const int tiles = (V + kTileSites - 1) / kTileSites;
  const int g = std::min(tiles, 148 * 16);
  const size_t smem = tile_smem(sizeof(double2), false, 0);
  const uintptr_t al = (uintptr_t)in | (uintptr_t)out;
  KernelTimer kt("wilson", s);
  auto go = [&](auto kern) -> gmg_status {
    if (smem > 48 * 1024)
      GMG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    kern<<<g, kTileSites * rt, smem, s>>>(h->hop.as<double2>(), h->clover.as<double2>(), h->nbr.as<int32_t>(),
                                          reinterpret_cast<const float2*>(in), reinterpret_cast<double2*>(out), V,
                                          nrhs, rt, 4.0 + h->mass, op, 0, 0, h->apbc, tvol, h->dims.d[3], nullptr,
                                          nullptr, nullptr, 0, nullptr, nullptr);
    GMG_CUDA(cudaGetLastError());
    return GMG_OK;
  };
  if ((al & 31) == 0) return go(wilson_tile_kernel<double, false, 2, false, 2, true, float>);
  if ((al & 15) == 0) return go(wilson_tile_kernel<double, false, 2, false, 1, true, float>);
  return go(wilson_tile_kernel<double, false, 2, false, 0, true, float>);
}

// out = M in with the minimal-residual inner products d1[r] = <out, in>,
// d2[r].x = <out, out> (zeroed here), on BF16 fields (one 32-bit word per
// complex number) [V][nrhs][12], or site-blocked [V][3][nrhs][4] with
// `blocked`: FP32 arithmetic on the widened records, the products from the
// FP32 result, the result rounded to BF16.  The tile kernel at 3 CTAs per SM
// with the records prefetched.
gmg_status wilson_apply_mr_bf16(gmg_wilson* h, int nrhs, const uint32_t* in, uint32_t* out, double2* d1, double2* d2,
                                cudaStream_t s, bool blocked) {
  GMG_CHECK(((((uintptr_t)in | (uintptr_t)out) & 15) == 0), GMG_ERR_ARGUMENT,
            "wilson apply (BF16): fields must be 16-byte aligned");
  GMG_CHECK(!blocked || h->dims.vol() * 3 * nrhs < ((int64_t)1 << 31), GMG_ERR_UNSUPPORTED,
            "wilson apply (BF16, site-blocked): field above 2^31 16-byte units");
  const int V = (int)h->dims.vol();
  const int tvol = h->dims.d[0] * h->dims.d[1] * h->dims.d[2];
  int rt = 1;
  for (int c = std::min(nrhs, 16); c >= 1; --c)
    if (nrhs % c == 0) {
      rt = c;
      break;
    }
  if (nrhs > 16 && rt < 8) rt = 16;
  const int tiles = (V + kTileSites - 1) / kTileSites;

  const size_t smem = tile_smem(sizeof(float2), false, sizeof(double) * 3 * (size_t)nrhs);
  KernelTimer kt("wilson", s);
  GMG_CUDA(cudaMemsetAsync(d1, 0, sizeof(double2) * nrhs, s));
  GMG_CUDA(cudaMemsetAsync(d2, 0, sizeof(double2) * nrhs, s));
  auto k = blocked ? wilson_tile_kernel<float, true, 3, false, 3, true, bf16s, bf16s>
                   : wilson_tile_kernel<float, true, 3, false, 1, true, bf16s, bf16s>;
  if (smem > 48 * 1024) GMG_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int g = wave_grid(k, kTileSites * rt, smem, tiles);
  k<<<g, kTileSites * rt, smem, s>>>(h->hop_f.as<float2>(), h->clover_f.as<float2>(), h->nbr.as<int32_t>(), in, out, V,
                                     nrhs, rt, (float)(4.0 + h->mass), GMG_OP_M, 0, 0, h->apbc, tvol, h->dims.d[3], d1,
                                     d2, nullptr, 0, nullptr, nullptr);
  GMG_CUDA(cudaGetLastError());
  return GMG_OK;
}

// out = bf16(b - M x) in the site-blocked BF16 layout [V][3][nrhs][4] words,
// x and b FP32 [V][nrhs][12] (32-byte aligned): the first residual of the
// BF16 smoother in one pass.  The tile kernel at 3 CTAs per SM with the
// records prefetched.
gmg_status wilson_residual_bf16(gmg_wilson* h, int nrhs, const float* b, const float* x, uint32_t* out,
                                cudaStream_t s) {
  GMG_CHECK((((uintptr_t)b | (uintptr_t)x) & 31) == 0 && ((uintptr_t)out & 15) == 0, GMG_ERR_ARGUMENT,
            "wilson residual (BF16): FP32 fields must be 32-byte aligned");
  GMG_CHECK(h->dims.vol() * 3 * nrhs < ((int64_t)1 << 31), GMG_ERR_UNSUPPORTED,
            "wilson residual (BF16): field above 2^31 16-byte units");
  const int V = (int)h->dims.vol();
  const int tvol = h->dims.d[0] * h->dims.d[1] * h->dims.d[2];
  int rt = 1;
  for (int c = std::min(nrhs, 16); c >= 1; --c)
    if (nrhs % c == 0) {
      rt = c;
      break;
    }
  if (nrhs > 16 && rt < 8) rt = 16;
  const int tiles = (V + kTileSites - 1) / kTileSites;
  const size_t smem = tile_smem(sizeof(float2), false, 0);
  KernelTimer kt("wilson", s);
  auto k = wilson_tile_kernel<float, false, 3, false, 2, true, float, bf16s, 3, true>;
  if (smem > 48 * 1024) GMG_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int g = wave_grid(k, kTileSites * rt, smem, tiles);
  k<<<g, kTileSites * rt, smem, s>>>(h->hop_f.as<float2>(), h->clover_f.as<float2>(), h->nbr.as<int32_t>(),
                                     reinterpret_cast<const float2*>(x), out, V, nrhs, rt, (float)(4.0 + h->mass),
                                     GMG_OP_M, 0, 0, h->apbc, tvol, h->dims.d[3], nullptr, nullptr, nullptr, 0,
                                     nullptr, reinterpret_cast<const float2*>(b));
  GMG_CUDA(cudaGetLastError());
  return GMG_OK;
}

// r = b - M x in FP64 ([V][nrhs][12], 32-byte aligned), one tile-kernel pass:
// the outer solver's residual without a separate subtraction sweep
gmg_status wilson_residual_f64(gmg_wilson* h, int nrhs, const double* b, const double* x, double* r,
                               cudaStream_t s) {
  GMG_CHECK((((uintptr_t)b | (uintptr_t)x | (uintptr_t)r) & 31) == 0, GMG_ERR_ARGUMENT,
            "wilson residual (FP64): fields must be 32-byte aligned");
  const int V = (int)h->dims.vol();
  const int tvol = h->dims.d[0] * h->dims.d[1] * h->dims.d[2];
  int rt = 1;
  for (int c = std::min(nrhs, 16); c >= 1; --c)
    if (nrhs % c == 0) {
      rt = c;
      break;
    }
  if (nrhs > 16 && rt < 8) rt = 16;
  const int tiles = (V + kTileSites - 1) / kTileSites;
  const size_t smem = tile_smem(sizeof(double2), false, 0);
  KernelTimer kt("wilson", s);
  auto k = wilson_tile_kernel<double, false, 2, false, 2, true, double, double, 2, true>;
  if (smem > 48 * 1024) GMG_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int g = wave_grid(k, kTileSites * rt, smem, tiles);
  k<<<g, kTileSites * rt, smem, s>>>(h->hop.as<double2>(), h->clover.as<double2>(), h->nbr.as<int32_t>(),
                                     reinterpret_cast<const double2*>(x), reinterpret_cast<double2*>(r), V, nrhs, rt,
                                     4.0 + h->mass, GMG_OP_M, 0, 0, h->apbc, tvol, h->dims.d[3], nullptr, nullptr,
                                     nullptr, 0, nullptr, reinterpret_cast<const double2*>(b));
  GMG_CUDA(cudaGetLastError());
  return GMG_OK;
}

gmg_status wilson_apply(gmg_wilson* h, int op, int dir, int disp, int vec_prec, int nrhs,
                        const void* in, void* out, cudaStream_t s) {
  if (vec_prec != GMG_F64 && vec_prec != GMG_F32)
    return fail(GMG_ERR_UNSUPPORTED, "wilson apply: vectors must be F64 or F32");
  KernelTimer kt("wilson", s);
  return wilson_dispatch(h, false, op, dir, disp, vec_prec, nrhs, in, out, nullptr, nullptr, s);
}

// out = M in, and the minimal-residual inner products d1[r] = <out, in>,
// d2[r].x = <out, out> (d1, d2: nrhs entries each, zeroed here)
gmg_status wilson_apply_mr(gmg_wilson* h, int vec_prec, int nrhs, const void* in, void* out, double2* d1,
                           double2* d2, cudaStream_t s) {
  if (vec_prec != GMG_F64 && vec_prec != GMG_F32)
    return fail(GMG_ERR_UNSUPPORTED, "wilson apply: vectors must be F64 or F32");
  KernelTimer kt("wilson", s);
  return wilson_dispatch(h, true, GMG_OP_M, 0, 0, vec_prec, nrhs, in, out, d1, d2, s);
}

}  // namespace gmg

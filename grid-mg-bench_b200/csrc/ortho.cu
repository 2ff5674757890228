// ortho.cu -- block orthonormalisation of the aggregation basis (FP64) and the
// orthogonality check.
//
// Restates blockLutedOrthonormalise (include/CoarsenedMatrixUpstreamImprovedDirsaveLut.h:
// 172-240; per-chirality form AggregationKernelsRework.h:266-341) and
// Aggregation::CheckOrthogonal (...LutMRHS.h:326-340).  The reference runs a
// modified Gram-Schmidt per block, one thread per block.  Here each pass is a
// Cholesky QR of every block's N x K panel V_c (K = block sites x site dof):
//
//   G_c = conj(V_c) V_c^T          (N x N Hermitian Gram matrix, G[i][j] = <v_i, v_j>_c)
//   G_c = L L^dag                   (Cholesky, L lower with a positive diagonal)
//   conj(L) W_c = V_c               (forward substitution, one column of V_c at a time)
//
// W_c is orthonormal and lower-triangularly related to V_c with a positive
// diagonal, the properties that fix the result of Gram-Schmidt: a thin QR with
// a positive R diagonal is unique, so both give the same basis up to rounding.
// Cholesky QR loses orthogonality as cond(V_c)^2; when a factorisation breaks
// down (smoothed test vectors can be nearly dependent inside a block) it is
// redone with the diagonal shift of shifted Cholesky QR (Fukaya, Kannan,
// Nakatsukasa, Yamamoto, Yanagisawa, SIAM J. Sci. Comput. 42 (2020)),
// s = 11 (K N + N (N + 1)) u ||V_c||_F^2, which always factors, and that block
// gets two extra plain passes.
//
// Three kernels per pass (nbasis up to 40):
//   gram_kernel      CTA per block (persistent over blocks): the Gram matrix on
//                    the FP64 tensor cores (mma m8n8k4 over the lower 8 x 8 tiles
//                    of the real panel's Gram matrix), fed by a three-stage
//                    cp.async pipeline of K-chunks with one barrier per chunk;
//                    writes the packed lower triangle.
//   factor_kernel    warp per block: the Cholesky factor in shared memory, lane
//                    i owning row i; the shifted retry re-reads the Gram matrix;
//                    writes conj(L) and 1 / diag(L) packed (row i: i + 1 entries).
//   tri_solve_kernel thread per column of V_c: the column in registers, forward
//                    substitution against conj(L) in shared memory (every thread
//                    reads the same entry: a broadcast), the column written back
//                    in place; the next column batch is copied into shared
//                    memory (cp.async) while the current one is solved.  (The
//                    same product as a block-lower-triangular real GEMM on the
//                    FP64 tensor cores, with T = conj(L)^{-1} formed explicitly,
//                    measured slower: 3.88 against 3.48 ms at 32^4 x 32, bound by
//                    the shared-memory reads of T's fragments.)
// Traffic per pass: the basis read twice and written once (3 x 8 B x 2 x N x K
// per block) plus the small factors; flops 8 K N (N + 1) / 2 for the Gram
// matrix (lower triangle) and the same for the substitution.
//
// Layout: basis_blk [c][i][k] complex128, k = sb * dof + a (one block's panel
// contiguous).
#include <algorithm>
#include <cmath>
#include <cstring>

#include "gmg_internal.cuh"

namespace gmg {
namespace ortho {

constexpr int kThreads = 256;
constexpr int kStages = 3;      // cp.async pipeline depth of the Gram kernel
constexpr int kSolveMax = 40;   // largest nbasis of the three-kernel path
constexpr int kFactorWarps = 4;  // blocks (one per warp) per factor CTA

__device__ __forceinline__ double2 cfma_conj(double2 acc, double2 a, double2 b) {  // acc += conj(a) b
  acc.x = fma(a.x, b.x, acc.x);
  acc.x = fma(a.y, b.y, acc.x);
  acc.y = fma(a.x, b.y, acc.y);
  acc.y = fma(-a.y, b.x, acc.y);
  return acc;
}

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(static_cast<uint32_t>(__cvta_generic_to_shared(smem))),
               "l"(gmem)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N_>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N_) : "memory"); }

// Geometry of the Gram kernel for nbasis N.  The block panel is staged as
// [KC][Np] complex (k-major), which read as doubles is the real 2N x KC panel W
// with rows 2i = Re v_i, 2i + 1 = Im v_i (rows 2N .. 8 NT - 1 zero).  Its real
// Gram matrix P = W W^T is formed with FP64 tensor-core MMAs (m8n8k4) over 8 x 8
// tiles: NT = ceil(N / 4) row tiles, the NT (NT + 1) / 2 lower tiles split over
// ntw "tile warps" (warp w takes the tile rows w and NT - 1 - w, so every warp
// has NT + 1 tiles) and K split over kgw groups of them.  Np = 4 mod 8 (16-byte
// units) puts the 32 lanes' fragment reads of one k-step on distinct bank
// pairs.  KC (a multiple of 4 kgw) and three stages fit three CTAs per SM
// (80 registers a thread): at N = 32, 2.49 ms per C3 pass (32^4, 4^4 blocks)
// against 2.83 ms at two CTAs per SM with 64-value chunks.
constexpr int kMaxNT = 10;  // nbasis <= 40 on this path
struct Geo {
  int N, NT, Np, ntw, kgw, KC, ntiles;
  size_t stage_bytes, pbuf_bytes, smem;
};

inline Geo geometry(int N) {
  Geo g;
  g.N = N;
  g.NT = (N + 3) / 4;
  g.Np = 4 * g.NT + (g.NT % 2 == 0 ? 4 : 0);
  g.ntw = (g.NT + 1) / 2;
  g.kgw = std::max(1, 8 / g.ntw);
  g.ntiles = g.NT * (g.NT + 1) / 2;
  g.KC = 32;
  for (int kc : {64, 32}) {  // both divide kThreads (the copy mapping relies on it)
    if ((kc / 4) % g.kgw) continue;
    if (sizeof(double2) * kStages * (size_t)kc * g.Np <= 72 * 1024) {
      g.KC = kc;
      break;
    }
  }
  g.stage_bytes = sizeof(double2) * kStages * (size_t)g.KC * g.Np;
  g.pbuf_bytes = sizeof(double) * 64 * (size_t)g.kgw * g.ntiles;
  g.smem = std::max(g.stage_bytes, g.pbuf_bytes);
  return g;
}

struct Params {
  double2* basis;              // [Vc][N][K]
  double2* gram;               // [Vc][N (N + 1) / 2]: G[i][j], j <= i
  double2* lfac;               // [Vc][N (N + 1) / 2]: conj(L[i][j]) for j < i, (1 / L[i][i], 0) for j = i
  int* need;                   // [Vc]: 1 once a block needed the shifted factorisation
  int* status;                 // 1 when a shifted factorisation failed too
  unsigned long long* maxerr;  // check mode: max |G - 1| (as the bits of a non-negative double)
  int Vc, N, K, Np, ntw, kgw, KC, ntiles;
  int pass, passes;
};

__device__ __forceinline__ bool block_active(const Params& P, int c) { return P.pass < P.passes || P.need[c] != 0; }

// D (8 x 8, two elements per lane) += A (8 x 4) B (4 x 8), FP64 tensor cores
__device__ __forceinline__ void dmma(double (&d)[2], double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
               : "+d"(d[0]), "+d"(d[1])
               : "d"(a), "d"(b));
}

// The k-steps of one chunk for the warp whose tile rows are TW and NT - 1 - TW:
// per step of 4 k values one fragment load per tile row it needs and one MMA
// per tile, all indices compile-time.
template <int NT, int TW>
__device__ __forceinline__ void gram_steps(double (&acc)[NT + 1][2], const double* fb, int stride_d, int grp, int nk4,
                                           int kgw) {
  constexpr int I1 = TW, I2 = NT - 1 - TW;
  if (NT > 4) {
    // (the register budget of three CTAs per SM holds one set of fragments only)
    for (int k4 = grp; k4 < nk4; k4 += kgw) {
      const double* f = fb + 4 * k4 * stride_d;
      double fr[I2 + 1];
#pragma unroll
      for (int X = 0; X <= I2; ++X) fr[X] = f[8 * X];
#pragma unroll
      for (int J = 0; J <= I1; ++J) dmma(acc[J], fr[I1], fr[J]);
      if (I2 != I1) {
#pragma unroll
        for (int J = 0; J <= I2; ++J) dmma(acc[I1 + 1 + J], fr[I2], fr[J]);
      }
    }
    return;
  }
  if (grp >= nk4) return;
  // the fragments of the next step are loaded while this step's MMAs issue
  double fr[I2 + 1], fn[I2 + 1];
#pragma unroll
  for (int X = 0; X <= I2; ++X) fr[X] = fb[4 * grp * stride_d + 8 * X];
  for (int k4 = grp; k4 < nk4; k4 += kgw) {
    const int kn = k4 + kgw;
    if (kn < nk4) {
      const double* f = fb + 4 * kn * stride_d;
#pragma unroll
      for (int X = 0; X <= I2; ++X) fn[X] = f[8 * X];
    }
#pragma unroll
    for (int J = 0; J <= I1; ++J) dmma(acc[J], fr[I1], fr[J]);
    if (I2 != I1) {
#pragma unroll
      for (int J = 0; J <= I2; ++J) dmma(acc[I1 + 1 + J], fr[I2], fr[J]);
    }
#pragma unroll
    for (int X = 0; X <= I2; ++X) fr[X] = fn[X];
  }
}

template <int NT>
__device__ __forceinline__ void gram_steps_tw(int tw, double (&acc)[NT + 1][2], const double* fb, int stride_d, int grp,
                                              int nk4, int kgw) {
  switch (tw) {
    case 0: gram_steps<NT, 0>(acc, fb, stride_d, grp, nk4, kgw); break;
    case 1: if (NT > 2) gram_steps<NT, (NT > 2 ? 1 : 0)>(acc, fb, stride_d, grp, nk4, kgw); break;
    case 2: if (NT > 4) gram_steps<NT, (NT > 4 ? 2 : 0)>(acc, fb, stride_d, grp, nk4, kgw); break;
    case 3: if (NT > 6) gram_steps<NT, (NT > 6 ? 3 : 0)>(acc, fb, stride_d, grp, nk4, kgw); break;
    default: if (NT > 8) gram_steps<NT, (NT > 8 ? 4 : 0)>(acc, fb, stride_d, grp, nk4, kgw); break;
  }
}

// Gram matrices of the blocks (packed lower triangles into P.gram), or in
// CHECK mode the largest |G - 1| over all blocks into P.maxerr.
template <int NT, bool CHECK>
__global__ void __launch_bounds__(kThreads, 3) gram_kernel(Params P) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double2* stage = reinterpret_cast<double2*>(smem_raw);  // [kStages][KC][Np], then the P tiles
  double* pbuf = reinterpret_cast<double*>(smem_raw);
  const int t = threadIdx.x, lane = t & 31, w = t >> 5;
  const int Np = P.Np, N = P.N, K = P.K, KC = P.KC, kgw = P.kgw, ntw = P.ntw;
  const int stride_d = 2 * Np;  // doubles per staged k row
  const int tw = w % ntw, grp = w / ntw;
  const bool active = grp < kgw;
  const int I1 = tw, I2 = NT - 1 - tw;  // this warp's tile rows (the same when NT is odd and tw is the middle)
  const int nch = (K + KC - 1) / KC;
  const int stage_elems = kStages * KC * Np;
  // KC (32 or 64) divides the thread count: a thread copies one k offset of
  // every chunk, for every (kThreads / KC)-th row, with no division per copy
  const int kshift = KC == 64 ? 6 : 5;
  const int ckk = t & (KC - 1), ci0 = t >> kshift, istep = kThreads >> kshift;
  // zero the staging buffers once: rows i >= N and k rows past the end of a
  // partial last chunk must read as zero
  for (int e = t; e < stage_elems; e += kThreads) stage[e] = make_double2(0.0, 0.0);
  __syncthreads();
  double mx = 0.0;
  for (int c = blockIdx.x; c < P.Vc; c += gridDim.x) {
    if (!CHECK && !block_active(P, c)) continue;  // uniform over the CTA
    const double2* Vb = P.basis + (int64_t)c * N * K;
    auto issue = [&](int ch) {
      if (ch < nch) {
        double2* buf = stage + (ch % kStages) * KC * Np;
        const int k0 = ch * KC;
        const int kc = min(KC, K - k0);
        // this thread's copies: k offset ckk, rows ci0, ci0 + istep, ...
        if (ckk < kc) {
          const double2* src = Vb + (int64_t)ci0 * K + k0 + ckk;
          for (int i = ci0; i < N; i += istep, src += (int64_t)istep * K) cp_async16(buf + ckk * Np + i, src);
        }
        if (kc < KC) {
          // a partial last chunk: the k rows up to the next multiple of 4 read as zero
          const int kc4 = (kc + 3) & ~3;
          for (int e = t; e < (kc4 - kc) * Np; e += kThreads)
            buf[(kc + e / Np) * Np + e % Np] = make_double2(0.0, 0.0);
        }
      }
      cp_async_commit();  // an empty group past the last chunk keeps the group count uniform
    };
    double acc[NT + 1][2];
#pragma unroll
    for (int q = 0; q <= NT; ++q) acc[q][0] = acc[q][1] = 0.0;
    __syncthreads();  // the previous block's P tiles are no longer read
#pragma unroll
    for (int sidx = 0; sidx < kStages - 1; ++sidx) issue(sidx);
    for (int ch = 0; ch < nch; ++ch) {
      cp_async_wait<kStages - 2>();  // this thread's copies of chunk ch have landed
      __syncthreads();               // everyone's have; chunk ch - 1 is no longer read
      issue(ch + kStages - 1);       // into the buffer chunk ch - 1 used
      if (active) {
        const double* buf = reinterpret_cast<const double*>(stage + (ch % kStages) * KC * Np);
        const int nk4 = (min(KC, K - ch * KC) + 3) >> 2;
        // lane (r, q) = (lane / 4, lane % 4): A / B fragment element W[8 X + r][k + q]
        const double* fb = buf + (lane & 3) * stride_d + (lane >> 2);
        gram_steps_tw<NT>(tw, acc, fb, stride_d, grp, nk4, kgw);
      }
    }
    cp_async_wait<0>();
    __syncthreads();  // all chunks consumed: the stage area takes the P tiles
    if (active) {
      // tile (I, J) of group grp: element (m, n) at pbuf[((grp * ntiles + I (I + 1) / 2 + J) * 8 + m) * 8 + n];
      // this lane holds (m, n) = (lane / 4, 2 (lane % 4) + {0, 1}); tile slot q of the accumulators is
      // (I1, q) for q <= I1, (I2, q - I1 - 1) after
      const int off = (lane >> 2) * 8 + 2 * (lane & 3);
#pragma unroll
      for (int q = 0; q <= NT; ++q) {
        const int I = q <= I1 ? I1 : I2, J = q <= I1 ? q : q - I1 - 1;
        if (q <= I1 || (I2 != I1 && J <= I2)) {
          double* d = pbuf + ((size_t)(grp * P.ntiles + I * (I + 1) / 2 + J) * 64) + off;
          d[0] = acc[q][0];
          d[1] = acc[q][1];
        }
      }
    }
    __syncthreads();
    // P(R, R') for R >= R', summed over the K groups
    auto pel = [&](int R, int R2) {
      if (R < R2) {
        const int tmp = R;
        R = R2;
        R2 = tmp;
      }
      const int I = R >> 3, J = R2 >> 3;
      const double* src = pbuf + (size_t)(I * (I + 1) / 2 + J) * 64 + (R & 7) * 8 + (R2 & 7);
      double v = 0.0;
      for (int g = 0; g < kgw; ++g) v += src[(size_t)g * P.ntiles * 64];
      return v;
    };
    double2* Gc = P.gram + (int64_t)c * (N * (N + 1) / 2);
    for (int e = t; e < N * N; e += kThreads) {
      const int i = e / N, j = e - (e / N) * N;
      if (j > i) continue;
      const double gr = pel(2 * i, 2 * j) + pel(2 * i + 1, 2 * j + 1);
      const double gi = i == j ? 0.0 : pel(2 * i, 2 * j + 1) - pel(2 * i + 1, 2 * j);
      if (CHECK) {
        const double re = gr - (i == j ? 1.0 : 0.0);
        mx = fmax(mx, sqrt(re * re + gi * gi));
      } else {
        Gc[i * (i + 1) / 2 + j] = make_double2(gr, gi);
      }
    }
    __syncthreads();  // P tiles read: zero the staging rows i >= N again for the next block
    if (N < 4 * NT)
      for (int e = t; e < kStages * KC * (4 * NT - N); e += kThreads) {
        const int row = e / (4 * NT - N), col = N + e % (4 * NT - N);
        stage[row * Np + col] = make_double2(0.0, 0.0);
      }
  }
  if (CHECK) atomicMax(P.maxerr, (unsigned long long)__double_as_longlong(mx));  // non-negative doubles order as integers
}

// Cholesky factor of one block's Gram matrix by one warp: G + shift I = L L^dag,
// rows in shared memory at stride N + 1 (lane i owns rows i and i + 32), the
// strict lower triangle of L in place of G, the diagonal in diag[].  Returns
// false when a pivot is not positive (replaced by 1 so that L stays finite).
__device__ bool warp_cholesky(double2* G, double* diag, int N, double shift) {
  const int lane = threadIdx.x & 31, Sp = N + 1;
  bool ok = true;
  for (int j = 0; j < N; ++j) {
    double d = G[j * Sp + j].x + shift;
    if (!(d > 0.0)) {
      ok = false;
      d = 1.0;
    }
    const double dj = sqrt(d), inv = 1.0 / dj;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int i = lane + 32 * h;
      if (i > j && i < N) {
        const double2 v = G[i * Sp + j];
        G[i * Sp + j] = make_double2(v.x * inv, v.y * inv);
      }
    }
    if (lane == 0) diag[j] = dj;
    __syncwarp();
    // trailing update G[i][k] -= L[i][j] conj(L[k][j]), j < k <= i: lane i walks
    // k in step with the other lanes, so L[k][j] is one broadcast read
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int i = lane + 32 * h;
      if (i > j && i < N) {
        const double2 a = G[i * Sp + j];
#pragma unroll 4
        for (int k = j + 1; k <= i; ++k) {
          const double2 b = G[k * Sp + j];
          double2 g = G[i * Sp + k];
          g.x -= a.x * b.x + a.y * b.y;
          g.y -= a.y * b.x - a.x * b.y;
          G[i * Sp + k] = g;
        }
      }
    }
    __syncwarp();
  }
  return ok;
}

__global__ void __launch_bounds__(32 * kFactorWarps) factor_kernel(Params P) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int N = P.N, Sp = N + 1, lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int c = blockIdx.x * kFactorWarps + w;
  if (c >= P.Vc || !block_active(P, c)) return;  // whole warps leave; no block-wide barrier follows
  double2* G = reinterpret_cast<double2*>(smem_raw) + (size_t)w * N * Sp;
  double* diag = reinterpret_cast<double*>(reinterpret_cast<double2*>(smem_raw) + (size_t)kFactorWarps * N * Sp) +
                 (size_t)w * N;
  const int nl = N * (N + 1) / 2;
  const double2* Gc = P.gram + (int64_t)c * nl;
  auto load = [&]() {
    for (int i = 0; i < N; ++i)
      for (int j = lane; j <= i; j += 32) G[i * Sp + j] = Gc[i * (i + 1) / 2 + j];
    __syncwarp();
  };
  load();
  bool ok = warp_cholesky(G, diag, N, 0.0);
  if (!ok) {
    // shifted Cholesky QR on the same Gram matrix, and two extra passes for this block
    load();
    double tr = 0.0;
    for (int i = lane; i < N; i += 32) tr += G[i * Sp + i].x;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) tr += __shfl_xor_sync(0xffffffffu, tr, off);
    const double shift = 11.0 * ((double)P.K * N + (double)N * (N + 1)) * 1.1102230246251565e-16 * tr;
    ok = warp_cholesky(G, diag, N, shift);
    if (lane == 0) {
      P.need[c] = 1;
      if (!ok) atomicExch(P.status, 1);
    }
  }
  double2* Lc = P.lfac + (int64_t)c * nl;
  for (int i = 0; i < N; ++i)
    for (int j = lane; j <= i; j += 32) {
      const double2 v = G[i * Sp + j];
      Lc[i * (i + 1) / 2 + j] = j < i ? make_double2(v.x, -v.y) : make_double2(1.0 / diag[i], 0.0);
    }
}

constexpr int kSolveThreads = 128;  // columns per solve chunk (three CTAs per SM at N = 32)

// W = conj(L)^{-1} V for every column of every block: thread per column, the
// column in registers (NMAX entries, rows >= N unused), conj(L) in shared
// memory; the CTA walks the blocks of its grid stride and every 256-column
// chunk of each, with the next chunk's columns copied into shared memory while
// the current chunk is solved.
// EXACT: nbasis equals NMAX, so that every row bound is a compile-time
// constant (no guards between the row groups' independent products; at
// N = 32 that also frees registers: 176 instead of 214, and 168 without
// spills at three CTAs per SM, tri_solve32_kernel).  C3 (32^4, 4^4 blocks,
// N 32): 3.26 ms with the guards at two CTAs per SM, 2.98 ms without, 2.83 ms
// without at three.
template <int NMAX, bool EXACT>
__device__ __forceinline__ void tri_solve_body(const Params& P) {
  constexpr int NTS = kSolveThreads;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double2* pre = reinterpret_cast<double2*>(smem_raw);  // [NMAX][NTS]: the prefetched columns
  double2* L = pre + NMAX * NTS;                        // packed conj(L) of the current block
  const int N = EXACT ? NMAX : P.N, K = P.K, t = threadIdx.x;
  const int nl = N * (N + 1) / 2;
  const int chunks = (K + NTS - 1) / NTS;
  // this CTA's work items (block, chunk) in order, skipping inactive blocks
  auto next_block = [&](int c) {
    for (; c < P.Vc; c += gridDim.x)
      if (block_active(P, c)) return c;
    return P.Vc;
  };
  auto prefetch = [&](int c, int ch) {
    const int k = ch * NTS + t;
    if (c < P.Vc && k < K) {
      const double2* col = P.basis + (int64_t)c * N * K + k;
#pragma unroll
      for (int i = 0; i < NMAX; ++i)
        if (i < N) cp_async16(pre + i * NTS + t, col + (int64_t)i * K);
    }
    cp_async_commit();
  };
  int c = next_block(blockIdx.x), ch = 0;
  int lc = -1;  // the block whose factor is in L
  prefetch(c, ch);
  while (c < P.Vc) {
    // the item after this one
    int nc = c, nch = ch + 1;
    if (nch == chunks) {
      nc = next_block(c + gridDim.x);
      nch = 0;
    }
    if (c != lc) {
      __syncthreads();  // every thread is done with the previous block's factor
      const double2* src = P.lfac + (int64_t)c * nl;
      for (int e = t; e < nl; e += NTS) L[e] = src[e];
      __syncthreads();
      lc = c;
    }
    cp_async_wait<0>();  // this thread's columns of the current item (its own slots only)
    const int k = ch * NTS + t;
    double2 w[NMAX];
#pragma unroll
    for (int i = 0; i < NMAX; ++i) w[i] = (i < N && k < K) ? pre[i * NTS + t] : make_double2(0.0, 0.0);
    prefetch(nc, nch);  // the slots are free again: copy the next item's columns meanwhile
    if (k < K) {
      // rows in groups of four: the products with the already solved entries
      // (j below the group) are independent across the group's rows, two
      // partial sums each, so eight chains run side by side; then the group's
      // own 4 x 4 triangle in order
#pragma unroll
      for (int i0 = 0; i0 < NMAX; i0 += 4) {
        if (i0 < N) {
          double2 sp[4][2];
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            sp[q][0] = (i0 + q < N) ? w[i0 + q] : make_double2(0.0, 0.0);
            sp[q][1] = make_double2(0.0, 0.0);
          }
#pragma unroll
          for (int j = 0; j < i0; ++j) {
#pragma unroll
            for (int q = 0; q < 4; ++q) {  // s -= conj(L[i][j]) w[j]
              const int i = i0 + q;
              if (i < NMAX && i < N) {  // L holds the N (N + 1) / 2 entries of rows i < N only
                const double2 a = L[i * (i + 1) / 2 + j];
                double2& sq = sp[q][j & 1];
                sq.x = fma(-a.x, w[j].x, sq.x);
                sq.x = fma(a.y, w[j].y, sq.x);
                sq.y = fma(-a.x, w[j].y, sq.y);
                sq.y = fma(-a.y, w[j].x, sq.y);
              }
            }
          }
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            const int i = i0 + q;
            if (i < NMAX && i < N) {
              const double2* Li = L + i * (i + 1) / 2;
              double2 sq = make_double2(sp[q][0].x + sp[q][1].x, sp[q][0].y + sp[q][1].y);
#pragma unroll
              for (int j = i0; j < i; ++j) {
                const double2 a = Li[j];
                sq.x = fma(-a.x, w[j].x, sq.x);
                sq.x = fma(a.y, w[j].y, sq.x);
                sq.y = fma(-a.x, w[j].y, sq.y);
                sq.y = fma(-a.y, w[j].x, sq.y);
              }
              const double inv = Li[i].x;
              w[i] = make_double2(sq.x * inv, sq.y * inv);
            }
          }
        }
      }
      double2* col = P.basis + (int64_t)c * N * K + k;
#pragma unroll
      for (int i = 0; i < NMAX; ++i)
        if (i < N) col[(int64_t)i * K] = w[i];
    }
    c = nc;
    ch = nch;
  }
  cp_async_wait<0>();
}

template <int NMAX, bool EXACT>
__global__ void __launch_bounds__(kSolveThreads) tri_solve_kernel(Params P) {
  tri_solve_body<NMAX, EXACT>(P);
}

__global__ void __launch_bounds__(kSolveThreads, 3) tri_solve32_kernel(Params P) { tri_solve_body<32, true>(P); }

// Cholesky G + shift I = L L^dag in place by the whole CTA (strict lower
// triangle of G, row-major N x N; the diagonal goes to diag[]); false to every
// thread when a pivot is not positive (replaced by 1).  Used by the one-CTA-
// per-block path below.
__device__ bool block_cholesky(double2* G, double* diag, int N, double shift, int* fail_s) {
  const int t = threadIdx.x;
  if (t == 0) *fail_s = 0;
  __syncthreads();
  for (int j = 0; j < N; ++j) {
    double d = G[j * N + j].x + shift;
    const bool bad = !(d > 0.0);
    if (bad) d = 1.0;
    const double dj = sqrt(d), inv = 1.0 / dj;
    for (int i = j + 1 + t; i < N; i += kThreads) {
      const double2 v = G[i * N + j];
      G[i * N + j] = make_double2(v.x * inv, v.y * inv);
    }
    if (t == 0) {
      diag[j] = dj;
      if (bad) *fail_s = 1;
    }
    __syncthreads();
    const int m = N - j - 1;
    for (int e = t; e < m * (m + 1) / 2; e += kThreads) {
      int ii = (int)((sqrtf(8.0f * e + 1.0f) - 1.0f) * 0.5f);
      while (ii * (ii + 1) / 2 > e) --ii;
      while ((ii + 1) * (ii + 2) / 2 <= e) ++ii;
      const int kk = e - ii * (ii + 1) / 2;
      const int i = j + 1 + ii, k = j + 1 + kk;
      const double2 a = G[i * N + j], b = G[k * N + j];
      double2 g = G[i * N + k];
      g.x -= a.x * b.x + a.y * b.y;
      g.y -= a.y * b.x - a.x * b.y;
      G[i * N + k] = g;
    }
    __syncthreads();
  }
  return *fail_s == 0;
}

// ---------------------------------------------------------------------------
// one CTA per block for nbasis above the two-kernel path (up to 64): the same
// Cholesky QR with the whole block's transform applied from shared memory
// ---------------------------------------------------------------------------
constexpr int kBigKS = 2;  // sites per K chunk

__device__ void big_gram(const double2* __restrict__ Vb, int N, int64_t K, int dof, double2* VT, double2* G) {
  const int t = threadIdx.x;
  const int NTl = (N + 3) / 4;
  const int ntiles = NTl * NTl;
  const int ti = t % NTl, tj = t / NTl;
  double2 acc[4][4];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) acc[a][b] = make_double2(0, 0);
  const int KC = kBigKS * dof;
  for (int64_t k0 = 0; k0 < K; k0 += KC) {
    const int kc = (int)((K - k0) < (int64_t)KC ? (K - k0) : (int64_t)KC);
    __syncthreads();
    for (int e = t; e < N * kc; e += blockDim.x) {
      const int i = e / kc, kk = e % kc;
      VT[kk * N + i] = Vb[(int64_t)i * K + k0 + kk];
    }
    __syncthreads();
    if (t < ntiles) {
      for (int kk = 0; kk < kc; ++kk) {
        double2 a[4], b[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const int i = ti * 4 + q, j = tj * 4 + q;
          a[q] = i < N ? VT[kk * N + i] : make_double2(0, 0);
          b[q] = j < N ? VT[kk * N + j] : make_double2(0, 0);
        }
#pragma unroll
        for (int x = 0; x < 4; ++x)
#pragma unroll
          for (int y = 0; y < 4; ++y) acc[x][y] = cfma_conj(acc[x][y], a[x], b[y]);
      }
    }
  }
  __syncthreads();
  if (t < ntiles) {
#pragma unroll
    for (int x = 0; x < 4; ++x)
#pragma unroll
      for (int y = 0; y < 4; ++y) {
        const int i = ti * 4 + x, j = tj * 4 + y;
        if (i < N && j < N) G[i * N + j] = acc[x][y];
      }
  }
  __syncthreads();
}

__global__ void __launch_bounds__(kThreads) big_ortho_kernel(double2* __restrict__ basis, int Vc, int N, int dof,
                                                             int bv, int passes, int* __restrict__ status) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double2* G = reinterpret_cast<double2*>(smem_raw);  // [N][N]  Gram, then L
  double2* Li = G + N * N;                             // [N][N]  conj(L^{-1})
  double* diag = reinterpret_cast<double*>(Li + N * N);
  double2* VT = reinterpret_cast<double2*>(diag + N + (N & 1));  // [KC][N] staging
  __shared__ int fail_s;
  __shared__ double trace_s;
  const int64_t K = (int64_t)bv * dof;
  const int t = threadIdx.x;
  for (int c = blockIdx.x; c < Vc; c += gridDim.x) {
    double2* Vb = basis + (int64_t)c * N * K;
    int extra = 0;
    for (int pass = 0; pass < passes + extra; ++pass) {
      big_gram(Vb, N, K, dof, VT, G);
      if (!block_cholesky(G, diag, N, 0.0, &fail_s)) {
        big_gram(Vb, N, K, dof, VT, G);
        if (t == 0) {
          double tr = 0.0;
          for (int i = 0; i < N; ++i) tr += G[i * N + i].x;
          trace_s = tr;
        }
        __syncthreads();
        const double shift = 11.0 * ((double)K * N + (double)N * (N + 1)) * 1.1102230246251565e-16 * trace_s;
        if (!block_cholesky(G, diag, N, shift, &fail_s) && t == 0) atomicExch(status, 1);
        if (extra < 2) extra = 2;
      }
      // conj(L^{-1}) column by column (one thread per column)
      for (int j = t; j < N; j += blockDim.x) {
        for (int i = 0; i < N; ++i) Li[i * N + j] = make_double2(0, 0);
        Li[j * N + j] = make_double2(1.0 / diag[j], 0.0);
        for (int i = j + 1; i < N; ++i) {
          double2 sacc = make_double2(0, 0);
          for (int k = j; k < i; ++k) {
            const double2 a = k == i ? make_double2(diag[i], 0.0) : G[i * N + k], x = Li[k * N + j];
            sacc.x += a.x * x.x - a.y * x.y;
            sacc.y += a.x * x.y + a.y * x.x;
          }
          const double inv = 1.0 / diag[i];
          Li[i * N + j] = make_double2(-sacc.x * inv, -sacc.y * inv);
        }
        for (int i = j; i < N; ++i) Li[i * N + j].y = -Li[i * N + j].y;
      }
      __syncthreads();
      const int KC = kBigKS * dof;
      for (int64_t k0 = 0; k0 < K; k0 += KC) {
        const int kc = (int)((K - k0) < (int64_t)KC ? (K - k0) : (int64_t)KC);
        __syncthreads();
        for (int e = t; e < N * kc; e += blockDim.x) {
          const int i = e / kc, kk = e % kc;
          VT[kk * N + i] = Vb[(int64_t)i * K + k0 + kk];
        }
        __syncthreads();
        for (int e = t; e < N * kc; e += blockDim.x) {
          const int i = e / kc, kk = e % kc;
          double2 acc = make_double2(0, 0);
          for (int j = 0; j <= i; ++j) {
            const double2 l = Li[i * N + j], v = VT[kk * N + j];
            acc.x = fma(l.x, v.x, acc.x);
            acc.x = fma(-l.y, v.y, acc.x);
            acc.y = fma(l.x, v.y, acc.y);
            acc.y = fma(l.y, v.x, acc.y);
          }
          Vb[(int64_t)i * K + k0 + kk] = acc;
        }
      }
      __syncthreads();
    }
  }
}

// the orthogonality check above nbasis 40: one CTA per block, max |G - 1|
__global__ void __launch_bounds__(kThreads) big_check_kernel(const double2* __restrict__ basis, int Vc, int N, int dof,
                                                             int bv, unsigned long long* __restrict__ maxerr) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double2* G = reinterpret_cast<double2*>(smem_raw);  // [N][N]
  double2* VT = G + N * N;                             // [KC][N] staging
  const int64_t K = (int64_t)bv * dof;
  double mx = 0.0;
  for (int c = blockIdx.x; c < Vc; c += gridDim.x) {
    big_gram(basis + (int64_t)c * N * K, N, K, dof, VT, G);
    for (int e = threadIdx.x; e < N * N; e += blockDim.x) {
      const int i = e / N, j = e % N;
      const double re = G[e].x - (i == j ? 1.0 : 0.0), im = G[e].y;
      mx = fmax(mx, sqrt(re * re + im * im));
    }
    __syncthreads();
  }
  atomicMax(maxerr, (unsigned long long)__double_as_longlong(mx));
}

static int num_sms() {
  int dev = 0, n = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
  return n;
}

// workspace: [status int + max error][need int Vc][Gram Vc x N (N + 1) / 2][conj(L) same]
static gmg_status workspace(gmg_agg* h, Params* P) {
  const int64_t Vc = h->cdims.vol();
  const size_t head = 256, need_b = (size_t)(Vc * sizeof(int) + 255) / 256 * 256;
  const size_t lf_b = sizeof(double2) * (size_t)Vc * (h->N * (h->N + 1) / 2);
  const void* before = h->ortho_ws.p;
  GMG_TRY(h->ortho_ws.alloc(head + need_b + 2 * lf_b));
  char* p = h->ortho_ws.as<char>();
  if (p != before) GMG_CUDA(cudaMemset(p, 0, head));  // fresh memory: no failure recorded yet
  const Geo g = geometry(h->N);
  P->basis = h->basis_blk.as<double2>();
  P->status = reinterpret_cast<int*>(p);
  P->maxerr = reinterpret_cast<unsigned long long*>(p + 8);
  P->need = reinterpret_cast<int*>(p + head);
  P->gram = reinterpret_cast<double2*>(p + head + need_b);
  P->lfac = reinterpret_cast<double2*>(p + head + need_b + lf_b);
  P->Vc = (int)Vc;
  P->N = h->N;
  P->K = h->bv * h->dof;
  P->Np = g.Np;
  P->ntw = g.ntw;
  P->kgw = g.kgw;
  P->KC = g.KC;
  P->ntiles = g.ntiles;
  P->pass = 0;
  P->passes = 1;
  return GMG_OK;
}

template <int NT, bool CHECK>
static gmg_status launch_gram_nt(const Params& P, const Geo& g, cudaStream_t s) {
  auto kern = gram_kernel<NT, CHECK>;
  GMG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)g.smem));
  int per_sm = 1;
  GMG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kThreads, g.smem));
  const int grid = std::min(P.Vc, num_sms() * std::max(per_sm, 1));
  kern<<<grid, kThreads, g.smem, s>>>(P);
  GMG_CUDA(cudaGetLastError());
  return GMG_OK;
}

template <bool CHECK>
static gmg_status launch_gram(const Params& P, cudaStream_t s) {
  const Geo g = geometry(P.N);
  GMG_CHECK(g.NT <= kMaxNT, GMG_ERR_UNSUPPORTED, "orthonormalise: nbasis above the tensor-core Gram path");
  GMG_CHECK(g.smem <= 227 * 1024, GMG_ERR_UNSUPPORTED, "orthonormalise: tile does not fit shared memory");
  GMG_CHECK((g.KC == 32 || g.KC == 64) && kThreads % g.KC == 0, GMG_ERR_UNSUPPORTED, "orthonormalise: chunk size");
  switch (g.NT) {
    case 1: return launch_gram_nt<1, CHECK>(P, g, s);
    case 2: return launch_gram_nt<2, CHECK>(P, g, s);
    case 3: return launch_gram_nt<3, CHECK>(P, g, s);
    case 4: return launch_gram_nt<4, CHECK>(P, g, s);
    case 5: return launch_gram_nt<5, CHECK>(P, g, s);
    case 6: return launch_gram_nt<6, CHECK>(P, g, s);
    case 7: return launch_gram_nt<7, CHECK>(P, g, s);
    case 8: return launch_gram_nt<8, CHECK>(P, g, s);
    case 9: return launch_gram_nt<9, CHECK>(P, g, s);
    default: return launch_gram_nt<10, CHECK>(P, g, s);
  }
}

static gmg_status launch_factor(const Params& P, cudaStream_t s) {
  const size_t smem = (sizeof(double2) * (size_t)P.N * (P.N + 1) + sizeof(double) * P.N) * kFactorWarps;
  GMG_CUDA(cudaFuncSetAttribute(factor_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  factor_kernel<<<(P.Vc + kFactorWarps - 1) / kFactorWarps, 32 * kFactorWarps, smem, s>>>(P);
  GMG_CUDA(cudaGetLastError());
  return GMG_OK;
}

template <int NMAX>
static gmg_status launch_solve(const Params& P, cudaStream_t s) {
  const size_t smem = sizeof(double2) * ((size_t)NMAX * kSolveThreads + (size_t)P.N * (P.N + 1) / 2);
  void (*kern)(Params) = tri_solve_kernel<NMAX, false>;
  if (P.N == NMAX) {
    if constexpr (NMAX == 32)
      kern = tri_solve32_kernel;
    else
      kern = tri_solve_kernel<NMAX, true>;
  }
  GMG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int per_sm = 1;
  GMG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kSolveThreads, smem));
  const int grid = std::min(P.Vc, num_sms() * std::max(per_sm, 1));
  kern<<<grid, kSolveThreads, smem, s>>>(P);
  GMG_CUDA(cudaGetLastError());
  return GMG_OK;
}

static gmg_status solve(const Params& P, cudaStream_t s) {
  if (P.N <= 8) return launch_solve<8>(P, s);
  if (P.N <= 16) return launch_solve<16>(P, s);
  if (P.N <= 24) return launch_solve<24>(P, s);
  if (P.N <= 32) return launch_solve<32>(P, s);
  return launch_solve<40>(P, s);
}

}  // namespace ortho

gmg_status agg_orthonormalise(gmg_agg* h, int passes, cudaStream_t s) {
  using namespace ortho;
  const int N = h->N;
  Params P;
  GMG_TRY(workspace(h, &P));
  const int Vc = P.Vc;
  GMG_CUDA(cudaMemsetAsync(P.status, 0, sizeof(int), s));
  if (N > kSolveMax) {
    GMG_CHECK(N <= 64, GMG_ERR_UNSUPPORTED, "orthonormalise: nbasis > 64");
    const size_t smem = sizeof(double2) * ((size_t)2 * N * N + (size_t)kBigKS * h->dof * N) +
                        sizeof(double) * (N + (N & 1));
    GMG_CHECK(smem <= 227 * 1024, GMG_ERR_UNSUPPORTED, "orthonormalise: nbasis x site dof too large");
    GMG_CUDA(cudaFuncSetAttribute(big_ortho_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    KernelTimer kt("ortho", s);
    big_ortho_kernel<<<std::min(Vc, num_sms() * 8), kThreads, smem, s>>>(h->basis_blk.as<double2>(), Vc, N, h->dof,
                                                                        h->bv, passes, P.status);
    GMG_CUDA(cudaGetLastError());
  } else {
    GMG_CUDA(cudaMemsetAsync(P.need, 0, sizeof(int) * Vc, s));
    P.passes = passes;
    KernelTimer kt("ortho", s);
    // passes + 2 rounds: the last two only touch blocks that needed the shift
    for (int pass = 0; pass < passes + 2; ++pass) {
      P.pass = pass;
      {
        KernelTimer k1("ortho_gram", s);
        GMG_TRY(launch_gram<false>(P, s));
      }
      {
        KernelTimer k2("ortho_factor", s);
        GMG_TRY(launch_factor(P, s));
      }
      KernelTimer k3("ortho_solve", s);
      GMG_TRY(solve(P, s));
    }
  }
  h->basis_f_ok = false;
  h->basis_tc_ok = false;
  return GMG_OK;
}

gmg_status agg_check_orthogonal(gmg_agg* h, double* max_err, cudaStream_t s) {
  using namespace ortho;
  Params P;
  GMG_TRY(workspace(h, &P));
  GMG_CUDA(cudaMemsetAsync(P.maxerr, 0, sizeof(unsigned long long), s));
  if (h->N > kSolveMax) {
    const size_t smem = sizeof(double2) * ((size_t)h->N * h->N + (size_t)kBigKS * h->dof * h->N);
    GMG_CHECK(smem <= 227 * 1024, GMG_ERR_UNSUPPORTED, "check orthogonal: nbasis x site dof too large");
    GMG_CUDA(cudaFuncSetAttribute(big_check_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    big_check_kernel<<<std::min(P.Vc, num_sms() * 8), kThreads, smem, s>>>(h->basis_blk.as<double2>(), P.Vc, h->N,
                                                                          h->dof, h->bv, P.maxerr);
    GMG_CUDA(cudaGetLastError());
  } else {
    GMG_TRY(launch_gram<true>(P, s));
  }
  unsigned long long v = 0;
  int st = 0;
  GMG_CUDA(cudaMemcpyAsync(&v, P.maxerr, sizeof(v), cudaMemcpyDeviceToHost, s));
  GMG_CUDA(cudaMemcpyAsync(&st, P.status, sizeof(int), cudaMemcpyDeviceToHost, s));
  GMG_CUDA(cudaStreamSynchronize(s));
  double r;
  memcpy(&r, &v, sizeof(r));
  *max_err = r;
  if (st) return fail(GMG_ERR_NONFINITE, "orthonormalise: a block Gram matrix was singular even with the shift");
  return GMG_OK;
}

}  // namespace gmg

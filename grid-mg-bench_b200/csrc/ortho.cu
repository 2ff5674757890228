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
//   gram_kernel      CTA per block (persistent over blocks): the Gram matrix
//                    from FP64 register tiles over the lower block triangle, fed
//                    by a three-stage cp.async pipeline of K-chunks with one
//                    barrier per chunk; writes the packed lower triangle.
//   factor_kernel    warp per block: the Cholesky factor in shared memory, lane
//                    i owning row i; the shifted retry re-reads the Gram matrix;
//                    writes conj(L) and 1 / diag(L) packed (row i: i + 1 entries).
//   tri_solve_kernel thread per column of V_c: the column in registers, forward
//                    substitution against conj(L) in shared memory (every thread
//                    reads the same entry: a broadcast), the column written back
//                    in place; the next column batch is copied into shared
//                    memory (cp.async) while the current one is solved.
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
constexpr int kKC = 64;         // K values per pipeline stage (at most)
constexpr int kStages = 3;      // cp.async pipeline depth of the Gram kernel
constexpr int kMaxKG = 16;      // K-interleaved groups of tile threads
constexpr int kSolveMax = 40;   // largest nbasis of the three-kernel path
constexpr int kFactorWarps = 4;  // blocks (one per warp) per factor CTA
constexpr int kSolveThreads = 128;  // columns per solve chunk (three CTAs per SM at 170 registers)

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

// Tile geometry of the Gram matrix for nbasis N: NT tiles per side, tile (ti, tj)
// owning rows ti + NT q and columns tj + NT r (q, r < 4), only ti >= tj (the
// others are conjugate transposes); KG groups of tile threads take interleaved
// K entries of a chunk of KC = KG * floor(kKC / KG) entries (equal shares).
// Staging tiles are [kKC][Np] complex with Np = 4 NT + 1 (the odd row length
// spreads the transposed 16-byte writes over the banks).
struct Geo {
  int N, NT, Np, ntiles, KG, KC;
  size_t stage_bytes, red_bytes, smem;
};

inline Geo geometry(int N) {
  Geo g;
  g.N = N;
  g.NT = (N + 3) / 4;
  g.Np = 4 * g.NT + 1;
  g.ntiles = g.NT * (g.NT + 1) / 2;
  g.KG = std::max(1, std::min(kMaxKG, kThreads / g.ntiles));
  g.KC = g.KG * std::max(1, kKC / g.KG);
  g.stage_bytes = sizeof(double2) * kStages * kKC * (size_t)g.Np;
  g.red_bytes = sizeof(double2) * 16 * (size_t)g.KG * g.ntiles;
  g.smem = std::max(g.stage_bytes, g.red_bytes);
  return g;
}

struct Params {
  double2* basis;              // [Vc][N][K]
  double2* gram;               // [Vc][N (N + 1) / 2]: G[i][j], j <= i
  double2* lfac;               // [Vc][N (N + 1) / 2]: conj(L[i][j]) for j < i, (1 / L[i][i], 0) for j = i
  int* need;                   // [Vc]: 1 once a block needed the shifted factorisation
  int* status;                 // 1 when a shifted factorisation failed too
  unsigned long long* maxerr;  // check mode: max |G - 1| (as the bits of a non-negative double)
  int Vc, N, K, NT, Np, ntiles, KG, KC;
  int pass, passes;
};

__device__ __forceinline__ bool block_active(const Params& P, int c) { return P.pass < P.passes || P.need[c] != 0; }

// Gram matrices of the blocks (packed lower triangles into P.gram), or in
// CHECK mode the largest |G - 1| over all blocks into P.maxerr.
template <bool CHECK>
__global__ void __launch_bounds__(kThreads, 2) gram_kernel(Params P) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double2* stage = reinterpret_cast<double2*>(smem_raw);  // [kStages][kKC][Np], then the partial tiles
  const int t = threadIdx.x;
  const int NT = P.NT, Np = P.Np, N = P.N, K = P.K, KC = P.KC, KG = P.KG;
  const int tile = t % P.ntiles, grp = t / P.ntiles;
  const bool active = grp < KG;
  int ti = 0;
  while ((ti + 1) * (ti + 2) / 2 <= tile) ++ti;
  const int tj = tile - ti * (ti + 1) / 2;
  const int nch = (K + KC - 1) / KC;
  double mx = 0.0;
  for (int c = blockIdx.x; c < P.Vc; c += gridDim.x) {
    if (!CHECK && !block_active(P, c)) continue;  // uniform over the CTA
    const double2* Vb = P.basis + (int64_t)c * N * K;
    auto issue = [&](int ch) {
      if (ch < nch) {
        double2* buf = stage + (ch % kStages) * kKC * Np;
        const int k0 = ch * KC;
        const int kc = min(KC, K - k0);
        for (int e = t; e < N * KC; e += kThreads) {
          const int i = e / KC, kk = e - i * KC;
          if (kk < kc) cp_async16(buf + kk * Np + i, Vb + (int64_t)i * K + k0 + kk);
        }
      }
      cp_async_commit();  // an empty group past the last chunk keeps the group count uniform
    };
    double2 acc[4][4];
#pragma unroll
    for (int q = 0; q < 4; ++q)
#pragma unroll
      for (int r = 0; r < 4; ++r) acc[q][r] = make_double2(0.0, 0.0);
    __syncthreads();  // the previous block's reduction no longer reads `stage`
#pragma unroll
    for (int sidx = 0; sidx < kStages - 1; ++sidx) issue(sidx);
    for (int ch = 0; ch < nch; ++ch) {
      cp_async_wait<kStages - 2>();  // this thread's copies of chunk ch have landed
      __syncthreads();               // everyone's have; chunk ch - 1 is no longer read
      issue(ch + kStages - 1);       // into the buffer chunk ch - 1 used
      if (active) {
        const double2* buf = stage + (ch % kStages) * kKC * Np;
        const int kc = min(KC, K - ch * KC);
#pragma unroll 2
        for (int kk = grp; kk < kc; kk += KG) {
          double2 a[4], b[4];
#pragma unroll
          for (int q = 0; q < 4; ++q) a[q] = buf[kk * Np + ti + NT * q];
#pragma unroll
          for (int r = 0; r < 4; ++r) b[r] = buf[kk * Np + tj + NT * r];
          // conj(a) b in two sweeps over the 16 accumulators, so that the two
          // dependent FMAs of each component are 32 instructions apart
#pragma unroll
          for (int q = 0; q < 4; ++q)
#pragma unroll
            for (int r = 0; r < 4; ++r) {
              acc[q][r].x = fma(a[q].x, b[r].x, acc[q][r].x);
              acc[q][r].y = fma(a[q].x, b[r].y, acc[q][r].y);
            }
#pragma unroll
          for (int q = 0; q < 4; ++q)
#pragma unroll
            for (int r = 0; r < 4; ++r) {
              acc[q][r].x = fma(a[q].y, b[r].y, acc[q][r].x);
              acc[q][r].y = fma(-a[q].y, b[r].x, acc[q][r].y);
            }
        }
      }
    }
    cp_async_wait<0>();
    __syncthreads();  // all chunks consumed: `stage` takes the partial tiles
    if (active) {
      double2* red = stage + ((size_t)grp * P.ntiles + tile) * 16;
#pragma unroll
      for (int q = 0; q < 4; ++q)
#pragma unroll
        for (int r = 0; r < 4; ++r) red[q * 4 + r] = acc[q][r];
    }
    __syncthreads();
    double2* Gc = P.gram + (int64_t)c * (N * (N + 1) / 2);
    for (int e = t; e < N * N; e += kThreads) {
      const int i = e / N, j = e - (e / N) * N;
      if (j > i) continue;
      const int qi = i / NT, ti2 = i - qi * NT, rj = j / NT, tj2 = j - rj * NT;
      double2 sum = make_double2(0.0, 0.0);
      if (ti2 >= tj2) {
        const double2* src = stage + (size_t)(ti2 * (ti2 + 1) / 2 + tj2) * 16 + qi * 4 + rj;
        for (int g = 0; g < KG; ++g) {
          const double2 v = src[(size_t)g * P.ntiles * 16];
          sum.x += v.x;
          sum.y += v.y;
        }
      } else {  // the conjugate of entry (j, i), held by tile (tj2, ti2)
        const double2* src = stage + (size_t)(tj2 * (tj2 + 1) / 2 + ti2) * 16 + rj * 4 + qi;
        for (int g = 0; g < KG; ++g) {
          const double2 v = src[(size_t)g * P.ntiles * 16];
          sum.x += v.x;
          sum.y -= v.y;
        }
      }
      if (CHECK) {
        const double re = sum.x - (i == j ? 1.0 : 0.0);
        mx = fmax(mx, sqrt(re * re + sum.y * sum.y));
      } else {
        Gc[i * (i + 1) / 2 + j] = sum;
      }
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

// W = conj(L)^{-1} V for every column of every block: thread per column, the
// column in registers (NMAX entries, rows >= N unused), conj(L) in shared
// memory; the CTA walks the blocks of its grid stride and every 256-column
// chunk of each, with the next chunk's columns copied into shared memory while
// the current chunk is solved.
template <int NMAX>
__global__ void __launch_bounds__(kSolveThreads) tri_solve_kernel(Params P) {
  constexpr int NTS = kSolveThreads;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double2* pre = reinterpret_cast<double2*>(smem_raw);  // [NMAX][NTS]: the prefetched columns
  double2* L = pre + NMAX * NTS;                        // packed conj(L) of the current block
  const int N = P.N, K = P.K, t = threadIdx.x;
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
#pragma unroll
      for (int i = 0; i < NMAX; ++i) {
        if (i < N) {
          // four partial sums (j mod 4) shorten the dependent chains
          const double2* Li = L + i * (i + 1) / 2;
          double2 sp[4] = {w[i], make_double2(0.0, 0.0), make_double2(0.0, 0.0), make_double2(0.0, 0.0)};
#pragma unroll
          for (int j = 0; j < i; ++j) {  // s -= conj(L[i][j]) w[j]
            const double2 a = Li[j];
            double2& s = sp[j & 3];
            s.x = fma(-a.x, w[j].x, s.x);
            s.x = fma(a.y, w[j].y, s.x);
            s.y = fma(-a.x, w[j].y, s.y);
            s.y = fma(-a.y, w[j].x, s.y);
          }
          const double inv = Li[i].x;
          w[i] = make_double2(((sp[0].x + sp[1].x) + (sp[2].x + sp[3].x)) * inv,
                              ((sp[0].y + sp[1].y) + (sp[2].y + sp[3].y)) * inv);
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
  P->NT = g.NT;
  P->Np = g.Np;
  P->ntiles = g.ntiles;
  P->KG = g.KG;
  P->KC = g.KC;
  P->pass = 0;
  P->passes = 1;
  return GMG_OK;
}

template <bool CHECK>
static gmg_status launch_gram(const Params& P, cudaStream_t s) {
  const Geo g = geometry(P.N);
  GMG_CHECK(g.smem <= 227 * 1024, GMG_ERR_UNSUPPORTED, "orthonormalise: tile does not fit shared memory");
  GMG_CUDA(cudaFuncSetAttribute(gram_kernel<CHECK>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)g.smem));
  int per_sm = 1;
  GMG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, gram_kernel<CHECK>, kThreads, g.smem));
  const int grid = std::min(P.Vc, num_sms() * std::max(per_sm, 1));
  gram_kernel<CHECK><<<grid, kThreads, g.smem, s>>>(P);
  GMG_CUDA(cudaGetLastError());
  return GMG_OK;
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
  GMG_CUDA(cudaFuncSetAttribute(tri_solve_kernel<NMAX>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int per_sm = 1;
  GMG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, tri_solve_kernel<NMAX>, kSolveThreads, smem));
  const int grid = std::min(P.Vc, num_sms() * std::max(per_sm, 1));
  tri_solve_kernel<NMAX><<<grid, kSolveThreads, smem, s>>>(P);
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
  GMG_TRY(launch_gram<true>(P, s));
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

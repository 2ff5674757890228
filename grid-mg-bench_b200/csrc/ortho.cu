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
// Two kernels per pass:
//   gram_chol_kernel   CTA per block (persistent over blocks): the Gram matrix
//                      from FP64 register tiles over the lower block triangle,
//                      fed by a cp.async double buffer of K-chunks, then the
//                      Cholesky factor in shared memory; writes conj(L) and
//                      1 / diag(L) packed (row i: i + 1 entries) per block.
//   tri_solve_kernel   thread per column of V_c: the N entries of the column in
//                      registers, forward substitution against conj(L) held in
//                      shared memory (every thread reads the same entry: a
//                      broadcast), the column written back in place.
// Traffic per pass: the basis read twice and written once (3 x 8 B x 2 x N x K
// per block); flops 8 K N (N + 1) / 2 for the Gram matrix (lower triangle) and
// the same for the substitution.
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
constexpr int kKC = 64;        // K values per staged chunk
constexpr int kMaxKG = 16;     // K-interleaved groups of tile threads
constexpr int kSolveMax = 40;  // largest nbasis of the two-kernel path

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
// K entries of a chunk.  Staging tiles are [kKC][Np] complex with Np = 4 NT + 1
// (the odd row length spreads the transposed 16-byte writes over the banks).
struct Geo {
  int N, NT, Np, ntiles, KG;
  size_t stage_bytes, red_bytes, g_bytes, smem;
};

inline Geo geometry(int N) {
  Geo g;
  g.N = N;
  g.NT = (N + 3) / 4;
  g.Np = 4 * g.NT + 1;
  g.ntiles = g.NT * (g.NT + 1) / 2;
  g.KG = std::max(1, std::min(kMaxKG, kThreads / g.ntiles));
  g.stage_bytes = sizeof(double2) * 2 * kKC * (size_t)g.Np;
  g.red_bytes = sizeof(double2) * 16 * (size_t)g.KG * g.ntiles;
  g.g_bytes = sizeof(double2) * (size_t)N * N + sizeof(double) * N;
  g.smem = std::max(g.stage_bytes, g.red_bytes) + g.g_bytes;
  return g;
}

struct Params {
  double2* basis;          // [Vc][N][K]
  double2* lfac;           // [Vc][N (N + 1) / 2]: conj(L[i][j]) for j < i, (1 / L[i][i], 0) for j = i
  int* need;               // [Vc]: 1 once a block needed the shifted factorisation
  int* status;             // 1 when a shifted factorisation failed too
  unsigned long long* maxerr;  // check mode: max |G - 1| (as the bits of a non-negative double)
  int Vc, N, K, NT, Np, ntiles, KG;
  int pass, passes;
};

// Gram matrix of block c into G (lower triangle, row-major N x N).  All threads
// call it; `stage` holds two chunk buffers, then the per-group partial tiles.
__device__ void block_gram(const Params& P, const double2* __restrict__ Vb, double2* stage, double2* G) {
  const int t = threadIdx.x;
  const int NT = P.NT, Np = P.Np, N = P.N, K = P.K;
  const int tile = t % P.ntiles, grp = t / P.ntiles;
  const bool active = grp < P.KG;
  int ti = 0;
  while ((ti + 1) * (ti + 2) / 2 <= tile) ++ti;
  const int tj = tile - ti * (ti + 1) / 2;
  double2 acc[4][4];
#pragma unroll
  for (int q = 0; q < 4; ++q)
#pragma unroll
    for (int r = 0; r < 4; ++r) acc[q][r] = make_double2(0.0, 0.0);
  const int nch = (K + kKC - 1) / kKC;
  auto issue = [&](int ch) {
    double2* buf = stage + (ch & 1) * kKC * Np;
    const int k0 = ch * kKC;
    const int kc = min(kKC, K - k0);
    for (int e = t; e < N * kKC; e += kThreads) {
      const int i = e / kKC, kk = e % kKC;
      if (kk < kc) cp_async16(buf + kk * Np + i, Vb + (int64_t)i * K + k0 + kk);
    }
    cp_async_commit();
  };
  __syncthreads();  // the previous user of `stage` (reduction or solve) is done
  issue(0);
  for (int ch = 0; ch < nch; ++ch) {
    if (ch + 1 < nch) {
      issue(ch + 1);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    if (active) {
      const double2* buf = stage + (ch & 1) * kKC * Np;
      const int kc = min(kKC, K - ch * kKC);
#pragma unroll 2
      for (int kk = grp; kk < kc; kk += P.KG) {
        double2 a[4], b[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) a[q] = buf[kk * Np + ti + NT * q];
#pragma unroll
        for (int r = 0; r < 4; ++r) b[r] = buf[kk * Np + tj + NT * r];
#pragma unroll
        for (int q = 0; q < 4; ++q)
#pragma unroll
          for (int r = 0; r < 4; ++r) acc[q][r] = cfma_conj(acc[q][r], a[q], b[r]);
      }
    }
    __syncthreads();  // buffer (ch & 1) is refilled by the issue of chunk ch + 2
  }
  // partial tiles of every group, then the sum over groups per lower entry
  if (active) {
    double2* red = stage + ((size_t)grp * P.ntiles + tile) * 16;
#pragma unroll
    for (int q = 0; q < 4; ++q)
#pragma unroll
      for (int r = 0; r < 4; ++r) red[q * 4 + r] = acc[q][r];
  }
  __syncthreads();
  for (int e = t; e < N * N; e += kThreads) {
    const int i = e / N, j = e % N;
    if (j > i) continue;
    const int qi = i / NT, ti2 = i % NT, rj = j / NT, tj2 = j % NT;
    double2 s = make_double2(0.0, 0.0);
    if (ti2 >= tj2) {
      const double2* src = stage + (size_t)(ti2 * (ti2 + 1) / 2 + tj2) * 16 + qi * 4 + rj;
      for (int g = 0; g < P.KG; ++g) {
        const double2 v = src[(size_t)g * P.ntiles * 16];
        s.x += v.x;
        s.y += v.y;
      }
    } else {  // the conjugate of entry (j, i), held by tile (tj2, ti2)
      const double2* src = stage + (size_t)(tj2 * (tj2 + 1) / 2 + ti2) * 16 + rj * 4 + qi;
      for (int g = 0; g < P.KG; ++g) {
        const double2 v = src[(size_t)g * P.ntiles * 16];
        s.x += v.x;
        s.y -= v.y;
      }
    }
    G[i * N + j] = s;
  }
  __syncthreads();
}

// Cholesky G + shift I = L L^dag in place (strict lower triangle of G; the
// diagonal goes to diag[]).  Returns false to every thread when a pivot is not
// positive (that pivot is replaced by 1 so that the factor stays finite).
__device__ bool block_cholesky(double2* G, double* diag, int N, double shift, int* fail_s) {
  const int t = threadIdx.x;
  if (t == 0) *fail_s = 0;
  __syncthreads();
  for (int j = 0; j < N; ++j) {
    // column j: every thread takes the pivot from G[j][j] (final after step j - 1)
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
    // trailing update G[i][k] -= L[i][j] conj(L[k][j]), j < k <= i
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

template <bool CHECK>
__global__ void __launch_bounds__(kThreads, 2) gram_chol_kernel(Params P) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int N = P.N;
  const size_t st_a = (size_t)2 * kKC * P.Np, st_b = (size_t)16 * P.KG * P.ntiles;
  const size_t stage_elems = st_a > st_b ? st_a : st_b;  // double2 units
  double2* stage = reinterpret_cast<double2*>(smem_raw);
  double2* G = stage + stage_elems;
  double* diag = reinterpret_cast<double*>(G + (size_t)N * N);
  __shared__ int fail_s;
  __shared__ double trace_s;
  const int t = threadIdx.x;
  for (int c = blockIdx.x; c < P.Vc; c += gridDim.x) {
    if (!CHECK && P.pass >= P.passes && P.need[c] == 0) continue;  // extra passes: broken-down blocks only
    const double2* Vb = P.basis + (int64_t)c * N * P.K;
    block_gram(P, Vb, stage, G);
    if (CHECK) {
      double m = 0.0;
      for (int e = t; e < N * N; e += kThreads) {
        const int i = e / N, j = e % N;
        if (j > i) continue;
        const double re = G[e].x - (i == j ? 1.0 : 0.0), im = G[e].y;
        m = fmax(m, sqrt(re * re + im * im));
      }
      atomicMax(P.maxerr, (unsigned long long)__double_as_longlong(m));  // non-negative doubles order as integers
      continue;
    }
    bool ok = block_cholesky(G, diag, N, 0.0, &fail_s);
    if (!ok) {
      // shifted Cholesky QR on the same Gram matrix (formed again: the failed
      // factorisation overwrote it), then two extra plain passes for this block
      block_gram(P, Vb, stage, G);
      if (t == 0) {
        double tr = 0.0;
        for (int i = 0; i < N; ++i) tr += G[i * N + i].x;
        trace_s = tr;
      }
      __syncthreads();
      const double shift = 11.0 * ((double)P.K * N + (double)N * (N + 1)) * 1.1102230246251565e-16 * trace_s;
      ok = block_cholesky(G, diag, N, shift, &fail_s);
      if (t == 0) {
        P.need[c] = 1;
        if (!ok) atomicExch(P.status, 1);
      }
    }
    // packed conj(L) with the reciprocal diagonal
    double2* Lc = P.lfac + (int64_t)c * (N * (N + 1) / 2);
    for (int e = t; e < N * N; e += kThreads) {
      const int i = e / N, j = e % N;
      if (j > i) continue;
      const double2 v = G[e];
      Lc[i * (i + 1) / 2 + j] = j < i ? make_double2(v.x, -v.y) : make_double2(1.0 / diag[i], 0.0);
    }
    __syncthreads();  // G and diag are rewritten for the next block
  }
}

// W = conj(L)^{-1} V for every column of every block: thread per column, the
// column in registers (NMAX entries, rows >= N unused), conj(L) in shared memory.
template <int NMAX>
__global__ void __launch_bounds__(kThreads) tri_solve_kernel(Params P) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double2* L = reinterpret_cast<double2*>(smem_raw);  // packed, N (N + 1) / 2
  const int N = P.N, K = P.K;
  const int nL = N * (N + 1) / 2;
  const int chunks = (K + kThreads - 1) / kThreads;
  const int64_t items = (int64_t)P.Vc * chunks;
  int prev_c = -1;
  for (int64_t it = blockIdx.x; it < items; it += gridDim.x) {
    const int c = (int)(it / chunks);
    const int k = (int)(it % chunks) * kThreads + threadIdx.x;
    if (P.pass >= P.passes && P.need[c] == 0) continue;  // uniform over the CTA
    if (c != prev_c) {
      __syncthreads();
      const double2* src = P.lfac + (int64_t)c * nL;
      for (int e = threadIdx.x; e < nL; e += kThreads) L[e] = src[e];
      __syncthreads();
      prev_c = c;
    }
    if (k >= K) continue;
    double2* col = P.basis + (int64_t)c * N * K + k;
    double2 w[NMAX];
#pragma unroll
    for (int i = 0; i < NMAX; ++i) w[i] = i < N ? col[(int64_t)i * K] : make_double2(0.0, 0.0);
#pragma unroll
    for (int i = 0; i < NMAX; ++i) {
      if (i < N) {
        const double2* Li = L + i * (i + 1) / 2;
        double2 s = w[i];
#pragma unroll
        for (int j = 0; j < i; ++j) {  // s -= conj(L[i][j]) w[j]
          const double2 a = Li[j];
          s.x = fma(-a.x, w[j].x, s.x);
          s.x = fma(a.y, w[j].y, s.x);
          s.y = fma(-a.x, w[j].y, s.y);
          s.y = fma(-a.y, w[j].x, s.y);
        }
        const double inv = Li[i].x;
        w[i] = make_double2(s.x * inv, s.y * inv);
      }
    }
#pragma unroll
    for (int i = 0; i < NMAX; ++i)
      if (i < N) col[(int64_t)i * K] = w[i];
  }
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

// workspace: [status int + max error][need int Vc][conj(L) Vc x N (N + 1) / 2]
static gmg_status workspace(gmg_agg* h, int** status, unsigned long long** maxerr, int** need, double2** lfac) {
  const int64_t Vc = h->cdims.vol();
  const size_t head = 256, need_b = (size_t)(Vc * sizeof(int) + 255) / 256 * 256;
  const size_t lf_b = sizeof(double2) * (size_t)Vc * (h->N * (h->N + 1) / 2);
  GMG_TRY(h->ortho_ws.alloc(head + need_b + lf_b));
  char* p = h->ortho_ws.as<char>();
  *status = reinterpret_cast<int*>(p);
  *maxerr = reinterpret_cast<unsigned long long*>(p + 8);
  *need = reinterpret_cast<int*>(p + head);
  *lfac = reinterpret_cast<double2*>(p + head + need_b);
  return GMG_OK;
}

static Params params(gmg_agg* h, const Geo& g, int* status, unsigned long long* maxerr, int* need, double2* lfac) {
  Params P;
  P.basis = h->basis_blk.as<double2>();
  P.lfac = lfac;
  P.need = need;
  P.status = status;
  P.maxerr = maxerr;
  P.Vc = (int)h->cdims.vol();
  P.N = h->N;
  P.K = h->bv * h->dof;
  P.NT = g.NT;
  P.Np = g.Np;
  P.ntiles = g.ntiles;
  P.KG = g.KG;
  P.pass = 0;
  P.passes = 1;
  return P;
}

template <int NMAX>
static gmg_status launch_solve(const Params& P, cudaStream_t s) {
  const size_t smem = sizeof(double2) * (size_t)(P.N * (P.N + 1) / 2);
  const int chunks = (P.K + kThreads - 1) / kThreads;
  const int64_t items = (int64_t)P.Vc * chunks;
  int per_sm = 1;
  GMG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, tri_solve_kernel<NMAX>, kThreads, smem));
  const int grid = (int)std::min<int64_t>(items, (int64_t)num_sms() * std::max(per_sm, 1) * 4);
  tri_solve_kernel<NMAX><<<grid, kThreads, smem, s>>>(P);
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
  int *status, *need;
  unsigned long long* maxerr;
  double2* lfac;
  GMG_TRY(workspace(h, &status, &maxerr, &need, &lfac));
  const int Vc = (int)h->cdims.vol();
  GMG_CUDA(cudaMemsetAsync(status, 0, sizeof(int), s));
  if (N > kSolveMax) {
    GMG_CHECK(N <= 64, GMG_ERR_UNSUPPORTED, "orthonormalise: nbasis > 64");
    const size_t smem = sizeof(double2) * ((size_t)2 * N * N + (size_t)kBigKS * h->dof * N) +
                        sizeof(double) * (N + (N & 1));
    GMG_CHECK(smem <= 227 * 1024, GMG_ERR_UNSUPPORTED, "orthonormalise: nbasis x site dof too large");
    GMG_CUDA(cudaFuncSetAttribute(big_ortho_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    KernelTimer kt("ortho", s);
    big_ortho_kernel<<<std::min(Vc, num_sms() * 8), kThreads, smem, s>>>(h->basis_blk.as<double2>(), Vc, N, h->dof,
                                                                        h->bv, passes, status);
    GMG_CUDA(cudaGetLastError());
  } else {
    const Geo g = geometry(N);
    GMG_CHECK(g.smem <= 227 * 1024, GMG_ERR_UNSUPPORTED, "orthonormalise: tile does not fit shared memory");
    GMG_CUDA(cudaFuncSetAttribute(gram_chol_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)g.smem));
    GMG_CUDA(cudaMemsetAsync(need, 0, sizeof(int) * Vc, s));
    Params P = params(h, g, status, maxerr, need, lfac);
    P.passes = passes;
    int per_sm = 1;
    GMG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, gram_chol_kernel<false>, kThreads, g.smem));
    const int grid = std::min(Vc, num_sms() * std::max(per_sm, 1));
    KernelTimer kt("ortho", s);
    // passes + 2 rounds: the last two only touch blocks that needed the shift
    for (int pass = 0; pass < passes + 2; ++pass) {
      P.pass = pass;
      gram_chol_kernel<false><<<grid, kThreads, g.smem, s>>>(P);
      GMG_CUDA(cudaGetLastError());
      GMG_TRY(solve(P, s));
    }
  }
  h->basis_f_ok = false;
  h->basis_tc_ok = false;
  return GMG_OK;
}

gmg_status agg_check_orthogonal(gmg_agg* h, double* max_err, cudaStream_t s) {
  using namespace ortho;
  const int N = h->N;
  int *status, *need;
  unsigned long long* maxerr;
  double2* lfac;
  GMG_TRY(workspace(h, &status, &maxerr, &need, &lfac));
  const Geo g = geometry(N);
  GMG_CHECK(g.smem <= 227 * 1024, GMG_ERR_UNSUPPORTED, "check orthogonal: tile does not fit shared memory");
  GMG_CUDA(cudaFuncSetAttribute(gram_chol_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)g.smem));
  GMG_CUDA(cudaMemsetAsync(maxerr, 0, sizeof(unsigned long long), s));
  const int Vc = (int)h->cdims.vol();
  Params P = params(h, g, status, maxerr, need, lfac);
  int per_sm = 1;
  GMG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, gram_chol_kernel<true>, kThreads, g.smem));
  gram_chol_kernel<true><<<std::min(Vc, num_sms() * std::max(per_sm, 1)), kThreads, g.smem, s>>>(P);
  GMG_CUDA(cudaGetLastError());
  unsigned long long v = 0;
  int st = 0;
  GMG_CUDA(cudaMemcpyAsync(&v, maxerr, sizeof(v), cudaMemcpyDeviceToHost, s));
  GMG_CUDA(cudaMemcpyAsync(&st, status, sizeof(int), cudaMemcpyDeviceToHost, s));
  GMG_CUDA(cudaStreamSynchronize(s));
  double r;
  memcpy(&r, &v, sizeof(r));
  *max_err = r;
  if (st) return fail(GMG_ERR_NONFINITE, "orthonormalise: a block Gram matrix was singular even with the shift");
  return GMG_OK;
}

}  // namespace gmg

// coarse_stencil.cu -- 9-point coarse Dirac stencil on CUDA cores (FP64 / FP32).
//
// Restates CoarsenedMatrix::M / Mdag / MdirCalc / Mdiag
// (include/CoarsenedMatrixUpstream.h:546-742) and the multi-RHS form
// (include/CoarsenedMatrixUpstreamImprovedDirsaveLutMRHS.h:736-947):
//
//   out(x, r) = sum_{p in [p0,p1)} A_p(x) in(nbr_p(x), r)        (N x N times N)
//
// with Mdag = G5C M G5C (sign flip of the upper half of the basis index on
// load and store, no temporary).  The reference runs one thread per (site,
// row) and re-reads every link element once per RHS; here one CTA owns a
// site, stages A_p(x) and the neighbour's R x N tile in shared memory
// (transposed so that the basis index is the contiguous one), and every
// thread accumulates a TR x TB register tile of (rhs, row) outputs, so a link
// element is read from HBM once for all R right-hand sides.
//
// Links are kept site-major, [V][9][N][N], so that one site's 9 matrices are
// one contiguous stream.
#include <algorithm>

#include "gmg_internal.cuh"

namespace gmg {

template <class T> struct cplx_t;
template <> struct cplx_t<double> { typedef double2 type; };
template <> struct cplx_t<float> { typedef float2 type; };

template <class C> __device__ __forceinline__ C cmul_add(C acc, C a, C b) {
  acc.x = fma(a.x, b.x, acc.x);
  acc.x = fma(-a.y, b.y, acc.x);
  acc.y = fma(a.x, b.y, acc.y);
  acc.y = fma(a.y, b.x, acc.y);
  return acc;
}

// ---------------------------------------------------------------------------
// layout conversion [p][V][N][N] (exchange) -> [V][p][N][N] (site-major)
// ---------------------------------------------------------------------------
template <class To>
__global__ void links_site_major_kernel(const double2* __restrict__ src, To* __restrict__ dst,
                                        int64_t V, int NN) {
  const int64_t total = 9 * V * NN;
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < total;
       k += (int64_t)gridDim.x * blockDim.x) {
    const int64_t e = k % NN;
    const int64_t ps = k / NN;
    const int64_t s = ps % V;
    const int64_t p = ps / V;
    const double2 v = src[k];
    To o;
    o.x = v.x;
    o.y = v.y;
    dst[(s * 9 + p) * NN + e] = o;
  }
}

static int grid_for(int64_t n, int threads) {
  int64_t b = (n + threads - 1) / threads;
  return (int)std::min<int64_t>(std::max<int64_t>(b, 1), 148 * 32);
}

gmg_status coarse_links_to_site_major(gmg_coarse* h, cudaStream_t s) {
  const int64_t V = h->dims.vol();
  const int NN = h->N * h->N;
  GMG_TRY(h->links_d.alloc(sizeof(double2) * 9 * V * NN));
  links_site_major_kernel<double2><<<grid_for(9 * V * NN, 256), 256, 0, s>>>(
      h->links_ref.as<double2>(), h->links_d.as<double2>(), V, NN);
  GMG_CUDA(cudaGetLastError());
  return GMG_OK;
}

gmg_status coarse_prepare_f32(gmg_coarse* h, cudaStream_t s) {
  const int64_t V = h->dims.vol();
  const int NN = h->N * h->N;
  GMG_TRY(h->links_f.alloc(sizeof(float2) * 9 * V * NN));
  links_site_major_kernel<float2><<<grid_for(9 * V * NN, 256), 256, 0, s>>>(
      h->links_ref.as<double2>(), h->links_f.as<float2>(), V, NN);
  GMG_CUDA(cudaGetLastError());
  h->links_f_ok = true;
  return GMG_OK;
}

// ---------------------------------------------------------------------------
// the stencil kernel
// ---------------------------------------------------------------------------
// Link source and site geometry of one apply.  Output index o (V of them: all
// sites, or the sites of one parity) takes its links from link site
// site_map[o] (identity when null): matrix (p - pbase) of the link_pts matrices
// stored per site; its neighbour for point p is input index nbr[p][o] (o
// itself when nbr is null).  dag applies the conjugate transpose of each matrix.
struct LinkSel {
  const void* links;
  int link_pts, pbase;
  const int32_t* site_map;
  const int32_t* nbr;
  int dag;
};

template <class C> __device__ __forceinline__ C cconj(C a) {
  a.y = -a.y;
  return a;
}

template <class T, int TR, int TB>
__global__ void __launch_bounds__(256) coarse_simt_kernel(
    const typename cplx_t<T>::type* __restrict__ links, int link_pts, int pbase, const int32_t* __restrict__ site_map,
    const int32_t* __restrict__ nbr, int dag,
    const typename cplx_t<T>::type* __restrict__ in, typename cplx_t<T>::type* __restrict__ out,
    int V, int N, int nrhs, const int32_t* __restrict__ active, int R, int p0, int p1, int g5) {
  typedef typename cplx_t<T>::type C;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* AT = reinterpret_cast<C*>(smem_raw);  // [N][N]   AT[bb][b] = A[b][bb]
  C* XT = AT + N * N;                      // [N][R]   XT[bb][r] = in(nbr, r)[bb]
  const int NBT = (N + TB - 1) / TB;
  const int NRT = (R + TR - 1) / TR;
  const int ntiles = NBT * NRT;
  const int t = threadIdx.x;
  const int bt = t % NBT, rt = t / NBT;
  const int half = N / 2;

  for (int site = blockIdx.x; site < V; site += gridDim.x) {
    const int64_t lsite = site_map ? site_map[site] : site;
    C acc[TR][TB];
#pragma unroll
    for (int j = 0; j < TR; ++j)
#pragma unroll
      for (int i = 0; i < TB; ++i) acc[j][i] = C{0, 0};

    for (int p = p0; p < p1; ++p) {
      const C* Ap = links + (lsite * link_pts + (p - pbase)) * N * N;
      const int nb = nbr ? nbr[(int64_t)p * V + site] : site;
      __syncthreads();
      if (dag) {  // AT[bb][b] = (A^dag)[b][bb] = conj(A[bb][b])
        for (int k = t; k < N * N; k += blockDim.x) AT[k] = cconj(Ap[k]);
      } else {
        for (int k = t; k < N * N; k += blockDim.x) {
          const int b = k / N, bb = k % N;
          AT[bb * N + b] = Ap[k];
        }
      }
      for (int k = t; k < R * N; k += blockDim.x) {
        const int r = k / N, bb = k % N;
        const int slot = active ? active[r] : r;
        C v = in[((int64_t)nb * nrhs + slot) * N + bb];
        if (g5 && bb >= half) { v.x = -v.x; v.y = -v.y; }
        XT[bb * R + r] = v;
      }
      __syncthreads();
      if (t < ntiles) {
        for (int bb = 0; bb < N; ++bb) {
          C a[TB], x[TR];
#pragma unroll
          for (int i = 0; i < TB; ++i) {
            const int b = bt * TB + i;
            a[i] = b < N ? AT[bb * N + b] : C{0, 0};
          }
#pragma unroll
          for (int j = 0; j < TR; ++j) {
            const int r = rt * TR + j;
            x[j] = r < R ? XT[bb * R + r] : C{0, 0};
          }
#pragma unroll
          for (int j = 0; j < TR; ++j)
#pragma unroll
            for (int i = 0; i < TB; ++i) acc[j][i] = cmul_add(acc[j][i], a[i], x[j]);
        }
      }
    }
    if (t < ntiles) {
#pragma unroll
      for (int j = 0; j < TR; ++j) {
        const int r = rt * TR + j;
        if (r >= R) continue;
        const int slot = active ? active[r] : r;
        C* o = out + ((int64_t)site * nrhs + slot) * N;
#pragma unroll
        for (int i = 0; i < TB; ++i) {
          const int b = bt * TB + i;
          if (b >= N) continue;
          C v = acc[j][i];
          if (g5 && b >= half) { v.x = -v.x; v.y = -v.y; }
          o[b] = v;
        }
      }
    }
  }
}

// ---------------------------------------------------------------------------
// The multi-RHS stencil on the CUDA cores, pipelined: a CTA walks the (site,
// point) items of its sites; while it multiplies item k, the link matrix and
// the neighbour's R vectors of item k + 1 are copied into the other half of
// its shared memory with cp.async.  A thread owns a TR x TB tile of the R x N
// output, its rows and columns interleaved (r = rt + (R / TR) j, b = bt + (N /
// TB) i), so that the lanes of a warp read consecutive rows of the padded
// shared-memory tiles (row stride N + 1 complex numbers: no bank conflicts).
// Needs TB | N and TR | R.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void cp_async_c(void* dst, const double2* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 16;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)), "l"(src)
               : "memory");
}
__device__ __forceinline__ void cp_async_c(void* dst, const float2* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)), "l"(src)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// acc[j][i] += (or -= with NEG) a_i x_j over bb in [bb0, bb1), a_i = A[b_i][bb]
// (DAG: conj(A[bb][b_i])), x_j = X[r_j][bb]; the signs are folded into the FMAs
template <bool DAG, bool NEG, int TR, int TB, class C>
__device__ __forceinline__ void pipe_mac(C (&acc)[TR][TB], const C* __restrict__ A, const C* __restrict__ X, int bb0,
                                         int bb1, int NP, int bt, int NBT, int rt, int NRT) {
  for (int bb = bb0; bb < bb1; ++bb) {
    C a[TB], x[TR];
#pragma unroll
    for (int i = 0; i < TB; ++i) a[i] = DAG ? A[bb * NP + bt + NBT * i] : A[(bt + NBT * i) * NP + bb];
#pragma unroll
    for (int j = 0; j < TR; ++j) x[j] = X[(rt + NRT * j) * NP + bb];
#pragma unroll
    for (int j = 0; j < TR; ++j)
#pragma unroll
      for (int i = 0; i < TB; ++i) {
        // (ar + i s ai)(xr + i xi) with s = -1 for the conjugate, the product negated with NEG
        const auto ar = NEG ? -a[i].x : a[i].x;
        const auto ai = (NEG != DAG) ? -a[i].y : a[i].y;
        acc[j][i].x = fma(ar, x[j].x, acc[j][i].x);
        acc[j][i].x = fma(-ai, x[j].y, acc[j][i].x);
        acc[j][i].y = fma(ar, x[j].y, acc[j][i].y);
        acc[j][i].y = fma(ai, x[j].x, acc[j][i].y);
      }
  }
}

template <class T, int TR, int TB, int NC>  // NC: N as a compile-time constant (0: runtime)
__global__ void __launch_bounds__(256) coarse_simt_pipe_kernel(
    const typename cplx_t<T>::type* __restrict__ links, int link_pts, int pbase, const int32_t* __restrict__ site_map,
    const int32_t* __restrict__ nbr, int dag, const typename cplx_t<T>::type* __restrict__ in,
    typename cplx_t<T>::type* __restrict__ out, int V, int N_, int nrhs, const int32_t* __restrict__ active, int R,
    int p0, int p1, int g5) {
  typedef typename cplx_t<T>::type C;
  const int N = NC ? NC : N_;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int NP = N + 1;                     // padded row stride
  const int stage = (N + R) * NP;           // complex numbers per stage: A [N][NP], X [R][NP]
  C* S = reinterpret_cast<C*>(smem_raw);
  const int t = threadIdx.x, nthr = blockDim.x;
  const int NBT = N / TB, NRT = R / TR;
  const int bt = t % NBT, rt = t / NBT;
  const bool comp = t < NBT * NRT;
  const int half = N / 2;
  const int npts = p1 - p0;
  const int nsites = (V - (int)blockIdx.x + (int)gridDim.x - 1) / (int)gridDim.x;
  const int nitems = nsites * npts;

  // copies of item k (site blockIdx.x + (k / npts) gridDim.x, point p0 + k % npts) into stage k & 1
  auto issue = [&](int k) {
    const int site = blockIdx.x + (k / npts) * gridDim.x;
    const int p = p0 + k % npts;
    const int64_t lsite = site_map ? site_map[site] : site;
    const C* Ap = links + (lsite * link_pts + (p - pbase)) * (int64_t)N * N;
    const int nb = nbr ? nbr[(int64_t)p * V + site] : site;
    C* A = S + (k & 1) * stage;
    C* X = A + N * NP;
    for (int e = t; e < N * N; e += nthr) cp_async_c(A + (e / N) * NP + e % N, Ap + e);
    const C* xs = in + (int64_t)nb * nrhs * N;
    for (int e = t; e < R * N; e += nthr) {
      const int r = e / N, bb = e - r * N;
      const int slot = active ? active[r] : r;
      cp_async_c(X + r * NP + bb, xs + slot * N + bb);
    }
    cp_async_commit();
  };

  C acc[TR][TB];
  if (nitems > 0) issue(0);
  for (int k = 0; k < nitems; ++k) {
    if (k + 1 < nitems) {
      issue(k + 1);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    const int kp = k % npts;
    if (kp == 0) {
#pragma unroll
      for (int j = 0; j < TR; ++j)
#pragma unroll
        for (int i = 0; i < TB; ++i) acc[j][i] = C{0, 0};
    }
    if (comp) {
      const C* A = S + (k & 1) * stage;
      const C* X = A + N * NP;
      // the dagger and the input G5C (the sign of components bb >= N / 2) are
      // uniform per launch and per half of bb: four loop forms, no per-element
      // selects or sign multiplies
      if (!dag) {
        pipe_mac<false, false, TR, TB>(acc, A, X, 0, half, NP, bt, NBT, rt, NRT);
        if (g5) pipe_mac<false, true, TR, TB>(acc, A, X, half, N, NP, bt, NBT, rt, NRT);
        else pipe_mac<false, false, TR, TB>(acc, A, X, half, N, NP, bt, NBT, rt, NRT);
      } else {
        pipe_mac<true, false, TR, TB>(acc, A, X, 0, half, NP, bt, NBT, rt, NRT);
        if (g5) pipe_mac<true, true, TR, TB>(acc, A, X, half, N, NP, bt, NBT, rt, NRT);
        else pipe_mac<true, false, TR, TB>(acc, A, X, half, N, NP, bt, NBT, rt, NRT);
      }
      if (kp == npts - 1) {
        const int site = blockIdx.x + (k / npts) * gridDim.x;
#pragma unroll
        for (int j = 0; j < TR; ++j) {
          const int r = rt + NRT * j;
          const int slot = active ? active[r] : r;
          C* o = out + ((int64_t)site * nrhs + slot) * N;
#pragma unroll
          for (int i = 0; i < TB; ++i) {
            const int b = bt + NBT * i;
            C v = acc[j][i];
            if (g5 && b >= half) {
              v.x = -v.x;
              v.y = -v.y;
            }
            o[b] = v;
          }
        }
      }
    }
    __syncthreads();  // stage k & 1 is refilled by the issue of item k + 2
  }
}

template <class T, int TR, int TB>
static bool launch_simt_pipe(const LinkSel& L, const void* in, void* out, int V, int N, int nrhs,
                             const int32_t* active, int R, int p0, int p1, int g5, cudaStream_t s,
                             gmg_status* st) {
  typedef typename cplx_t<T>::type C;
  if (N % TB || R % TR || (N / TB) * (R / TR) > 256 || p1 <= p0) return false;
  const size_t smem = sizeof(C) * 2 * (size_t)(N + R) * (N + 1);
  // at least 3 CTAs per SM: with two (FP64 nbasis 40 x 40 RHS, the coarse-of-
  // coarse construction) the kernel without the pipeline, at 4, was faster
  if (smem > 72 * 1024) return false;
  const int threads = std::max(32, ((N / TB) * (R / TR) + 31) / 32 * 32);
  auto kern = N == 32 ? coarse_simt_pipe_kernel<T, TR, TB, 32>
             : N == 24 ? coarse_simt_pipe_kernel<T, TR, TB, 24>
             : N == 40 ? coarse_simt_pipe_kernel<T, TR, TB, 40>
                       : coarse_simt_pipe_kernel<T, TR, TB, 0>;
  *st = GMG_OK;
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) {
    *st = fail(GMG_ERR_CUDA, "coarse apply: shared-memory attribute");
    return true;
  }
  int dev = 0, nsm = 148, per_sm = 1;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem);
  const int grid = std::min(V, nsm * std::max(per_sm, 1));
  KernelTimer kt("coarse_simt", s);
  kern<<<grid, threads, smem, s>>>(reinterpret_cast<const C*>(L.links), L.link_pts, L.pbase, L.site_map, L.nbr, L.dag,
                                   reinterpret_cast<const C*>(in), reinterpret_cast<C*>(out), V, N, nrhs, active, R,
                                   p0, p1, g5);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) *st = fail(GMG_ERR_CUDA, std::string("coarse apply: ") + cudaGetErrorString(e));
  return true;
}

template <class T, int TR, int TB>
static gmg_status launch_simt(const LinkSel& L, const void* in, void* out,
                              int V, int N, int nrhs, const int32_t* active, int R, int p0, int p1,
                              int g5, cudaStream_t s) {
  typedef typename cplx_t<T>::type C;
  const int ntiles = ((N + TB - 1) / TB) * ((R + TR - 1) / TR);
  GMG_CHECK(ntiles <= 256, GMG_ERR_UNSUPPORTED, "coarse apply: nbasis x nrhs tile too large");
  const int threads = std::max(32, (ntiles + 31) / 32 * 32);
  const size_t smem = sizeof(C) * ((size_t)N * N + (size_t)N * R);
  GMG_CHECK(smem <= 227 * 1024, GMG_ERR_UNSUPPORTED, "coarse apply: shared-memory tile too large");
  auto kern = coarse_simt_kernel<T, TR, TB>;
  GMG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int dev = 0, nsm = 148, per_sm = 1;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem);
  const int grid = std::min(V, nsm * std::max(per_sm, 1) * 4);
  KernelTimer kt("coarse_simt", s);
  kern<<<grid, threads, smem, s>>>(reinterpret_cast<const C*>(L.links), L.link_pts, L.pbase, L.site_map, L.nbr, L.dag,
                                   reinterpret_cast<const C*>(in), reinterpret_cast<C*>(out), V, N,
                                   nrhs, active, R, p0, p1, g5);
  GMG_CUDA(cudaGetLastError());
  return GMG_OK;
}

// ---------------------------------------------------------------------------
// Single right-hand side (CoarsenedMatrixUpstream.h:572-597 with nrhs = 1).
// The work per site is 9 GEMVs of N x N, too little for register tiling, and
// the 4^4 lattices of the coarse levels have only 256 sites.  One CTA per site,
// one thread per (point, row): the neighbour vectors are staged in shared
// memory, each thread forms one row product from a contiguous link row, and
// the 9 partial rows are summed in shared memory.
// ---------------------------------------------------------------------------
template <class T>
__global__ void __launch_bounds__(576) coarse_1rhs_kernel(const typename cplx_t<T>::type* __restrict__ links,
                                                          int link_pts, int pbase,
                                                          const int32_t* __restrict__ site_map,
                                                          const int32_t* __restrict__ nbr, int dag,
                                                          const typename cplx_t<T>::type* __restrict__ in,
                                                          typename cplx_t<T>::type* __restrict__ out, int V, int N,
                                                          int nrhs, int slot, int p0, int p1, int g5) {
  typedef typename cplx_t<T>::type C;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* X = reinterpret_cast<C*>(smem_raw);  // [9][N] neighbour vectors
  C* part = X + 9 * N;                    // [9][N] partial rows
  const int t = threadIdx.x;
  const int p = t / N, b = t % N;  // blockDim = 9 N
  const int half = N / 2;
  for (int site = blockIdx.x; site < V; site += gridDim.x) {
    const int64_t lsite = site_map ? site_map[site] : site;
    if (p >= p0 && p < p1) {
      const int nb = nbr ? nbr[(int64_t)p * V + site] : site;
      C v = in[((int64_t)nb * nrhs + slot) * N + b];
      if (g5 && b >= half) { v.x = -v.x; v.y = -v.y; }
      X[p * N + b] = v;
    }
    __syncthreads();
    C acc{0, 0};
    if (p >= p0 && p < p1) {
      const C* Mp = links + (lsite * link_pts + (p - pbase)) * N * N;
      if (dag) {  // row b of A^dag: conj(A[bb][b])
        for (int bb = 0; bb < N; ++bb) acc = cmul_add(acc, cconj(Mp[(int64_t)bb * N + b]), X[p * N + bb]);
      } else {
        const C* row = Mp + (int64_t)b * N;
        for (int bb = 0; bb < N; ++bb) acc = cmul_add(acc, row[bb], X[p * N + bb]);
      }
    }
    part[p * N + b] = acc;
    __syncthreads();
    if (t < N) {
      C o{0, 0};
      for (int q = p0; q < p1; ++q) {
        o.x += part[q * N + t].x;
        o.y += part[q * N + t].y;
      }
      if (g5 && t >= half) { o.x = -o.x; o.y = -o.y; }
      out[((int64_t)site * nrhs + slot) * N + t] = o;
    }
    __syncthreads();
  }
}

// Single RHS with the site's links staged in shared memory: the CTA first
// copies the (p1 - p0) N x N link matrices of its site with cp.async (every
// 16-byte chunk in flight at once: one memory round trip instead of a
// dependent chain per row), then thread (p, b) forms row b of point p from
// shared memory, starting
// its row at column (b + k) mod N so that the 16-byte reads of a quarter warp
// fall in distinct banks (N a multiple of 8).
template <class T>
__global__ void __launch_bounds__(576) coarse_1rhs_smem_kernel(const typename cplx_t<T>::type* __restrict__ links,
                                                               int link_pts, int pbase,
                                                               const int32_t* __restrict__ site_map,
                                                               const int32_t* __restrict__ nbr, int dag,
                                                               const typename cplx_t<T>::type* __restrict__ in,
                                                               typename cplx_t<T>::type* __restrict__ out, int V,
                                                               int N, int nrhs, int slot, int p0, int p1, int g5) {
  typedef typename cplx_t<T>::type C;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int np = p1 - p0, NN = N * N;
  C* Ls = reinterpret_cast<C*>(smem_raw);  // [np][N][N]
  C* X = Ls + (size_t)np * NN;             // [9][N] neighbour vectors
  C* part = X + 9 * N;                     // [9][N] partial rows
  const int t = threadIdx.x;
  const int p = t / N, b = t % N;  // blockDim = 9 N
  const int half = N / 2;
  for (int site = blockIdx.x; site < V; site += gridDim.x) {
    const int64_t lsite = site_map ? site_map[site] : site;
    // every 16-byte chunk of the site's links in flight at once (cp.async),
    // one wait for all of them
    const unsigned char* src = reinterpret_cast<const unsigned char*>(links + (lsite * link_pts + (p0 - pbase)) * NN);
    const int nchunk = (int)(np * NN * sizeof(C) / 16);
    const uint32_t dst0 = (uint32_t)__cvta_generic_to_shared(Ls);
    for (int e = t; e < nchunk; e += blockDim.x)
      asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst0 + 16u * e), "l"(src + 16 * (size_t)e)
                   : "memory");
    asm volatile("cp.async.commit_group;\n cp.async.wait_group 0;" ::: "memory");
    if (p >= p0 && p < p1) {
      const int nb = nbr ? nbr[(int64_t)p * V + site] : site;
      C v = in[((int64_t)nb * nrhs + slot) * N + b];
      if (g5 && b >= half) { v.x = -v.x; v.y = -v.y; }
      X[p * N + b] = v;
    }
    __syncthreads();
    C acc{0, 0};
    if (p >= p0 && p < p1) {
      const C* Mp = Ls + (size_t)(p - p0) * NN;
      const C* xp = X + p * N;
      int bb = b;
      if (dag) {  // row b of A^dag: conj(A[bb][b])
        for (int k = 0; k < N; ++k) {
          acc = cmul_add(acc, cconj(Mp[bb * N + b]), xp[bb]);
          bb = bb + 1 == N ? 0 : bb + 1;
        }
      } else {
        const C* row = Mp + b * N;
        for (int k = 0; k < N; ++k) {
          acc = cmul_add(acc, row[bb], xp[bb]);
          bb = bb + 1 == N ? 0 : bb + 1;
        }
      }
    }
    part[p * N + b] = acc;
    __syncthreads();
    if (t < N) {
      C o{0, 0};
      for (int q = p0; q < p1; ++q) {
        o.x += part[q * N + t].x;
        o.y += part[q * N + t].y;
      }
      if (g5 && t >= half) { o.x = -o.x; o.y = -o.y; }
      out[((int64_t)site * nrhs + slot) * N + t] = o;
    }
    __syncthreads();
  }
}

template <class T>
static gmg_status launch_1rhs(const LinkSel& L, const void* in, void* out, int V, int N,
                              int nrhs, int slot, int p0, int p1, int g5, cudaStream_t s) {
  typedef typename cplx_t<T>::type C;
  const int threads = 9 * N;
  KernelTimer kt("coarse_simt", s);
  // links staged in shared memory when they fit two CTAs per SM
  const size_t smem_staged = sizeof(C) * ((size_t)(p1 - p0) * N * N + 18 * (size_t)N);
  if (N % 8 == 0 && smem_staged <= 100 * 1024) {
    if (smem_staged > 48 * 1024)
      GMG_CUDA(cudaFuncSetAttribute(coarse_1rhs_smem_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)smem_staged));
    coarse_1rhs_smem_kernel<T><<<V, threads, smem_staged, s>>>(
        reinterpret_cast<const C*>(L.links), L.link_pts, L.pbase, L.site_map, L.nbr, L.dag,
        reinterpret_cast<const C*>(in), reinterpret_cast<C*>(out), V, N, nrhs, slot, p0, p1, g5);
    GMG_CUDA(cudaGetLastError());
    return GMG_OK;
  }
  const size_t smem = sizeof(C) * 18 * (size_t)N;
  coarse_1rhs_kernel<T><<<V, threads, smem, s>>>(reinterpret_cast<const C*>(L.links), L.link_pts, L.pbase, L.site_map,
                                                 L.nbr, L.dag, reinterpret_cast<const C*>(in),
                                                 reinterpret_cast<C*>(out), V, N, nrhs, slot, p0, p1, g5);
  GMG_CUDA(cudaGetLastError());
  return GMG_OK;
}

// `src`: 0 = the stencil links, 1 = the self-link inverse (one matrix per site,
// addressed as point 8).  V / site_map / nbr: the output geometry (full grid
// when site_map is null and nbr is the handle's table).
gmg_status coarse_apply_simt_ex(gmg_coarse* h, int src, int V, const int32_t* site_map, const int32_t* nbr,
                                bool dag, int p0, int p1, bool g5, int compute, int vec_prec, int nrhs,
                                const void* in, void* out, const int32_t* active, int n_active, cudaStream_t s) {
  const int N = h->N;
  const int R = active ? n_active : nrhs;
  if (R == 0) return GMG_OK;
  LinkSel L{nullptr, src == 1 ? 1 : 9, src == 1 ? 8 : 0, site_map, nbr, dag ? 1 : 0};
  if (compute == GMG_F64) {
    GMG_CHECK(vec_prec == GMG_F64, GMG_ERR_UNSUPPORTED, "F64 compute needs F64 vectors");
    L.links = src == 1 ? h->self_inv.p : h->links_d.p;
  } else if (compute == GMG_F32) {
    GMG_CHECK(vec_prec == GMG_F32, GMG_ERR_UNSUPPORTED, "F32 compute needs F32 vectors");
    GMG_CHECK(src == 1 ? h->self_inv_f_ok : h->links_f_ok, GMG_ERR_STATE,
              "F32 links not prepared (gmg_coarse_prepare)");
    L.links = src == 1 ? h->self_inv_f.p : h->links_f.p;
  } else {
    return fail(GMG_ERR_UNSUPPORTED, "coarse apply: unsupported compute precision for SIMT path");
  }
  GMG_CHECK(L.links != nullptr, GMG_ERR_STATE, "coarse apply: link source not built");
  if (R == 1 && !active && N <= 64) {
    if (compute == GMG_F64) return launch_1rhs<double>(L, in, out, V, N, nrhs, 0, p0, p1, g5, s);
    return launch_1rhs<float>(L, in, out, V, N, nrhs, 0, p0, p1, g5, s);
  }
  gmg_status st = GMG_OK;
  if (compute == GMG_F64) {
    if (R >= 4 && launch_simt_pipe<double, 4, 2>(L, in, out, V, N, nrhs, active, R, p0, p1, g5, s, &st)) return st;
    if (R >= 4) return launch_simt<double, 4, 4>(L, in, out, V, N, nrhs, active, R, p0, p1, g5, s);
    return launch_simt<double, 1, 2>(L, in, out, V, N, nrhs, active, R, p0, p1, g5, s);
  }
  if (R >= 4 && launch_simt_pipe<float, 4, 4>(L, in, out, V, N, nrhs, active, R, p0, p1, g5, s, &st)) return st;
  if (R >= 4) return launch_simt<float, 4, 4>(L, in, out, V, N, nrhs, active, R, p0, p1, g5, s);
  return launch_simt<float, 1, 2>(L, in, out, V, N, nrhs, active, R, p0, p1, g5, s);
}

gmg_status coarse_apply_simt(gmg_coarse* h, int p0, int p1, bool g5, int compute, int vec_prec,
                             int nrhs, const void* in, void* out, const int32_t* active,
                             int n_active, cudaStream_t s) {
  return coarse_apply_simt_ex(h, 0, (int)h->dims.vol(), nullptr, h->nbr.as<int32_t>(), false, p0, p1, g5, compute,
                              vec_prec, nrhs, in, out, active, n_active, s);
}

// ---------------------------------------------------------------------------
// ConstructRemainingLinks (...DirsaveLut.h:1164-1196) / ForceHermitian
// (CoarsenedMatrixUpstream.h:956-976) on the exchange layout:
//   A_{dir}(x)[n1][n2] = S(n1,n2) conj(A_{dir+4}(x + e_dir)[n2][n1])
// S = -1 iff n1 and n2 lie in different halves (1 if hermitian).
// ---------------------------------------------------------------------------
__global__ void construct_remaining_kernel(double2* __restrict__ A, const int32_t* __restrict__ nbr,
                                           int V, int N, int hermitian) {
  const int64_t NN = (int64_t)N * N;
  const int64_t total = 4 * (int64_t)V * NN;
  const int half = N / 2;
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < total;
       k += (int64_t)gridDim.x * blockDim.x) {
    const int n2 = (int)(k % N);
    const int n1 = (int)((k / N) % N);
    const int64_t s = (k / NN) % V;
    const int dir = (int)(k / (NN * V));
    const int sp = nbr[(int64_t)dir * V + s];  // x + e_dir
    double2 v = A[((int64_t)(dir + 4) * V + sp) * NN + (int64_t)n2 * N + n1];
    double f = 1.0;
    if (!hermitian && ((n1 / half + n2 / half) & 1)) f = -1.0;
    A[((int64_t)dir * V + s) * NN + (int64_t)n1 * N + n2] = make_double2(f * v.x, -f * v.y);
  }
}

gmg_status coarse_construct_remaining(gmg_coarse* h, cudaStream_t s) {
  const int V = (int)h->dims.vol();
  const int64_t total = 4 * (int64_t)V * h->N * h->N;
  construct_remaining_kernel<<<grid_for(total, 256), 256, 0, s>>>(
      h->links_ref.as<double2>(), h->nbr.as<int32_t>(), V, h->N, h->hermitian);
  GMG_CUDA(cudaGetLastError());
  return GMG_OK;
}

}  // namespace gmg

// ---------------------------------------------------------------------------
// Rework layout map for links (Layout_converters.h:49-56): flat [n1][n2] with
// n = s*Nc_c + c  <->  spin-split [s1][s2][c1][c2].
// ---------------------------------------------------------------------------
namespace gmg {
__global__ void layout_links_kernel(const double2* __restrict__ in, double2* __restrict__ out, int64_t V,
                                    int N, int ncs, int inverse) {
  const int ncc = N / ncs;
  const int64_t NN = (int64_t)N * N;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < V * NN;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t s = e / NN;
    const int n1 = (int)((e % NN) / N), n2 = (int)(e % N);
    const int s1 = n1 / ncc, c1 = n1 % ncc, s2 = n2 / ncc, c2 = n2 % ncc;
    const int64_t spin = s * NN + ((int64_t)(s1 * ncs + s2) * ncc + c1) * ncc + c2;
    if (!inverse) out[spin] = in[e];
    else out[e] = in[spin];
  }
}

// vectors: flat index n = s * Nc_c + c <-> spin form [s][c] (Layout_converters.h:92-139)
__global__ void layout_vectors_kernel(const double2* __restrict__ in, double2* __restrict__ out, int64_t rows,
                                      int N, int ncs, int inverse) {
  const int ncc = N / ncs;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < rows * N;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t row = e / N;
    const int n = (int)(e % N), sp = n / ncc, c = n % ncc;
    const int64_t spin = row * N + (int64_t)sp * ncc + c;  // [row][s][c]: the same order as the flat index
    if (!inverse) out[spin] = in[e];
    else out[e] = in[spin];
  }
}
}  // namespace gmg

extern "C" gmg_status gmg_layout_vectors(int64_t rows, int nbasis, int ncs, const double* in, double* out,
                                         int inverse, gmg_stream s) {
  GMG_CHECK(in && out && in != out, GMG_ERR_ARGUMENT, "gmg_layout_vectors: bad pointers");
  GMG_CHECK(rows > 0 && nbasis > 0 && ncs > 0 && nbasis % ncs == 0, GMG_ERR_ARGUMENT,
            "gmg_layout_vectors: nbasis must be a multiple of the coarse spin count");
  const int64_t n = rows * nbasis;
  gmg::layout_vectors_kernel<<<(int)std::min<int64_t>((n + 255) / 256, 148 * 32), 256, 0, gmg::S(s)>>>(
      reinterpret_cast<const double2*>(in), reinterpret_cast<double2*>(out), rows, nbasis, ncs, inverse);
  GMG_CUDA(cudaGetLastError());
  return GMG_OK;
}

extern "C" gmg_status gmg_layout_links(int64_t V, int nbasis, int ncs, const double* in, double* out,
                                       int inverse, gmg_stream s) {
  GMG_CHECK(in && out && in != out, GMG_ERR_ARGUMENT, "gmg_layout_links: bad pointers");
  GMG_CHECK(V > 0 && nbasis > 0 && ncs > 0 && nbasis % ncs == 0, GMG_ERR_ARGUMENT,
            "gmg_layout_links: nbasis must be a multiple of the coarse spin count");
  const int64_t n = V * nbasis * (int64_t)nbasis;
  gmg::layout_links_kernel<<<(int)std::min<int64_t>((n + 255) / 256, 148 * 32), 256, 0, gmg::S(s)>>>(
      reinterpret_cast<const double2*>(in), reinterpret_cast<double2*>(out), V, nbasis, ncs, inverse);
  GMG_CUDA(cudaGetLastError());
  return GMG_OK;
}

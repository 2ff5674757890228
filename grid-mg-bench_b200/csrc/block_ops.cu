// block_ops.cu -- block projection, promotion and orthonormalisation (CUDA cores).
//
// Restates blockLutedInnerProduct / blockLutedAxpy / blockLutedOrthonormalise
// (include/CoarsenedMatrixUpstreamImprovedDirsaveLut.h:70-240, multi-RHS form
// ...LutMRHS.h:70-236) as per-block complex GEMMs:
//
//   project   C_c (R x N)  = F_c^T (R x K) conj(V_c)^T (K x N)   K = bv * dof
//   promote   F_c (K x R)  = V_c^T (K x N) C_c (N x R)
//
// (the block orthonormalisation is in ortho.cu)
// The basis is kept block-major, basis_blk[c][i][k], k = sb*dof + a with sb the
// lexicographic in-block site index (CoarseningLookupTableRework.h:156-163),
// so one block's N x K panel is contiguous.  Fine fields stay in the caller's
// [site][rhs][dof] layout and are gathered through blk_sites[c][sb].
#include <algorithm>
#include <cmath>

#include "gmg_internal.cuh"

namespace gmg {

template <class T> struct ctype;
template <> struct ctype<double> { typedef double2 t; };
template <> struct ctype<float> { typedef float2 t; };

template <class Cx> __device__ __forceinline__ Cx cfma(Cx acc, Cx a, Cx b) {
  acc.x = fma(a.x, b.x, acc.x);
  acc.x = fma(-a.y, b.y, acc.x);
  acc.y = fma(a.x, b.y, acc.y);
  acc.y = fma(a.y, b.x, acc.y);
  return acc;
}
// acc += conj(a) b
template <class Cx> __device__ __forceinline__ Cx cfma_conj(Cx acc, Cx a, Cx b) {
  acc.x = fma(a.x, b.x, acc.x);
  acc.x = fma(a.y, b.y, acc.x);
  acc.y = fma(a.x, b.y, acc.y);
  acc.y = fma(-a.y, b.x, acc.y);
  return acc;
}

static int num_sms() {
  int dev = 0, n = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
  return n;
}

// ---------------------------------------------------------------------------
// tables and basis layout
// ---------------------------------------------------------------------------
gmg_status agg_build_tables(gmg_agg* h, cudaStream_t s) {
  const int64_t Vc = h->cdims.vol();
  std::vector<int32_t> t(Vc * h->bv);
  for (int64_t sc = 0; sc < Vc; ++sc) {
    int cc[4];
    int64_t q = sc;
    for (int d = 0; d < 4; ++d) { cc[d] = (int)(q % h->cdims.d[d]); q /= h->cdims.d[d]; }
    for (int sb = 0; sb < h->bv; ++sb) {
      int cb[4], cf[4];
      int r = sb;
      for (int d = 0; d < 4; ++d) { cb[d] = r % h->b[d]; r /= h->b[d]; }
      for (int d = 0; d < 4; ++d) cf[d] = cc[d] * h->b[d] + cb[d];
      int64_t sf = 0;
      for (int d = 3; d >= 0; --d) sf = sf * h->fdims.d[d] + cf[d];
      t[sc * h->bv + sb] = (int32_t)sf;
    }
  }
  GMG_TRY(h->blk_sites.alloc(t.size() * sizeof(int32_t)));
  GMG_CUDA(cudaMemcpyAsync(h->blk_sites.p, t.data(), t.size() * sizeof(int32_t),
                           cudaMemcpyHostToDevice, s));
  GMG_CUDA(cudaStreamSynchronize(s));
  return GMG_OK;
}

// basis [i][site][dof] <-> basis_blk [c][i][sb*dof + a]
template <bool TO_BLK>
__global__ void basis_layout_kernel(const double2* __restrict__ src, double2* __restrict__ dst,
                                    const int32_t* __restrict__ blk_sites, int64_t Vc, int N, int bv,
                                    int dof, int64_t Vf) {
  const int64_t K = (int64_t)bv * dof;
  const int64_t total = Vc * N * K;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t k = e % K;
    const int64_t i = (e / K) % N;
    const int64_t c = e / (K * N);
    const int64_t sf = blk_sites[c * bv + k / dof];
    const int64_t fi = (i * Vf + sf) * dof + k % dof;
    if (TO_BLK) dst[e] = src[fi];
    else dst[fi] = src[e];
  }
}

gmg_status agg_basis_to_blocked(gmg_agg* h, const double* basis_dev, cudaStream_t s) {
  const int64_t Vc = h->cdims.vol(), Vf = h->fdims.vol();
  const int64_t total = Vc * h->N * (int64_t)h->bv * h->dof;
  GMG_TRY(h->basis_blk.alloc(total * sizeof(double2)));
  const int grid = (int)std::min<int64_t>((total + 255) / 256, 148 * 64);
  basis_layout_kernel<true><<<grid, 256, 0, s>>>(reinterpret_cast<const double2*>(basis_dev),
                                                  h->basis_blk.as<double2>(), h->blk_sites.as<int32_t>(),
                                                  Vc, h->N, h->bv, h->dof, Vf);
  GMG_CUDA(cudaGetLastError());
  h->basis_f_ok = false;
  h->basis_tc_ok = false;
  // a new basis: the failure flag of the previous orthonormalisation no longer applies
  if (h->ortho_ws.p) GMG_CUDA(cudaMemsetAsync(h->ortho_ws.p, 0, sizeof(int), s));
  return GMG_OK;
}

gmg_status agg_basis_from_blocked(gmg_agg* h, double* basis_dev, cudaStream_t s) {
  const int64_t Vc = h->cdims.vol(), Vf = h->fdims.vol();
  const int64_t total = Vc * h->N * (int64_t)h->bv * h->dof;
  const int grid = (int)std::min<int64_t>((total + 255) / 256, 148 * 64);
  basis_layout_kernel<false><<<grid, 256, 0, s>>>(h->basis_blk.as<double2>(),
                                                   reinterpret_cast<double2*>(basis_dev),
                                                   h->blk_sites.as<int32_t>(), Vc, h->N, h->bv, h->dof, Vf);
  GMG_CUDA(cudaGetLastError());
  return GMG_OK;
}

__global__ void d2f_kernel(const double2* __restrict__ a, float2* __restrict__ b, int64_t n) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n;
       e += (int64_t)gridDim.x * blockDim.x)
    b[e] = make_float2((float)a[e].x, (float)a[e].y);
}

gmg_status agg_prepare_f32(gmg_agg* h, cudaStream_t s) {
  if (h->basis_f_ok) return GMG_OK;
  const int64_t n = h->cdims.vol() * h->N * (int64_t)h->bv * h->dof;
  GMG_TRY(h->basis_blk_f.alloc(n * sizeof(float2)));
  d2f_kernel<<<(int)std::min<int64_t>((n + 255) / 256, 148 * 64), 256, 0, s>>>(
      h->basis_blk.as<double2>(), h->basis_blk_f.as<float2>(), n);
  GMG_CUDA(cudaGetLastError());
  h->basis_f_ok = true;
  return GMG_OK;
}

// ---------------------------------------------------------------------------
// project: coarse[c][r][i] = sum_k conj(V[c][i][k]) F[site(c,k)][r][k % dof]
// CTA per block; K chunked by KS sites; TR x TB register tiles over (rhs, i).
// `mask` (nullable, int8 per fine site) restricts the sum to a face / parity
// subset as the masked LUTs of CoarsenOperator do (...DirsaveLut.h:985-1005).
// ---------------------------------------------------------------------------
// `sel` (nullable, nsel entries): the in-block site indices the sum runs over,
// the same for every block (a face of the block); without it all bv sites.
template <class T, int TR, int TB, int KS>
__global__ void __launch_bounds__(256) project_kernel(
    const typename ctype<T>::t* __restrict__ basis, const int32_t* __restrict__ blk_sites,
    const typename ctype<T>::t* __restrict__ fine, typename ctype<T>::t* __restrict__ coarse,
    int Vc, int N, int dof, int bv, int nrhs, const int8_t* __restrict__ mask, int accumulate,
    const int32_t* __restrict__ sel, int nsel) {
  typedef typename ctype<T>::t Cx;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int KC = KS * dof;
  Cx* VT = reinterpret_cast<Cx*>(smem_raw);  // [KC][N]
  Cx* FT = VT + KC * N;                       // [KC][R]
  const int R = nrhs;
  const int NBT = (N + TB - 1) / TB, NRT = (R + TR - 1) / TR;
  const int ntiles = NBT * NRT;
  const int t = threadIdx.x, bt = t % NBT, rt = t / NBT;
  const int64_t K = (int64_t)bv * dof;
  for (int c = blockIdx.x; c < Vc; c += gridDim.x) {
    Cx acc[TR][TB];
#pragma unroll
    for (int j = 0; j < TR; ++j)
#pragma unroll
      for (int i = 0; i < TB; ++i) acc[j][i] = Cx{0, 0};
    const Cx* Vb = basis + (int64_t)c * N * K;
    const int nsites = sel ? nsel : bv;
    for (int sb0 = 0; sb0 < nsites; sb0 += KS) {
      const int ns = min(KS, nsites - sb0);
      const int kc = ns * dof;
      __syncthreads();
      for (int e = t; e < N * kc; e += blockDim.x) {
        const int i = e / kc, kk = e % kc;
        const int sl = kk / dof, a = kk % dof;
        const int sb = sel ? sel[sb0 + sl] : sb0 + sl;
        VT[kk * N + i] = Vb[(int64_t)i * K + (int64_t)sb * dof + a];
      }
      for (int e = t; e < ns * R * dof; e += blockDim.x) {
        const int sl = e / (R * dof), rem = e % (R * dof);
        const int r = rem / dof, a = rem % dof;
        const int sf = blk_sites[(int64_t)c * bv + (sel ? sel[sb0 + sl] : sb0 + sl)];
        Cx v = fine[((int64_t)sf * nrhs + r) * dof + a];
        if (mask && !mask[sf]) v = Cx{0, 0};
        FT[(sl * dof + a) * R + r] = v;
      }
      __syncthreads();
      if (t < ntiles) {
        for (int kk = 0; kk < kc; ++kk) {
          Cx a[TB], x[TR];
#pragma unroll
          for (int i = 0; i < TB; ++i) {
            const int ii = bt * TB + i;
            a[i] = ii < N ? VT[kk * N + ii] : Cx{0, 0};
          }
#pragma unroll
          for (int j = 0; j < TR; ++j) {
            const int r = rt * TR + j;
            x[j] = r < R ? FT[kk * R + r] : Cx{0, 0};
          }
#pragma unroll
          for (int j = 0; j < TR; ++j)
#pragma unroll
            for (int i = 0; i < TB; ++i) acc[j][i] = cfma_conj(acc[j][i], a[i], x[j]);
        }
      }
    }
    if (t < ntiles) {
#pragma unroll
      for (int j = 0; j < TR; ++j) {
        const int r = rt * TR + j;
        if (r >= R) continue;
#pragma unroll
        for (int i = 0; i < TB; ++i) {
          const int ii = bt * TB + i;
          if (ii >= N) continue;
          Cx* o = coarse + ((int64_t)c * nrhs + r) * N + ii;
          if (accumulate) { Cx v = *o; v.x += acc[j][i].x; v.y += acc[j][i].y; *o = v; }
          else *o = acc[j][i];
        }
      }
    }
  }
}

template <class T, int TR, int TB, int KS>
static gmg_status launch_project(gmg_agg* h, const void* basis, int nrhs, const void* fine,
                                 void* coarse, const int8_t* mask, int accumulate, cudaStream_t s,
                                 const int32_t* sel = nullptr, int nsel = 0) {
  typedef typename ctype<T>::t Cx;
  const int N = h->N, R = nrhs;
  const int ntiles = ((N + TB - 1) / TB) * ((R + TR - 1) / TR);
  GMG_CHECK(ntiles <= 256, GMG_ERR_UNSUPPORTED, "project: nbasis x nrhs too large");
  const int threads = std::max(32, (ntiles + 31) / 32 * 32);
  const size_t smem = sizeof(Cx) * (size_t)KS * h->dof * (N + R);
  GMG_CHECK(smem <= 227 * 1024, GMG_ERR_UNSUPPORTED, "project: shared-memory tile too large");
  auto kern = project_kernel<T, TR, TB, KS>;
  GMG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int Vc = (int)h->cdims.vol();
  const int grid = std::min(Vc, num_sms() * 16);
  KernelTimer kt("project", s);
  kern<<<grid, threads, smem, s>>>(reinterpret_cast<const Cx*>(basis), h->blk_sites.as<int32_t>(),
                                   reinterpret_cast<const Cx*>(fine), reinterpret_cast<Cx*>(coarse),
                                   Vc, N, h->dof, h->bv, nrhs, mask, accumulate, sel, nsel);
  GMG_CUDA(cudaGetLastError());
  return GMG_OK;
}

// ---------------------------------------------------------------------------
// FP64 projection of spin-colour fields (dof 12, nrhs >= 4), pipelined: the
// same sums as project_kernel, with
//   - the next KS-site chunk of basis and fine field copied into the second
//     shared-memory buffer (cp.async, 16 B per complex number, written
//     straight into the transposed [k][N] / [k][R] tiles) while the current
//     one is multiplied, so the global loads no longer stall the FMA loop;
//   - basis rows and RHS interleaved over the threads (thread (bt, rt) owns
//     rows bt + NBT i and RHS rt + NRT j), so the 16-byte shared loads of
//     neighbouring threads fall on consecutive banks;
//   - the chunk's index arithmetic on compile-time strides.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(static_cast<uint32_t>(__cvta_generic_to_shared(smem))),
               "l"(gmem)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N_>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N_) : "memory"); }

template <int DOF, int KS, int TR, int TB, int NT>
__global__ void __launch_bounds__(NT, 384 / NT) project_f64_pipe_kernel(
    const double2* __restrict__ basis, const int32_t* __restrict__ blk_sites, const double2* __restrict__ fine,
    double2* __restrict__ coarse, int Vc, int N, int bv, int nrhs, const int32_t* __restrict__ sel, int nsel) {
  constexpr int KC = KS * DOF;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int R = nrhs;
  const int NBT = (N + TB - 1) / TB, NRT = (R + TR - 1) / TR;
  // tile widths padded to whole register tiles; the pad columns are zeroed
  // once and never copied to, so the multiply loop needs no bounds tests
  const int Np = NBT * TB, Rq = NRT * TR;
  double2* buf0 = reinterpret_cast<double2*>(smem_raw);  // per buffer: VT [KC][Np], FT [KC][Rq]
  const int bufsz = KC * (Np + Rq);
  const int ntiles = NBT * NRT;
  const int t = threadIdx.x, bt = t % NBT, rt = t / NBT;
  const int64_t K = (int64_t)bv * DOF;
  const int nsites = sel ? nsel : bv;
  const int nch = (nsites + KS - 1) / KS;
  for (int e = t; e < 2 * bufsz; e += NT) buf0[e] = make_double2(0.0, 0.0);
  for (int c = blockIdx.x; c < Vc; c += gridDim.x) {
    const double2* Vb = basis + (int64_t)c * N * K;
    // copies of chunk ch into buffer b (sites beyond nsites are skipped; the
    // multiply loop stops at the chunk's own length)
    auto issue = [&](int ch, int b) {
      double2* VT = buf0 + b * bufsz;
      double2* FT = VT + KC * Np;
      const int sb0 = ch * KS;
      const int ns = min(KS, nsites - sb0);
      for (int e = t; e < N * KC; e += NT) {
        const int i = e / KC, kk = e % KC;
        const int sl = kk / DOF, a = kk % DOF;
        if (sl < ns) {
          const int sb = sel ? sel[sb0 + sl] : sb0 + sl;
          cp_async16(VT + kk * Np + i, Vb + (int64_t)i * K + (int64_t)sb * DOF + a);
        }
      }
      for (int sl = 0; sl < ns; ++sl) {
        const int64_t sf = blk_sites[(int64_t)c * bv + (sel ? sel[sb0 + sl] : sb0 + sl)];
        const double2* src = fine + sf * nrhs * DOF;
        for (int e = t; e < R * DOF; e += NT) {
          const int r = e / DOF, a = e % DOF;
          cp_async16(FT + (sl * DOF + a) * Rq + r, src + e);
        }
      }
      cp_async_commit();
    };
    double2 acc[TR][TB];
#pragma unroll
    for (int j = 0; j < TR; ++j)
#pragma unroll
      for (int i = 0; i < TB; ++i) acc[j][i] = make_double2(0.0, 0.0);
    __syncthreads();  // zeroing done / the previous block's last chunk is no longer read
    issue(0, 0);
    for (int ch = 0; ch < nch; ++ch) {
      if (ch + 1 < nch) {
        issue(ch + 1, (ch + 1) & 1);
        cp_async_wait<1>();
      } else {
        cp_async_wait<0>();
      }
      __syncthreads();
      const double2* va = buf0 + (ch & 1) * bufsz + bt;
      const double2* xa = buf0 + (ch & 1) * bufsz + KC * Np + rt;
      const int kc = min(KS, nsites - ch * KS) * DOF;
      if (t < ntiles) {
#pragma unroll 1
        for (int kk = 0; kk < kc; ++kk) {
          double2 a[TB], x[TR];
#pragma unroll
          for (int i = 0; i < TB; ++i) a[i] = va[kk * Np + NBT * i];
#pragma unroll
          for (int j = 0; j < TR; ++j) x[j] = xa[kk * Rq + NRT * j];
#pragma unroll
          for (int j = 0; j < TR; ++j)
#pragma unroll
            for (int i = 0; i < TB; ++i) acc[j][i] = cfma_conj(acc[j][i], a[i], x[j]);
        }
      }
      __syncthreads();  // buffer (ch & 1) is refilled by the issue of chunk ch + 2
    }
    if (t < ntiles) {
#pragma unroll
      for (int j = 0; j < TR; ++j) {
        const int r = rt + NRT * j;
        if (r >= R) continue;
#pragma unroll
        for (int i = 0; i < TB; ++i) {
          const int ii = bt + NBT * i;
          if (ii < N) coarse[((int64_t)c * nrhs + r) * N + ii] = acc[j][i];
        }
      }
    }
  }
}

template <int KS, int TR, int TB, int NT>
static gmg_status launch_pipe(gmg_agg* h, int nrhs, const void* fine, void* coarse, const int32_t* sel, int nsel,
                              cudaStream_t s) {
  const int N = h->N, R = nrhs;
  const int Np = (N + TB - 1) / TB * TB, Rq = (R + TR - 1) / TR * TR;
  const size_t smem = sizeof(double2) * 2 * (size_t)KS * 12 * (Np + Rq);
  auto kern = project_f64_pipe_kernel<12, KS, TR, TB, NT>;
  GMG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int Vc = (int)h->cdims.vol();
  const int grid = std::min(Vc, num_sms() * 16);
  KernelTimer kt("project", s);
  kern<<<grid, NT, smem, s>>>(h->basis_blk.as<double2>(), h->blk_sites.as<int32_t>(),
                              reinterpret_cast<const double2*>(fine), reinterpret_cast<double2*>(coarse), Vc, N, h->bv,
                              nrhs, sel, nsel);
  GMG_CUDA(cudaGetLastError());
  return GMG_OK;
}

// the pipelined FP64 projection when it applies (dof 12, 4 <= nrhs, tiles and
// two buffers within limits); *launched = false otherwise.  5 x 5 register
// tiles on 64 threads when they fill more than one warp with nbasis and nrhs
// up to 40 (the coarsening's 40 x 40: 64 threads, no idle lanes), else 4 x 4
// on 128 threads.
static gmg_status launch_project_f64_pipe(gmg_agg* h, int nrhs, const void* fine, void* coarse, const int32_t* sel,
                                          int nsel, cudaStream_t s, bool* launched) {
  *launched = false;
  const int N = h->N, R = nrhs;
  if (h->dof != 12 || R < 4 || (reinterpret_cast<uintptr_t>(fine) & 15)) return GMG_OK;
  const int t5 = ((N + 4) / 5) * ((R + 4) / 5);
  if (N <= 40 && R <= 40 && t5 > 32) {
    GMG_TRY((launch_pipe<1, 5, 5, 64>(h, nrhs, fine, coarse, sel, nsel, s)));
  } else {
    const int t4 = ((N + 3) / 4) * ((R + 3) / 4);
    if (t4 > 128 || sizeof(double2) * 2 * 2 * 12 * (size_t)(N + R + 6) > 200 * 1024) return GMG_OK;
    GMG_TRY((launch_pipe<2, 4, 4, 128>(h, nrhs, fine, coarse, sel, nsel, s)));
  }
  *launched = true;
  return GMG_OK;
}

gmg_status agg_project(gmg_agg* h, int compute, int vec_prec, int nrhs, const void* fine,
                       void* coarse, const int32_t* mask_unused, cudaStream_t s) {
  (void)mask_unused;
  if (compute == GMG_BF16 && vec_prec == GMG_F32) return agg_project_tc(h, nrhs, (const float*)fine, (float*)coarse, s);
  GMG_CHECK(compute == vec_prec, GMG_ERR_UNSUPPORTED, "project: compute and vector precision differ");
  if (compute == GMG_F64) {
    bool done = false;
    GMG_TRY(launch_project_f64_pipe(h, nrhs, fine, coarse, nullptr, 0, s, &done));
    if (done) return GMG_OK;
    if (nrhs >= 4) return launch_project<double, 4, 4, 4>(h, h->basis_blk.p, nrhs, fine, coarse, nullptr, 0, s);
    return launch_project<double, 1, 2, 4>(h, h->basis_blk.p, nrhs, fine, coarse, nullptr, 0, s);
  }
  if (compute == GMG_F32) {
    GMG_TRY(agg_prepare_f32(h, s));
    if (nrhs >= 4) return launch_project<float, 4, 4, 4>(h, h->basis_blk_f.p, nrhs, fine, coarse, nullptr, 0, s);
    return launch_project<float, 1, 2, 4>(h, h->basis_blk_f.p, nrhs, fine, coarse, nullptr, 0, s);
  }
  return fail(GMG_ERR_UNSUPPORTED, "project: unsupported precision");
}

// FP64 projection over a subset of every block's sites (sel: nsel in-block
// indices on the device, the same for all blocks), used for the face terms of
// the coarse-operator construction
gmg_status agg_project_sel_f64(gmg_agg* h, int nrhs, const double* fine, double* coarse, const int32_t* sel,
                               int nsel, cudaStream_t s) {
  bool done = false;
  GMG_TRY(launch_project_f64_pipe(h, nrhs, fine, coarse, sel, nsel, s, &done));
  if (done) return GMG_OK;
  if (nrhs >= 4)
    return launch_project<double, 4, 4, 4>(h, h->basis_blk.p, nrhs, fine, coarse, nullptr, 0, s, sel, nsel);
  return launch_project<double, 1, 2, 4>(h, h->basis_blk.p, nrhs, fine, coarse, nullptr, 0, s, sel, nsel);
}

// masked FP64 single-RHS projection used by the coarse-operator construction
gmg_status agg_project_masked_f64(gmg_agg* h, int nrhs, const double* fine, double* coarse,
                                  const int8_t* mask, cudaStream_t s) {
  if (!mask) {
    bool done = false;
    GMG_TRY(launch_project_f64_pipe(h, nrhs, fine, coarse, nullptr, 0, s, &done));
    if (done) return GMG_OK;
  }
  if (nrhs >= 4) return launch_project<double, 4, 4, 4>(h, h->basis_blk.p, nrhs, fine, coarse, mask, 0, s);
  return launch_project<double, 1, 2, 4>(h, h->basis_blk.p, nrhs, fine, coarse, mask, 0, s);
}

// ---------------------------------------------------------------------------
// promote: F[site(c,k)][r][k%dof] = sum_i V[c][i][k] C[c][r][i]
// ---------------------------------------------------------------------------
template <class T, int TK, int TR, int KS>
__global__ void __launch_bounds__(256) promote_kernel(
    const typename ctype<T>::t* __restrict__ basis, const int32_t* __restrict__ blk_sites,
    const typename ctype<T>::t* __restrict__ coarse, typename ctype<T>::t* __restrict__ fine, int Vc,
    int N, int dof, int bv, int nrhs) {
  typedef typename ctype<T>::t Cx;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int KC = KS * dof;
  const int R = nrhs;
  Cx* CT = reinterpret_cast<Cx*>(smem_raw);  // [N][R]
  Cx* VS = CT + N * R;                        // [N][KC]
  const int NKT = KC / TK, NRT = (R + TR - 1) / TR;
  const int ntiles = NKT * NRT;
  const int t = threadIdx.x;
  const int64_t K = (int64_t)bv * dof;
  for (int c = blockIdx.x; c < Vc; c += gridDim.x) {
    __syncthreads();
    for (int e = t; e < N * R; e += blockDim.x) {
      const int r = e / N, i = e % N;
      CT[i * R + r] = coarse[((int64_t)c * nrhs + r) * N + i];
    }
    const Cx* Vb = basis + (int64_t)c * N * K;
    for (int sb0 = 0; sb0 < bv; sb0 += KS) {
      const int ns = min(KS, bv - sb0);
      const int kc = ns * dof;
      __syncthreads();
      for (int e = t; e < N * kc; e += blockDim.x) {
        const int i = e / kc, kk = e % kc;
        VS[i * KC + kk] = Vb[(int64_t)i * K + (int64_t)sb0 * dof + kk];
      }
      __syncthreads();
      for (int tile = t; tile < ntiles; tile += blockDim.x) {
        const int kt = tile % NKT, rt = tile / NKT;
        if (kt * TK >= kc) continue;
        Cx acc[TR][TK];
#pragma unroll
        for (int j = 0; j < TR; ++j)
#pragma unroll
          for (int q = 0; q < TK; ++q) acc[j][q] = Cx{0, 0};
        for (int i = 0; i < N; ++i) {
          Cx v[TK], x[TR];
#pragma unroll
          for (int q = 0; q < TK; ++q) v[q] = VS[i * KC + kt * TK + q];
#pragma unroll
          for (int j = 0; j < TR; ++j) {
            const int r = rt * TR + j;
            x[j] = r < R ? CT[i * R + r] : Cx{0, 0};
          }
#pragma unroll
          for (int j = 0; j < TR; ++j)
#pragma unroll
            for (int q = 0; q < TK; ++q) acc[j][q] = cfma(acc[j][q], x[j], v[q]);
        }
        const int k0 = kt * TK;
        const int sl = k0 / dof, a0 = k0 % dof;  // TK divides dof: one site per tile
        const int sf = blk_sites[(int64_t)c * bv + sb0 + sl];
#pragma unroll
        for (int j = 0; j < TR; ++j) {
          const int r = rt * TR + j;
          if (r >= R) continue;
          Cx* o = fine + ((int64_t)sf * nrhs + r) * dof + a0;
#pragma unroll
          for (int q = 0; q < TK; ++q) o[q] = acc[j][q];
        }
      }
    }
  }
}

template <class T, int TK, int TR, int KS>
static gmg_status launch_promote(gmg_agg* h, const void* basis, int nrhs, const void* coarse,
                                 void* fine, cudaStream_t s) {
  typedef typename ctype<T>::t Cx;
  const int N = h->N, R = nrhs, dof = h->dof;
  GMG_CHECK(dof % TK == 0, GMG_ERR_UNSUPPORTED, "promote: dof not a multiple of the k tile");
  const int ntiles = (KS * dof / TK) * ((R + TR - 1) / TR);
  const int threads = std::min(256, std::max(32, (ntiles + 31) / 32 * 32));
  const size_t smem = sizeof(Cx) * ((size_t)N * R + (size_t)N * KS * dof);
  GMG_CHECK(smem <= 227 * 1024, GMG_ERR_UNSUPPORTED, "promote: shared-memory tile too large");
  auto kern = promote_kernel<T, TK, TR, KS>;
  GMG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int Vc = (int)h->cdims.vol();
  const int grid = std::min(Vc, num_sms() * 16);
  KernelTimer kt("promote", s);
  kern<<<grid, threads, smem, s>>>(reinterpret_cast<const Cx*>(basis), h->blk_sites.as<int32_t>(),
                                   reinterpret_cast<const Cx*>(coarse), reinterpret_cast<Cx*>(fine),
                                   Vc, N, dof, h->bv, nrhs);
  GMG_CUDA(cudaGetLastError());
  return GMG_OK;
}

gmg_status agg_promote(gmg_agg* h, int compute, int vec_prec, int nrhs, const void* coarse,
                       void* fine, cudaStream_t s) {
  if (compute == GMG_BF16 && vec_prec == GMG_F32) return agg_promote_tc(h, nrhs, (const float*)coarse, (float*)fine, s);
  GMG_CHECK(compute == vec_prec, GMG_ERR_UNSUPPORTED, "promote: compute and vector precision differ");
  const bool tk4 = h->dof % 4 == 0;
  if (compute == GMG_F64) {
    if (nrhs >= 4 && tk4) return launch_promote<double, 4, 4, 4>(h, h->basis_blk.p, nrhs, coarse, fine, s);
    if (tk4) return launch_promote<double, 4, 1, 4>(h, h->basis_blk.p, nrhs, coarse, fine, s);
    return launch_promote<double, 1, 1, 4>(h, h->basis_blk.p, nrhs, coarse, fine, s);
  }
  if (compute == GMG_F32) {
    GMG_TRY(agg_prepare_f32(h, s));
    if (nrhs >= 4 && tk4) return launch_promote<float, 4, 4, 4>(h, h->basis_blk_f.p, nrhs, coarse, fine, s);
    if (tk4) return launch_promote<float, 4, 1, 4>(h, h->basis_blk_f.p, nrhs, coarse, fine, s);
    return launch_promote<float, 1, 1, 4>(h, h->basis_blk_f.p, nrhs, coarse, fine, s);
  }
  return fail(GMG_ERR_UNSUPPORTED, "promote: unsupported precision");
}

}  // namespace gmg

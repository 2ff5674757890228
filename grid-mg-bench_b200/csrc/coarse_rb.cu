// coarse_rb.cu -- red-black (checkerboarded) coarse operator.
//
// Restates the Schur-decomposition interface of Rework::CoarsenedMatrix
// (include/CoarsenedMatrixRework.h):
//   Dhop(in, out, dag)              :210-217   the 8 hopping points on the full grid
//   DhopOE / DhopEO -> Meooe[Dag]   :186-200, 219-237, DhopInternal :288-394
//   Mooee[Inv][Dag]                 :202-208, MooeeInternal :617-640
//   InvertSelfStencilPoint          :642-668   (a CPU + Eigen loop in the reference)
//   FillHalfCbs                     :670-679
// The dagger of a hop is G5C Dhop G5C (the Galerkin form the reference hard-
// codes, :289-346); the dagger of Mooee is the conjugate transpose of the self
// link (or of its inverse).
//
// Half fields hold the sites of one parity q = (x+y+z+t) % 2, at half index
// h = x/2 + (Lx/2)(y + Ly(z + Lz t)) (Grid's red-black grid, checkerboarded in
// x).  Instead of FillHalfCbs copies of the links, two tables map a half index
// to its full site (the links are read in place) and to the half indices of
// its 9 stencil neighbours; every apply then runs the full-grid kernels
// (CUDA-core FP64 / FP32, or the tcgen05 stencil for BF16 / FP16 hops) on that
// sub-geometry.
//
// The self-link inverse is computed on the device: one CTA per site, Gauss-
// Jordan elimination with partial pivoting on the N x 2N augmented matrix in
// shared memory, FP64.
#include <algorithm>
#include <vector>

#include "gmg_internal.cuh"

namespace gmg {

static int half_index_host(const int* L, int x, int y, int z, int t) {
  return x / 2 + (L[0] / 2) * (y + L[1] * (z + L[2] * t));
}

gmg_status coarse_rb_tables(gmg_coarse* h, cudaStream_t s) {
  if (h->rb_ok) return GMG_OK;
  const int* L = h->dims.d;
  for (int k = 0; k < 4; ++k)
    GMG_CHECK(L[k] % 2 == 0, GMG_ERR_SHAPE, "red-black coarse operator: lattice extents must be even");
  const int V = (int)h->dims.vol(), Vh = V / 2;
  std::vector<int32_t> nbr((size_t)9 * V), site((size_t)2 * Vh), rbn((size_t)2 * 9 * Vh);
  host_neighbors(h->dims, nbr.data());
  std::vector<int32_t> hidx(V);
  for (int t = 0; t < L[3]; ++t)
    for (int z = 0; z < L[2]; ++z)
      for (int y = 0; y < L[1]; ++y)
        for (int x = 0; x < L[0]; ++x) {
          const int f = x + L[0] * (y + L[1] * (z + L[2] * t));
          const int q = (x + y + z + t) & 1;
          const int hh = half_index_host(L, x, y, z, t);
          hidx[f] = hh;
          site[(size_t)q * Vh + hh] = f;
        }
  for (int q = 0; q < 2; ++q)
    for (int hh = 0; hh < Vh; ++hh) {
      const int f = site[(size_t)q * Vh + hh];
      for (int p = 0; p < 9; ++p) rbn[((size_t)q * 9 + p) * Vh + hh] = hidx[nbr[(size_t)p * V + f]];
    }
  GMG_TRY(h->rb_site.alloc(sizeof(int32_t) * site.size()));
  GMG_TRY(h->rb_nbr.alloc(sizeof(int32_t) * rbn.size()));
  GMG_CUDA(cudaMemcpyAsync(h->rb_site.p, site.data(), sizeof(int32_t) * site.size(), cudaMemcpyHostToDevice, s));
  GMG_CUDA(cudaMemcpyAsync(h->rb_nbr.p, rbn.data(), sizeof(int32_t) * rbn.size(), cudaMemcpyHostToDevice, s));
  GMG_CUDA(cudaStreamSynchronize(s));  // the host tables go out of scope
  h->rb_ok = true;
  return GMG_OK;
}

// ---------------------------------------------------------------------------
// self-link inverse
// ---------------------------------------------------------------------------
__device__ __forceinline__ double2 zmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// A8 at links_d + (s*9 + 8) N^2 (site-major); inverse -> inv + s N^2.  Singular
// sites set *err (GMG_ERR_NONFINITE) and leave garbage in their inverse.
__global__ void __launch_bounds__(256) invert_self_kernel(const double2* __restrict__ links, double2* __restrict__ inv,
                                                          float2* __restrict__ inv_f, int V, int N, int* err) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double2* M = reinterpret_cast<double2*>(smem_raw);  // [N][2N]
  double2* f = M + 2 * N * N;                         // [N] elimination factors
  __shared__ int piv;
  __shared__ double2 dinv;
  const int W = 2 * N;
  for (int s = blockIdx.x; s < V; s += gridDim.x) {
    const double2* A = links + ((int64_t)s * 9 + 8) * N * N;
    for (int k = threadIdx.x; k < N * W; k += blockDim.x) {
      const int i = k / W, j = k % W;
      M[k] = j < N ? A[i * N + j] : make_double2(j - N == i ? 1.0 : 0.0, 0.0);
    }
    __syncthreads();
    for (int col = 0; col < N; ++col) {
      if (threadIdx.x < 32) {  // pivot: the largest |M[r][col]|, r >= col
        double best = -1.0;
        int bi = col;
        for (int r = col + threadIdx.x; r < N; r += 32) {
          const double2 v = M[r * W + col];
          const double m = v.x * v.x + v.y * v.y;
          if (m > best) {
            best = m;
            bi = r;
          }
        }
        for (int o = 16; o > 0; o >>= 1) {
          const double ob = __shfl_xor_sync(0xffffffffu, best, o);
          const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
          if (ob > best || (ob == best && oi < bi)) {
            best = ob;
            bi = oi;
          }
        }
        if (threadIdx.x == 0) {
          piv = bi;
          if (!(best > 0.0)) atomicCAS(err, 0, (int)GMG_ERR_NONFINITE);
        }
      }
      __syncthreads();
      const int pr = piv;
      if (pr != col)
        for (int k = threadIdx.x; k < W; k += blockDim.x) {
          const double2 a = M[col * W + k];
          M[col * W + k] = M[pr * W + k];
          M[pr * W + k] = a;
        }
      __syncthreads();
      if (threadIdx.x == 0) {
        const double2 d = M[col * W + col];
        const double n = d.x * d.x + d.y * d.y;
        dinv = n > 0.0 ? make_double2(d.x / n, -d.y / n) : make_double2(0.0, 0.0);
      }
      __syncthreads();
      for (int k = threadIdx.x; k < W; k += blockDim.x) M[col * W + k] = zmul(M[col * W + k], dinv);
      for (int r = threadIdx.x; r < N; r += blockDim.x) f[r] = r == col ? make_double2(0.0, 0.0) : M[r * W + col];
      __syncthreads();
      for (int k = threadIdx.x; k < N * W; k += blockDim.x) {
        const int r = k / W, j = k % W;
        if (r == col) continue;  // the pivot row is read by every other row
        const double2 a = zmul(f[r], M[col * W + j]);
        M[k].x -= a.x;
        M[k].y -= a.y;
      }
      __syncthreads();
    }
    for (int k = threadIdx.x; k < N * N; k += blockDim.x) {
      const int i = k / N, j = k % N;
      const double2 v = M[i * W + N + j];
      inv[(int64_t)s * N * N + k] = v;
      if (inv_f) inv_f[(int64_t)s * N * N + k] = make_float2((float)v.x, (float)v.y);
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// pickCheckerboard / setCheckerboard on [site][per] complex fields
// ---------------------------------------------------------------------------
template <class C>
__global__ void checkerboard_kernel(const C* __restrict__ src, C* __restrict__ dst, int L0, int L1, int L2, int L3,
                                    int cb, int64_t per, int to_half) {
  const int64_t Vh = (int64_t)L0 * L1 * L2 * L3 / 2;
  const int Lh = L0 / 2;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < Vh * per;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t hh = e / per, k = e % per;
    int64_t rest = hh / Lh;
    const int xh = (int)(hh % Lh);
    const int y = (int)(rest % L1);
    rest /= L1;
    const int z = (int)(rest % L2);
    const int t = (int)(rest / L2);
    const int x = 2 * xh + ((y + z + t + cb) & 1);
    const int64_t f = x + (int64_t)L0 * (y + (int64_t)L1 * (z + (int64_t)L2 * t));
    if (to_half)
      dst[e] = src[f * per + k];
    else
      dst[f * per + k] = src[e];
  }
}

}  // namespace gmg

using namespace gmg;

extern "C" gmg_status gmg_coarse_invert_self(gmg_coarse* h, gmg_stream stream) {
  GMG_CHECK(h != nullptr, GMG_ERR_ARGUMENT, "gmg_coarse_invert_self: null handle");
  GMG_CHECK(h->links_set, GMG_ERR_STATE, "gmg_coarse_invert_self: links not set");
  GMG_CHECK(h->N <= 64, GMG_ERR_UNSUPPORTED, "gmg_coarse_invert_self: nbasis above 64");
  cudaStream_t s = S(stream);
  const int V = (int)h->dims.vol(), N = h->N;
  GMG_TRY(h->self_inv.alloc(sizeof(double2) * (size_t)V * N * N));
  GMG_TRY(h->self_inv_f.alloc(sizeof(float2) * (size_t)V * N * N));
  if (!h->dev_err.p) GMG_TRY(h->dev_err.alloc(256));
  GMG_CUDA(cudaMemsetAsync(h->dev_err.p, 0, sizeof(int), s));
  const size_t smem = sizeof(double2) * (2 * (size_t)N * N + N);
  GMG_CUDA(cudaFuncSetAttribute(invert_self_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  invert_self_kernel<<<std::min(V, 148 * 8), 256, smem, s>>>(h->links_d.as<double2>(), h->self_inv.as<double2>(),
                                                              h->self_inv_f.as<float2>(), V, N, h->dev_err.as<int>());
  GMG_CUDA(cudaGetLastError());
  int code = 0;
  GMG_CUDA(cudaMemcpyAsync(&code, h->dev_err.p, sizeof(int), cudaMemcpyDeviceToHost, s));
  GMG_CUDA(cudaStreamSynchronize(s));
  if (code) {
    GMG_CUDA(cudaMemset(h->dev_err.p, 0, sizeof(int)));
    h->self_inv_ok = h->self_inv_f_ok = false;
    return fail(GMG_ERR_NONFINITE, "gmg_coarse_invert_self: a self-stencil link is singular");
  }
  h->self_inv_ok = h->self_inv_f_ok = true;
  return GMG_OK;
}

static bool prec_is_vec(gmg_prec p) { return p == GMG_F64 || p == GMG_F32; }

// op in {MOOEE .. MOOEE_INV_DAG}: the self point on a geometry, as a SIMT apply
static gmg_status mooee_apply(gmg_coarse* h, gmg_rb_op op, int V, const int32_t* site_map, gmg_prec compute,
                              gmg_prec vec_prec, int nrhs, const void* in, void* out, cudaStream_t s) {
  const bool inv = op == GMG_RB_MOOEE_INV || op == GMG_RB_MOOEE_INV_DAG;
  const bool dag = op == GMG_RB_MOOEE_DAG || op == GMG_RB_MOOEE_INV_DAG;
  if (inv) GMG_CHECK(h->self_inv_ok, GMG_ERR_STATE, "MooeeInv: call gmg_coarse_invert_self first");
  // the self point is one N x N product per site: the CUDA-core kernel in the
  // vectors' precision (BF16 / FP16 requests use FP32 arithmetic here)
  int c = compute;
  if (c == GMG_BF16 || c == GMG_F16) c = GMG_F32;
  if (c == GMG_F32 && !inv && !h->links_f_ok) GMG_TRY(coarse_prepare_f32(h, s));
  return coarse_apply_simt_ex(h, inv ? 1 : 0, V, site_map, nullptr, dag, 8, 9, false, c, vec_prec, nrhs, in, out,
                              nullptr, 0, s);
}

static gmg_status check_apply(gmg_coarse* h, gmg_prec vec_prec, int nrhs, const void* in, void* out, const char* who) {
  GMG_CHECK(h != nullptr, GMG_ERR_ARGUMENT, std::string(who) + ": null handle");
  GMG_CHECK(in && out, GMG_ERR_ARGUMENT, std::string(who) + ": null vector");
  GMG_CHECK(in != out, GMG_ERR_ARGUMENT, std::string(who) + ": in and out must not alias");
  GMG_CHECK(h->links_set, GMG_ERR_STATE, std::string(who) + ": links not set");
  GMG_CHECK(nrhs >= 1 && nrhs <= 1024, GMG_ERR_ARGUMENT, std::string(who) + ": nrhs out of range");
  GMG_CHECK(prec_is_vec(vec_prec), GMG_ERR_ARGUMENT, std::string(who) + ": vectors must be F64 or F32");
  return GMG_OK;
}

// hops (points 0..7) on a geometry, tensor cores for BF16 / FP16
static gmg_status hop_apply(gmg_coarse* h, int V, int V_in, const int32_t* site_map, const int32_t* nbr, bool dag,
                            gmg_prec compute, gmg_prec vec_prec, int nrhs, const void* in, void* out,
                            cudaStream_t s) {
  if (compute == GMG_BF16 || compute == GMG_F16) {
    GMG_CHECK(vec_prec == GMG_F32, GMG_ERR_UNSUPPORTED, "tensor-core coarse apply takes F32 vectors");
    GMG_CHECK(h->links_h.kind == compute, GMG_ERR_STATE,
              "tensor-core links not prepared for this precision (gmg_coarse_prepare)");
    return coarse_apply_tc_ex(h, V, V_in, site_map, nbr, 0, 8, dag, compute, nrhs, (const float*)in, (float*)out,
                              nullptr, 0, s);
  }
  return coarse_apply_simt_ex(h, 0, V, site_map, nbr, false, 0, 8, dag, compute, vec_prec, nrhs, in, out, nullptr, 0,
                              s);
}

extern "C" gmg_status gmg_coarse_apply_rb(gmg_coarse* h, gmg_rb_op op, int cb, gmg_prec compute, gmg_prec vec_prec,
                                          int nrhs, const void* in, void* out, gmg_stream stream) {
  GMG_TRY(check_apply(h, vec_prec, nrhs, in, out, "gmg_coarse_apply_rb"));
  GMG_CHECK(cb == 0 || cb == 1, GMG_ERR_ARGUMENT, "gmg_coarse_apply_rb: cb must be 0 (even) or 1 (odd)");
  cudaStream_t s = S(stream);
  GMG_TRY(coarse_rb_tables(h, s));
  const int Vh = (int)(h->dims.vol() / 2);
  switch (op) {
    case GMG_RB_MEOOE:
    case GMG_RB_MEOOE_DAG: {
      const int q = 1 - cb;  // output parity
      return hop_apply(h, Vh, Vh, h->rb_site.as<int32_t>() + (size_t)q * Vh, h->rb_nbr.as<int32_t>() + (size_t)q * 9 * Vh,
                       op == GMG_RB_MEOOE_DAG, compute, vec_prec, nrhs, in, out, s);
    }
    case GMG_RB_MOOEE:
    case GMG_RB_MOOEE_DAG:
    case GMG_RB_MOOEE_INV:
    case GMG_RB_MOOEE_INV_DAG:
      return mooee_apply(h, op, Vh, h->rb_site.as<int32_t>() + (size_t)cb * Vh, compute, vec_prec, nrhs, in, out, s);
    default:
      return fail(GMG_ERR_ARGUMENT, "gmg_coarse_apply_rb: bad op");
  }
}

extern "C" gmg_status gmg_coarse_dhop(gmg_coarse* h, int dag, gmg_prec compute, gmg_prec vec_prec, int nrhs,
                                      const void* in, void* out, gmg_stream stream) {
  GMG_TRY(check_apply(h, vec_prec, nrhs, in, out, "gmg_coarse_dhop"));
  const int V = (int)h->dims.vol();
  return hop_apply(h, V, V, nullptr, h->nbr.as<int32_t>(), dag != 0, compute, vec_prec, nrhs, in, out, S(stream));
}

extern "C" gmg_status gmg_coarse_mooee(gmg_coarse* h, gmg_rb_op op, gmg_prec compute, gmg_prec vec_prec, int nrhs,
                                       const void* in, void* out, gmg_stream stream) {
  GMG_TRY(check_apply(h, vec_prec, nrhs, in, out, "gmg_coarse_mooee"));
  GMG_CHECK(op >= GMG_RB_MOOEE && op <= GMG_RB_MOOEE_INV_DAG, GMG_ERR_ARGUMENT, "gmg_coarse_mooee: bad op");
  return mooee_apply(h, op, (int)h->dims.vol(), nullptr, compute, vec_prec, nrhs, in, out, S(stream));
}

static gmg_status checkerboard(const int* dims, int cb, int per_site, gmg_prec prec, const void* src, void* dst,
                               int to_half, gmg_stream stream, const char* who) {
  GMG_CHECK(dims && src && dst, GMG_ERR_ARGUMENT, std::string(who) + ": null argument");
  GMG_TRY(check_dims(dims, who));
  for (int k = 0; k < 4; ++k) GMG_CHECK(dims[k] % 2 == 0, GMG_ERR_SHAPE, std::string(who) + ": extents must be even");
  GMG_CHECK(cb == 0 || cb == 1, GMG_ERR_ARGUMENT, std::string(who) + ": cb must be 0 or 1");
  GMG_CHECK(per_site >= 1, GMG_ERR_ARGUMENT, std::string(who) + ": per_site must be positive");
  GMG_CHECK(prec_is_vec(prec), GMG_ERR_ARGUMENT, std::string(who) + ": fields must be F64 or F32");
  const int64_t n = (int64_t)dims[0] * dims[1] * dims[2] * dims[3] / 2 * per_site;
  const int grid = (int)std::min<int64_t>((n + 255) / 256, 148 * 32);
  cudaStream_t s = S(stream);
  if (prec == GMG_F64)
    checkerboard_kernel<double2><<<grid, 256, 0, s>>>((const double2*)src, (double2*)dst, dims[0], dims[1], dims[2],
                                                      dims[3], cb, per_site, to_half);
  else
    checkerboard_kernel<float2><<<grid, 256, 0, s>>>((const float2*)src, (float2*)dst, dims[0], dims[1], dims[2],
                                                     dims[3], cb, per_site, to_half);
  GMG_CUDA(cudaGetLastError());
  return GMG_OK;
}

extern "C" gmg_status gmg_pick_checkerboard(const int dims[4], int cb, int per_site, gmg_prec prec, const void* full,
                                            void* half, gmg_stream s) {
  return checkerboard(dims, cb, per_site, prec, full, half, 1, s, "gmg_pick_checkerboard");
}

extern "C" gmg_status gmg_set_checkerboard(const int dims[4], int cb, int per_site, gmg_prec prec, const void* half,
                                           void* full, gmg_stream s) {
  return checkerboard(dims, cb, per_site, prec, half, full, 0, s, "gmg_set_checkerboard");
}

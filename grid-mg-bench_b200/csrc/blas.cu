// blas.cu -- per-RHS vector kernels for the multigrid solvers.
//
// Fields are [site][rhs][dof] complex (FP64 or FP32).  Every operation acts on
// each right-hand side separately (per-RHS scalars live on the device), which
// is what the reference's solvers do one field at a time (Grid's innerProduct,
// norm2, axpy used by its GMRES / FGMRES / MR, selected at include/Helpers.h:314-341).
// Reductions accumulate in FP64 whatever the field precision.
#include <algorithm>
#include <type_traits>

#include <cuda_bf16.h>

#include "mg_internal.cuh"

namespace gmg {
namespace blas {

template <class T> struct C2;
template <> struct C2<double> { typedef double2 t; };
template <> struct C2<float> { typedef float2 t; };

static int grid1(int64_t n) { return (int)std::min<int64_t>(std::max<int64_t>((n + 255) / 256, 1), 148 * 16); }

// The RHS index of element e of a [V][R][dof] field along a grid-stride loop,
// without a 64-bit division per element: q = e mod (R dof) advances by the
// stride modulo R dof, and r = q / dof is a multiply-high by ceil(2^32 / dof)
// (exact for q < 2^32 / dof, far above R dof here).
struct RhsWalk {
  int64_t e;
  uint32_t q, rd, dq, m;
  __device__ __forceinline__ RhsWalk(int64_t e0, int64_t stride, int R, int dof)
      : e(e0), rd((uint32_t)R * (uint32_t)dof) {
    q = (uint32_t)(e0 % rd);
    dq = (uint32_t)(stride % rd);
    m = 0xFFFFFFFFu / (uint32_t)dof + 1u;
  }
  __device__ __forceinline__ int r() const { return (int)__umulhi(q, m); }
  __device__ __forceinline__ void next(int64_t stride) {
    e += stride;
    q += dq;
    if (q >= rd) q -= rd;
  }
};

// out[(j0+j)*R + r] += sum_s <X_{j0+j}(s, r), Y(s, r)> for j < min(JB, nx - j0)
// (X_j = X + j*xstride).  Grid (gx, R): blockIdx.y is the RHS, threads walk the
// sites, then a warp-shuffle + shared-memory reduction and one FP64 atomic per
// (block, j).  Converged RHS (mask[r] == 0) are skipped.
template <class T, int JB>
__global__ void __launch_bounds__(256) multidot_kernel(const typename C2<T>::t* __restrict__ X, int64_t xstride,
                                                       int j0, int nx, const typename C2<T>::t* __restrict__ Y,
                                                       int64_t V, int R, int dof, double2* __restrict__ out,
                                                       const int* __restrict__ mask) {
  const int r = blockIdx.y;
  if (mask && !mask[r]) return;
  const int nj = min(JB, nx - j0);
  double ar[JB], ai[JB];
#pragma unroll
  for (int j = 0; j < JB; ++j) ar[j] = ai[j] = 0.0;
  for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < V; s += (int64_t)gridDim.x * blockDim.x) {
    const int64_t e = (s * R + r) * dof;
    for (int a = 0; a < dof; ++a) {
      const double yr = Y[e + a].x, yi = Y[e + a].y;
#pragma unroll
      for (int j = 0; j < JB; ++j) {
        if (j < nj) {
          const typename C2<T>::t x = X[(int64_t)(j0 + j) * xstride + e + a];
          ar[j] += (double)x.x * yr + (double)x.y * yi;
          ai[j] += (double)x.x * yi - (double)x.y * yr;
        }
      }
    }
  }
  __shared__ double sr[JB][8], si[JB][8];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int j = 0; j < JB; ++j) {
    double vr = ar[j], vi = ai[j];
    for (int o = 16; o > 0; o >>= 1) {
      vr += __shfl_xor_sync(0xffffffffu, vr, o);
      vi += __shfl_xor_sync(0xffffffffu, vi, o);
    }
    if (lane == 0) { sr[j][w] = vr; si[j][w] = vi; }
  }
  __syncthreads();
  if (threadIdx.x < nj) {
    double vr = 0, vi = 0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) { vr += sr[threadIdx.x][k]; vi += si[threadIdx.x][k]; }
    atomicAdd(&out[(j0 + threadIdx.x) * R + r].x, vr);
    atomicAdd(&out[(j0 + threadIdx.x) * R + r].y, vi);
  }
}

// Y(s, r) += sum_j a[j*R + r] X_j(s, r)   (a complex, FP64; X and Y may differ in precision)
template <class TX, class T>
__global__ void multiaxpy_kernel(const double2* __restrict__ a, const typename C2<TX>::t* __restrict__ X,
                                 int64_t xstride, int nx, typename C2<T>::t* __restrict__ Y, int64_t V, int R,
                                 int dof, double sgn) {
  const int64_t n = V * R * dof;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (RhsWalk w(blockIdx.x * (int64_t)blockDim.x + threadIdx.x, stride, R, dof); w.e < n; w.next(stride)) {
    const int64_t e = w.e;
    const int r = w.r();
    double yr = Y[e].x, yi = Y[e].y;
    for (int j = 0; j < nx; ++j) {
      double2 c = a[j * R + r];
      c.x *= sgn;
      c.y *= sgn;
      if (c.x == 0.0 && c.y == 0.0) continue;
      const typename C2<TX>::t x = X[j * xstride + e];
      yr += c.x * x.x - c.y * x.y;
      yi += c.x * x.y + c.y * x.x;
    }
    Y[e].x = (T)yr;
    Y[e].y = (T)yi;
  }
}

// Y(s, r) = a[r] * X(s, r) + b[r] * Y(s, r)
template <class T>
__global__ void axpby_kernel(const double2* __restrict__ a, const typename C2<T>::t* __restrict__ X,
                             const double2* __restrict__ b, typename C2<T>::t* __restrict__ Y, int64_t V, int R,
                             int dof) {
  const int64_t n = V * R * dof;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (RhsWalk w(blockIdx.x * (int64_t)blockDim.x + threadIdx.x, stride, R, dof); w.e < n; w.next(stride)) {
    const int64_t e = w.e;
    const int r = w.r();
    const double2 ca = a[r], cb = b[r];
    const typename C2<T>::t x = X[e], y = Y[e];
    const double re = ca.x * x.x - ca.y * x.y + cb.x * y.x - cb.y * y.y;
    const double im = ca.x * x.y + ca.y * x.x + cb.x * y.y + cb.y * y.x;
    Y[e].x = (T)re;
    Y[e].y = (T)im;
  }
}

template <class Ti, class To>
__global__ void convert_kernel(const typename C2<Ti>::t* __restrict__ X, typename C2<To>::t* __restrict__ Y, int64_t n) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    Y[e].x = (To)X[e].x;
    Y[e].y = (To)X[e].y;
  }
}

// Chirally doubled basis from a batch of nb vectors X [V][nb][dof]:
// B[n] = f (1 + G5) X_n and B[n + nb] = f (1 - G5) X_n with G5 = +1 on the
// upper half of the site's dof and -1 on the lower half (gamma5 =
// diag(1,1,-1,-1) on spin-colour, G5C on coarse vectors): 2 f X_n on one half,
// zero on the other.  f = 1/2 is performChiralDoublingG5C
// (include/Benchmark_helpers.h:156-181), f = 1 the G5R5 form (:130-154); the
// setup uses f = 1/2 (any factor is removed by the block orthonormalisation
// that follows).
template <class T>
__global__ void chiral_double_kernel(const typename C2<T>::t* __restrict__ X, double2* __restrict__ B, int64_t V,
                                     int nb, int dof, double f) {
  const int64_t n = V * nb * dof;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    const int a = (int)(e % dof);
    const int k = (int)((e / dof) % nb);
    const int64_t s = e / ((int64_t)dof * nb);
    const double m = 2.0 * f;
    const double2 v = make_double2(m * (double)X[e].x, m * (double)X[e].y);
    const double2 z = make_double2(0, 0);
    const bool upper = a < dof / 2;
    B[((int64_t)k * V + s) * dof + a] = upper ? v : z;
    B[((int64_t)(k + nb) * V + s) * dof + a] = upper ? z : v;
  }
}

// ---------------------------------------------------------------------------
// Row geometry.  A field row is one site: R * dof contiguous complex numbers.
// With RD = R * dof <= 1024, a block of spb * RD threads takes spb sites per
// step and every thread owns one fixed (rhs, dof) slot of the row, so the
// block's loads and stores are contiguous, the RHS index of a thread is
// computed once, and per-RHS sums reduce inside the block.
// ---------------------------------------------------------------------------
struct Row {
  int RD, spb, threads, grid;
};

static Row row_geom(int64_t V, int R, int dof) {
  Row g;
  g.RD = R * dof;
  g.spb = g.RD <= 256 ? std::max(1, 256 / g.RD) : 1;
  g.threads = (g.spb * g.RD + 31) / 32 * 32;
  g.grid = (int)std::max<int64_t>(1, std::min<int64_t>((V + g.spb - 1) / g.spb, 148 * 16));
  return g;
}

// out[(j0+j)*R + r] += sum_s <X_{j0+j}(s, r), Y(s, r)>, j < min(JB, nx - j0).
// Per-thread partial sums go to shared memory; then one thread per (j, r) adds
// the partials of the spb * dof threads that own RHS r (no shared-memory
// atomics: with few RHS every thread would hit the same address) and issues one
// global FP64 atomic per (block, j, r).
template <class T, int JB>
__global__ void __launch_bounds__(1024) multidot_row_kernel(const typename C2<T>::t* __restrict__ X, int64_t xstride,
                                                            int j0, int nx, const typename C2<T>::t* __restrict__ Y,
                                                            int64_t V, int R, int dof, int spb,
                                                            double2* __restrict__ out, const int* __restrict__ mask) {
  extern __shared__ double part[];  // [JB][2][blockDim]
  const int RD = R * dof, t = threadIdx.x, NT = blockDim.x;
  const int so = t / RD, i = t % RD, r = i / dof;
  const bool act = t < spb * RD && !(mask && !mask[r]);
  const int nj = min(JB, nx - j0);
  double ar[JB], ai[JB];
#pragma unroll
  for (int j = 0; j < JB; ++j) ar[j] = ai[j] = 0.0;
  if (act && sizeof(T) == 8) {
    for (int64_t s = (int64_t)blockIdx.x * spb + so; s < V; s += (int64_t)gridDim.x * spb) {
      const int64_t e = s * RD + i;
      const double yr = Y[e].x, yi = Y[e].y;
#pragma unroll
      for (int j = 0; j < JB; ++j) {
        if (j < nj) {
          const typename C2<T>::t x = X[(int64_t)(j0 + j) * xstride + e];
          ar[j] += (double)x.x * yr + (double)x.y * yi;
          ai[j] += (double)x.x * yi - (double)x.y * yr;
        }
      }
    }
  } else if (act) {
    // FP32: two sites per round, their loads issued together (short vectors on
    // the coarse levels give a thread a few dozen sites, each an L2 round trip)
    const int64_t step = (int64_t)gridDim.x * spb;
    for (int64_t s = (int64_t)blockIdx.x * spb + so; s < V; s += 2 * step) {
      const bool two = s + step < V;
      const int64_t e0 = s * RD + i, e1 = two ? (s + step) * RD + i : e0;
      const typename C2<T>::t y0 = Y[e0], y1 = Y[e1];
      typename C2<T>::t x0[JB], x1[JB];
#pragma unroll
      for (int j = 0; j < JB; ++j)
        if (j < nj) {
          x0[j] = X[(int64_t)(j0 + j) * xstride + e0];
          x1[j] = X[(int64_t)(j0 + j) * xstride + e1];
        }
#pragma unroll
      for (int j = 0; j < JB; ++j) {
        if (j < nj) {
          ar[j] += (double)x0[j].x * y0.x + (double)x0[j].y * y0.y;
          ai[j] += (double)x0[j].x * y0.y - (double)x0[j].y * y0.x;
          if (two) {
            ar[j] += (double)x1[j].x * y1.x + (double)x1[j].y * y1.y;
            ai[j] += (double)x1[j].x * y1.y - (double)x1[j].y * y1.x;
          }
        }
      }
    }
  }
#pragma unroll
  for (int j = 0; j < JB; ++j) {
    part[(2 * j) * NT + t] = ar[j];
    part[(2 * j + 1) * NT + t] = ai[j];
  }
  __syncthreads();
  // stage 1: fold the spb site slots onto slot 0, one (j, re/im, rhs-dof) per thread
  if (spb > 1) {
    for (int k = t; k < 2 * nj * RD; k += NT) {
      const int jc = k / RD, ii = k % RD;
      double v = part[jc * NT + ii];
      for (int o = 1; o < spb; ++o) v += part[jc * NT + o * RD + ii];
      part[jc * NT + ii] = v;
    }
    __syncthreads();
  }
  // stage 2: fold the dof components of each rhs
  for (int k = t; k < nj * R; k += NT) {
    const int j = k / R, rr = k % R;
    double vr = 0.0, vi = 0.0;
    for (int a = 0; a < dof; ++a) {
      vr += part[(2 * j) * NT + rr * dof + a];
      vi += part[(2 * j + 1) * NT + rr * dof + a];
    }
    atomicAdd(&out[(j0 + j) * R + rr].x, vr);
    atomicAdd(&out[(j0 + j) * R + rr].y, vi);
  }
}

// Y(s, r) += sgn * sum_j a[j*R + r] X_j(s, r), coefficients staged in shared memory
template <class TX, class T>
__global__ void __launch_bounds__(1024) multiaxpy_row_kernel(const double2* __restrict__ a,
                                                             const typename C2<TX>::t* __restrict__ X,
                                                             int64_t xstride, int nx, typename C2<T>::t* __restrict__ Y,
                                                             int64_t V, int R, int dof, int spb, double sgn) {
  extern __shared__ double2 cf[];  // [nx][R]
  const int RD = R * dof, t = threadIdx.x;
  const int so = t / RD, i = t % RD, r = i / dof;
  for (int k = t; k < nx * R; k += blockDim.x) cf[k] = make_double2(sgn * a[k].x, sgn * a[k].y);
  __syncthreads();
  if (t >= spb * RD) return;
  for (int64_t s = (int64_t)blockIdx.x * spb + so; s < V; s += (int64_t)gridDim.x * spb) {
    const int64_t e = s * RD + i;
    double yr = Y[e].x, yi = Y[e].y;
    for (int j = 0; j < nx; ++j) {
      const double2 c = cf[j * R + r];
      const typename C2<TX>::t x = X[j * xstride + e];
      yr += c.x * x.x - c.y * x.y;
      yi += c.x * x.y + c.y * x.x;
    }
    Y[e].x = (T)yr;
    Y[e].y = (T)yi;
  }
}

// Y(s, r) += sgn * sum_j a[j*R + r] X_j(s, r) and, in the same sweep over the
// updated Y, MODE 1: out[j*R + r] += <X_j(r), Y(r)> for j < nx (the next
// Gram-Schmidt pass's coefficients), MODE 2: out[r] += <Y(r), Y(r)> (the norm
// of the new Krylov vector).  nx <= kAxDotMaxJ (every restart length the MG
// levels use); MODE 1 keeps a site's X_j values in registers between the
// update and the products, so it runs at most kAxDot1Threads threads per block
// (MODE 2 needs no X after the update and runs up to kAxDotThreads).
constexpr int kAxDotMaxJ = 10;
constexpr int kAxDotThreads = 768;
constexpr int kAxDot1Threads = 384;

template <class TX, class T, int MODE, int MJ = kAxDotMaxJ>
__global__ void __launch_bounds__(MODE == 1 ? kAxDot1Threads : kAxDotThreads) multiaxpy_dot_row_kernel(const double2* __restrict__ a,
                                                                 const typename C2<TX>::t* __restrict__ X,
                                                                 int64_t xstride, int nx,
                                                                 typename C2<T>::t* __restrict__ Y, int64_t V, int R,
                                                                 int dof, int spb, double sgn,
                                                                 double2* __restrict__ out) {
  extern __shared__ double2 smd[];
  double2* cf = smd;                                        // [nx][R]
  double* part = reinterpret_cast<double*>(smd + kAxDotMaxJ * R);  // [8][NT]
  const int RD = R * dof, t = threadIdx.x, NT = blockDim.x;
  const int so = t / RD, i = t % RD, r = i / dof;
  for (int k = t; k < nx * R; k += NT) cf[k] = make_double2(sgn * a[k].x, sgn * a[k].y);
  __syncthreads();
  const bool act = t < spb * RD;
  double ar[MODE == 1 ? MJ : 1], ai[MODE == 1 ? MJ : 1];
#pragma unroll
  for (int j = 0; j < (MODE == 1 ? MJ : 1); ++j) ar[j] = ai[j] = 0.0;
  if (act) {
    for (int64_t s = (int64_t)blockIdx.x * spb + so; s < V; s += (int64_t)gridDim.x * spb) {
      const int64_t e = s * RD + i;
      double yr = Y[e].x, yi = Y[e].y;
      if (MODE == 1) {
        // MODE 1 is instantiated for the exact basis count (MJ == nx): the
        // loads carry no guard and all issue before the first use
        typename C2<TX>::t xv[MJ];
#pragma unroll
        for (int j = 0; j < MJ; ++j) xv[j] = X[j * xstride + e];
#pragma unroll
        for (int j = 0; j < MJ; ++j) {
          const double2 c = cf[j * R + r];
          yr += c.x * xv[j].x - c.y * xv[j].y;
          yi += c.x * xv[j].y + c.y * xv[j].x;
        }
#pragma unroll
        for (int j = 0; j < MJ; ++j) {
          ar[j] += xv[j].x * yr + xv[j].y * yi;
          ai[j] += xv[j].x * yi - xv[j].y * yr;
        }
      } else {
        for (int j = 0; j < nx; ++j) {
          const typename C2<TX>::t x = X[j * xstride + e];
          const double2 c = cf[j * R + r];
          yr += c.x * x.x - c.y * x.y;
          yi += c.x * x.y + c.y * x.x;
        }
      }
      Y[e].x = (T)yr;
      Y[e].y = (T)yi;
      if (MODE == 1) {
      } else {
        ar[0] += yr * yr + yi * yi;
      }
    }
  }
  // block reduction in chunks of 4 products: fold the spb site slots, then the
  // dof components of each RHS, then one global atomic per (j, r) and block
  const int nprod = MODE == 1 ? nx : 1;
#pragma unroll
  for (int j0 = 0; j0 < (MODE == 1 ? MJ : 1); j0 += 4) {
    if (j0 >= nprod) break;
    const int nj = min(4, nprod - j0);
    __syncthreads();
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int j = j0 + q;
      double vr = 0.0, vi = 0.0;
#pragma unroll
      for (int jj = 0; jj < (MODE == 1 ? MJ : 1); ++jj)
        if (jj == j) {
          vr = ar[jj];
          vi = ai[jj];
        }
      part[(2 * q) * NT + t] = act ? vr : 0.0;
      part[(2 * q + 1) * NT + t] = act ? vi : 0.0;
    }
    __syncthreads();
    if (spb > 1) {
      for (int k = t; k < 2 * nj * RD; k += NT) {
        const int jc = k / RD, ii = k % RD;
        double v = part[jc * NT + ii];
        for (int o = 1; o < spb; ++o) v += part[jc * NT + o * RD + ii];
        part[jc * NT + ii] = v;
      }
      __syncthreads();
    }
    for (int k = t; k < nj * R; k += NT) {
      const int q = k / R, rr = k % R;
      double vr = 0.0, vi = 0.0;
      for (int d = 0; d < dof; ++d) {
        vr += part[(2 * q) * NT + rr * dof + d];
        vi += part[(2 * q + 1) * NT + rr * dof + d];
      }
      atomicAdd(&out[(j0 + q) * R + rr].x, vr);
      if (MODE == 1) atomicAdd(&out[(j0 + q) * R + rr].y, vi);
    }
  }
}

// Delayed-reorthogonalisation Gram-Schmidt (DCGS2): vectors stored as T
// (FP64, or FP32 for an FP32 Arnoldi cycle), products and updates formed in
// FP64.  V_0 .. V_{NV-1}
// are the finished basis vectors, A = V_NV the last one after one projection
// (its second projection delayed to this step), B the new operator product.
// Pass 1 (one sweep): out[k * R + r] for k < NV: <V_k, A>; NV <= k < 2 NV:
// <V_{k-NV}, B>; 2 NV: <A, A>; 2 NV + 1: <A, B>; 2 NV + 2: <B, B>.
constexpr int kDcgsThreads = 384;
constexpr int kDcgsMaxNV = 9;

// Two consecutive complex numbers of a field (one 16-byte load FP32, two
// FP64), kept in the storage type until used; e is even and the field 16-byte
// aligned.
__device__ __forceinline__ void ld_pair(const float2* p, int64_t e, float2& u, float2& v) {
  const float4 q = *reinterpret_cast<const float4*>(p + e);
  u = make_float2(q.x, q.y);
  v = make_float2(q.z, q.w);
}
__device__ __forceinline__ void ld_pair(const double2* p, int64_t e, double2& u, double2& v) {
  u = p[e];
  v = p[e + 1];
}
template <class C>
__device__ __forceinline__ double2 wide(C a) { return make_double2(a.x, a.y); }
// an empty statement that reads and (as far as the compiler knows) rewrites
// v: applied to a batch of loaded values in turn, after the batch's loads, it
// keeps every use of the batch after every load of the batch has been issued
__device__ __forceinline__ void issued(float2& v) { asm volatile("" : "+f"(v.x), "+f"(v.y)); }
__device__ __forceinline__ void issued(double2& v) { asm volatile("" : "+d"(v.x), "+d"(v.y)); }
__device__ __forceinline__ void st_pair(float2* p, int64_t e, double ur, double ui, double vr, double vi) {
  *reinterpret_cast<float4*>(p + e) = make_float4((float)ur, (float)ui, (float)vr, (float)vi);
}
__device__ __forceinline__ void st_pair(double2* p, int64_t e, double ur, double ui, double vr, double vi) {
  p[e] = make_double2(ur, ui);
  p[e + 1] = make_double2(vr, vi);
}

// A thread takes two consecutive complex numbers of a site's R x dof row (dof
// even, so both belong to one RHS): twice the bytes in flight per thread for
// the same product accumulators, which bound the kernels' occupancy.
template <int NV, class T = double>
__global__ void __launch_bounds__(kDcgsThreads) dcgs_dots_row_kernel(const typename C2<T>::t* __restrict__ V0,
                                                                     int64_t vstride,
                                                                     const typename C2<T>::t* __restrict__ B, int64_t V,
                                                                     int R, int dof, int spb,
                                                                     double2* __restrict__ out) {
  extern __shared__ double part[];  // [8][NT]
  constexpr int NP = 2 * NV + 3;
  const int RD = R * dof, RH = RD / 2, dh = dof / 2, t = threadIdx.x, NT = blockDim.x;
  const int so = t / RH, i = t % RH;
  const bool act = t < spb * RH;
  double pr[NP], pi[NP];
#pragma unroll
  for (int k = 0; k < NP; ++k) pr[k] = pi[k] = 0.0;
  if (act) {
#pragma unroll 1
    for (int64_t st = (int64_t)blockIdx.x * spb + so; st < V; st += (int64_t)gridDim.x * spb) {
      const int64_t e = st * RD + 2 * i;
      typename C2<T>::t xv[NV + 1][2], bv[2];
#pragma unroll
      for (int k = 0; k <= NV; ++k) ld_pair(V0 + k * vstride, e, xv[k][0], xv[k][1]);
      ld_pair(B, e, bv[0], bv[1]);
#pragma unroll
      for (int k = 0; k <= NV; ++k) {
        issued(xv[k][0]);
        issued(xv[k][1]);
      }
      issued(bv[0]);
      issued(bv[1]);
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const double2 a = wide(xv[NV][h]), b = wide(bv[h]);
#pragma unroll
        for (int k = 0; k < NV; ++k) {
          const double2 x = wide(xv[k][h]);
          pr[k] += x.x * a.x + x.y * a.y;
          pi[k] += x.x * a.y - x.y * a.x;
          pr[NV + k] += x.x * b.x + x.y * b.y;
          pi[NV + k] += x.x * b.y - x.y * b.x;
        }
        pr[2 * NV] += a.x * a.x + a.y * a.y;
        pr[2 * NV + 1] += a.x * b.x + a.y * b.y;
        pi[2 * NV + 1] += a.x * b.y - a.y * b.x;
        pr[2 * NV + 2] += b.x * b.x + b.y * b.y;
      }
    }
  }
  // block reduction, four products at a time: the spb site slots, then the
  // dof / 2 pairs of each RHS, then one global atomic per (product, RHS)
#pragma unroll
  for (int k0 = 0; k0 < NP; k0 += 4) {
    const int nk = min(4, NP - k0);
    __syncthreads();
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      double vr = 0.0, vi = 0.0;
#pragma unroll
      for (int k = 0; k < NP; ++k)
        if (k == k0 + q) {
          vr = pr[k];
          vi = pi[k];
        }
      part[(2 * q) * NT + t] = act ? vr : 0.0;
      part[(2 * q + 1) * NT + t] = act ? vi : 0.0;
    }
    __syncthreads();
    if (spb > 1) {
      for (int k = t; k < 2 * nk * RH; k += NT) {
        const int jc = k / RH, ii = k % RH;
        double v = part[jc * NT + ii];
        for (int o = 1; o < spb; ++o) v += part[jc * NT + o * RH + ii];
        part[jc * NT + ii] = v;
      }
      __syncthreads();
    }
    for (int k = t; k < nk * R; k += NT) {
      const int q = k / R, rr = k % R;
      double vr = 0.0, vi = 0.0;
      for (int d = 0; d < dh; ++d) {
        vr += part[(2 * q) * NT + rr * dh + d];
        vi += part[(2 * q + 1) * NT + rr * dh + d];
      }
      atomicAdd(&out[(k0 + q) * R + rr].x, vr);
      atomicAdd(&out[(k0 + q) * R + rr].y, vi);
    }
  }
}

// Pass 2 (one sweep): A <- (A - sum_k c_k V_k) / alpha (the finished basis
// vector, in place), then V_{NV+1} <- (B - sum_k g_k V_k - d A) / beta (the
// next one after one projection).  cf per RHS: c[NV], g[NV], (1/alpha, 0),
// d, (1/beta, 0), at cf[k * R + r].  Two complex numbers per thread.
template <int NV, class T = double>
__global__ void __launch_bounds__(kDcgsThreads) dcgs_update_row_kernel(const double2* __restrict__ cfg,
                                                                       typename C2<T>::t* __restrict__ V0,
                                                                       int64_t vstride,
                                                                       const typename C2<T>::t* __restrict__ B,
                                                                       int64_t V, int R, int dof, int spb) {
  extern __shared__ double2 cf[];  // [2 NV + 3][R]
  constexpr int NC = 2 * NV + 3;
  const int RD = R * dof, RH = RD / 2, t = threadIdx.x;
  for (int k = t; k < NC * R; k += blockDim.x) cf[k] = cfg[k];
  __syncthreads();
  if (t >= spb * RH) return;
  const int so = t / RH, i = t % RH, r = (2 * i) / dof;
  const double ia = cf[(2 * NV) * R + r].x;
  const double2 d = cf[(2 * NV + 1) * R + r];
  const double ib = cf[(2 * NV + 2) * R + r].x;
  for (int64_t st = (int64_t)blockIdx.x * spb + so; st < V; st += (int64_t)gridDim.x * spb) {
    const int64_t e = st * RD + 2 * i;
    typename C2<T>::t xv[NV + 1][2], bv[2];
#pragma unroll
    for (int k = 0; k <= NV; ++k) ld_pair(V0 + k * vstride, e, xv[k][0], xv[k][1]);
    ld_pair(B, e, bv[0], bv[1]);
#pragma unroll
    for (int k = 0; k <= NV; ++k) {
      issued(xv[k][0]);
      issued(xv[k][1]);
    }
    issued(bv[0]);
    issued(bv[1]);
    double o[2][4];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      double ar = xv[NV][h].x, ai = xv[NV][h].y, br = bv[h].x, bi = bv[h].y;
#pragma unroll
      for (int k = 0; k < NV; ++k) {
        const double2 c = cf[k * R + r], g = cf[(NV + k) * R + r], x = wide(xv[k][h]);
        ar -= c.x * x.x - c.y * x.y;
        ai -= c.x * x.y + c.y * x.x;
        br -= g.x * x.x - g.y * x.y;
        bi -= g.x * x.y + g.y * x.x;
      }
      ar *= ia;
      ai *= ia;
      br -= d.x * ar - d.y * ai;
      bi -= d.x * ai + d.y * ar;
      o[h][0] = ar;
      o[h][1] = ai;
      o[h][2] = br * ib;
      o[h][3] = bi * ib;
    }
    st_pair(V0 + NV * vstride, e, o[0][0], o[0][1], o[1][0], o[1][1]);
    st_pair(V0 + (NV + 1) * vstride, e, o[0][2], o[0][3], o[1][2], o[1][3]);
  }
}

// Y(r) = X(r) / sqrt(n[r].x), X of type TX, Y of type T (FP64 -> FP32: the
// first Krylov vector of an FP32 Arnoldi cycle from the FP64 residual)
template <class T, class TX = T>
__global__ void __launch_bounds__(1024) scale_inv_norm_row_kernel(const double2* __restrict__ n,
                                                                  const typename C2<TX>::t* __restrict__ X,
                                                                  typename C2<T>::t* __restrict__ Y, int64_t V, int R,
                                                                  int dof, int spb) {
  const int RD = R * dof, t = threadIdx.x;
  if (t >= spb * RD) return;
  const int so = t / RD, i = t % RD, r = i / dof;
  const double nn = n[r].x;
  const double sc = nn > 0.0 ? rsqrt(nn) : 0.0;
  for (int64_t s = (int64_t)blockIdx.x * spb + so; s < V; s += (int64_t)gridDim.x * spb) {
    const int64_t e = s * RD + i;
    Y[e].x = (T)(sc * X[e].x);
    Y[e].y = (T)(sc * X[e].y);
  }
}

// MR step: alpha = <Ar, r> / <Ar, Ar>; x += alpha r, r -= alpha Ar
template <class T>
__global__ void __launch_bounds__(1024) mr_update_row_kernel(const double2* __restrict__ d1,
                                                             const double2* __restrict__ d2,
                                                             typename C2<T>::t* __restrict__ x,
                                                             typename C2<T>::t* __restrict__ rr_,
                                                             const typename C2<T>::t* __restrict__ Ar, int64_t V, int R,
                                                             int dof, int spb, bool update_r, double csg) {
  const int RD = R * dof, t = threadIdx.x;
  if (t >= spb * RD) return;
  const int so = t / RD, i = t % RD, k = i / dof;
  const double den = d2[k].x;
  const double ar = den > 0.0 ? d1[k].x / den : 0.0, ai = den > 0.0 ? csg * d1[k].y / den : 0.0;
  for (int64_t s = (int64_t)blockIdx.x * spb + so; s < V; s += (int64_t)gridDim.x * spb) {
    const int64_t e = s * RD + i;
    const double rr = rr_[e].x, ri = rr_[e].y;
    x[e].x = (T)(x[e].x + ar * rr - ai * ri);
    x[e].y = (T)(x[e].y + ar * ri + ai * rr);
    if (update_r) {
      const double qr = Ar[e].x, qi = Ar[e].y;
      rr_[e].x = (T)(rr - (ar * qr - ai * qi));
      rr_[e].y = (T)(ri - (ar * qi + ai * qr));
    }
  }
}

__device__ __forceinline__ float2 bf16w_to_f2(uint32_t w) {
  return make_float2(__uint_as_float(w << 16), __uint_as_float(w & 0xffff0000u));
}
__device__ __forceinline__ uint32_t f2_to_bf16w(float re, float im) {
  const __nv_bfloat162 b = __floats2bfloat162_rn(re, im);
  return *reinterpret_cast<const uint32_t*>(&b);
}

// the MR step on BF16 residual fields: x (FP32) += a r; r = bf16(r - a Ar)
__global__ void __launch_bounds__(1024) mr_update_bf16_row_kernel(const double2* __restrict__ d1,
                                                                  const double2* __restrict__ d2,
                                                                  float2* __restrict__ x, uint32_t* __restrict__ rr_,
                                                                  const uint32_t* __restrict__ Ar, int64_t V, int R,
                                                                  int dof, int spb, bool update_r) {
  const int RD = R * dof, t = threadIdx.x;
  if (t >= spb * RD) return;
  const int so = t / RD, i = t % RD, k = i / dof;
  const double den = d2[k].x;
  const float ar = den > 0.0 ? (float)(d1[k].x / den) : 0.f, ai = den > 0.0 ? (float)(d1[k].y / den) : 0.f;
  for (int64_t s = (int64_t)blockIdx.x * spb + so; s < V; s += (int64_t)gridDim.x * spb) {
    const int64_t e = s * RD + i;
    const float2 r = bf16w_to_f2(rr_[e]);
    float2 xv = x[e];
    xv.x += ar * r.x - ai * r.y;
    xv.y += ar * r.y + ai * r.x;
    x[e] = xv;
    if (update_r) {
      const float2 q = bf16w_to_f2(Ar[e]);
      rr_[e] = f2_to_bf16w(r.x - (ar * q.x - ai * q.y), r.y - (ar * q.y + ai * q.x));
    }
  }
}

// word i of a site's R x 12 block in the site-blocked BF16 layout [3][R][4]
// <-> (RHS, component) of the [R][12] layout
__device__ __forceinline__ int blocked_rhs(int i, int R) { return (i % (4 * R)) / 4; }
__device__ __forceinline__ int blocked_word(int r, int c, int R) { return (c / 4) * 4 * R + r * 4 + c % 4; }

// rn = bf16(r - a Ar): one MR step on residuals that the sweep keeps (fields
// [V][R][dof], or site-blocked [V][3][R][4] words with `blocked`, dof 12)
__global__ void __launch_bounds__(1024) mr_resid_bf16_row_kernel(const double2* __restrict__ d1,
                                                                 const double2* __restrict__ d2,
                                                                 const uint32_t* __restrict__ r,
                                                                 const uint32_t* __restrict__ Ar,
                                                                 uint32_t* __restrict__ rn, int64_t V, int R, int dof,
                                                                 int spb, bool blocked) {
  const int RD = R * dof, t = threadIdx.x;
  if (t >= spb * RD) return;
  const int so = t / RD, i = t % RD, k = blocked ? blocked_rhs(i, R) : i / dof;
  const double den = d2[k].x;
  const float ar = den > 0.0 ? (float)(d1[k].x / den) : 0.f, ai = den > 0.0 ? (float)(d1[k].y / den) : 0.f;
  for (int64_t s = (int64_t)blockIdx.x * spb + so; s < V; s += (int64_t)gridDim.x * spb) {
    const int64_t e = s * RD + i;
    const float2 v = bf16w_to_f2(r[e]), q = bf16w_to_f2(Ar[e]);
    rn[e] = f2_to_bf16w(v.x - (ar * q.x - ai * q.y), v.y - (ar * q.y + ai * q.x));
  }
}

// x += sum_j a_j r_j over the K kept residuals of an MR sweep: the solution is
// read and written once per sweep instead of once per step
// (K a template argument: the step lengths and the K loaded words stay in
// registers)
template <int K>
__global__ void __launch_bounds__(1024) mr_xsum_bf16_row_kernel(const double2* __restrict__ d, int dstride,
                                                                const uint32_t* __restrict__ r0, int64_t rstride,
                                                                float2* __restrict__ x, int64_t V, int R, int dof,
                                                                int spb, bool blocked) {
  const int RD = R * dof, t = threadIdx.x;
  if (t >= spb * RD) return;
  const int so = t / RD, i = t % RD, k = i / dof;
  const int ri = blocked ? blocked_word(k, i % dof, R) : i;  // the same (RHS, component) in the residuals
  float2 a[K];
#pragma unroll
  for (int j = 0; j < K; ++j) {
    a[j] = make_float2(0.f, 0.f);
    const double den = d[(int64_t)j * dstride + R + k].x;
    const double2 num = d[(int64_t)j * dstride + k];
    if (den > 0.0) a[j] = make_float2((float)(num.x / den), (float)(num.y / den));
  }
  for (int64_t s = (int64_t)blockIdx.x * spb + so; s < V; s += (int64_t)gridDim.x * spb) {
    const int64_t e = s * RD + i;
    uint32_t w[K];
#pragma unroll
    for (int j = 0; j < K; ++j) w[j] = __ldg(r0 + j * rstride + s * RD + ri);
    float2 acc = make_float2(0.f, 0.f);
#pragma unroll
    for (int j = 0; j < K; ++j) {
      const float2 v = bf16w_to_f2(w[j]);
      acc.x += a[j].x * v.x - a[j].y * v.y;
      acc.y += a[j].x * v.y + a[j].y * v.x;
    }
    float2 xv = x[e];
    xv.x += acc.x;
    xv.y += acc.y;
    x[e] = xv;
  }
}

// Z (BF16, site-blocked [V][3][R][4] words) = X - Y (FP32, [V][R][12])
__global__ void __launch_bounds__(1024) xmy_bf16_blocked_row_kernel(const float2* __restrict__ X,
                                                                    const float2* __restrict__ Y,
                                                                    uint32_t* __restrict__ Z, int64_t V, int R,
                                                                    int spb) {
  const int RD = R * 12, t = threadIdx.x;
  if (t >= spb * RD) return;
  const int so = t / RD, i = t % RD;
  const int src = blocked_rhs(i, R) * 12 + (i / (4 * R)) * 4 + i % 4;
  for (int64_t s = (int64_t)blockIdx.x * spb + so; s < V; s += (int64_t)gridDim.x * spb) {
    const float2 a = X[s * RD + src], b = Y[s * RD + src];
    Z[s * RD + i] = f2_to_bf16w(a.x - b.x, a.y - b.y);
  }
}

// The same two steps on site-blocked fields, one 16-byte quarter (four
// complex numbers of one RHS) per thread: a quarter of the threads and of the
// index arithmetic per element of the word-wise kernels.
// rn = bf16(r - a Ar), a = d1 / d2 per RHS
__global__ void __launch_bounds__(256) mr_resid_bf16_q_kernel(const double2* __restrict__ d1,
                                                              const double2* __restrict__ d2,
                                                              const uint4* __restrict__ r, const uint4* __restrict__ Ar,
                                                              uint4* __restrict__ rn, int64_t V, int R, int spb) {
  const int RQ = 3 * R, t = threadIdx.x;
  if (t >= spb * RQ) return;
  const int so = t / RQ, q = t % RQ, k = q % R;  // quarter q = g R + k of a site's block
  const double den = d2[k].x;
  const float ar = den > 0.0 ? (float)(d1[k].x / den) : 0.f, ai = den > 0.0 ? (float)(d1[k].y / den) : 0.f;
  for (int64_t s = (int64_t)blockIdx.x * spb + so; s < V; s += (int64_t)gridDim.x * spb) {
    const int64_t e = s * RQ + q;
    const uint4 u = r[e], v = Ar[e];
    const uint32_t uw[4] = {u.x, u.y, u.z, u.w}, vw[4] = {v.x, v.y, v.z, v.w};
    uint32_t o[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const float2 x = bf16w_to_f2(uw[j]), y = bf16w_to_f2(vw[j]);
      o[j] = f2_to_bf16w(x.x - (ar * y.x - ai * y.y), x.y - (ar * y.y + ai * y.x));
    }
    rn[e] = make_uint4(o[0], o[1], o[2], o[3]);
  }
}

// x (FP32 [V][R][12]) += sum_j a_j r_j, the r_j site-blocked; a thread takes
// components 4g .. 4g + 3 of RHS k (one quarter of every r_j, 32 bytes of x)
template <int K>
__global__ void __launch_bounds__(256) mr_xsum_bf16_q_kernel(const double2* __restrict__ d, int dstride,
                                                             const uint4* __restrict__ r0, int64_t rstride,
                                                             float4* __restrict__ x, int64_t V, int R, int spb) {
  const int RQ = 3 * R, t = threadIdx.x;
  if (t >= spb * RQ) return;
  const int so = t / RQ, q = t % RQ, k = q / 3, g = q % 3;
  float2 a[K];
#pragma unroll
  for (int j = 0; j < K; ++j) {
    a[j] = make_float2(0.f, 0.f);
    const double den = d[(int64_t)j * dstride + R + k].x;
    const double2 num = d[(int64_t)j * dstride + k];
    if (den > 0.0) a[j] = make_float2((float)(num.x / den), (float)(num.y / den));
  }
  const int rq = g * R + k;           // the quarter in the blocked layout
  const int xq = (k * 12 + 4 * g) / 2;  // the first float4 of x (two complex numbers each)
  for (int64_t s = (int64_t)blockIdx.x * spb + so; s < V; s += (int64_t)gridDim.x * spb) {
    uint4 w[K];
#pragma unroll
    for (int j = 0; j < K; ++j) w[j] = __ldg(r0 + j * rstride + s * RQ + rq);
    float2 acc[4] = {make_float2(0.f, 0.f), make_float2(0.f, 0.f), make_float2(0.f, 0.f), make_float2(0.f, 0.f)};
#pragma unroll
    for (int j = 0; j < K; ++j) {
      const uint32_t ww[4] = {w[j].x, w[j].y, w[j].z, w[j].w};
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        const float2 v = bf16w_to_f2(ww[c]);
        acc[c].x += a[j].x * v.x - a[j].y * v.y;
        acc[c].y += a[j].x * v.y + a[j].y * v.x;
      }
    }
    float4* xp = x + s * 6 * R + xq;
    float4 x0 = xp[0], x1 = xp[1];
    x0.x += acc[0].x;
    x0.y += acc[0].y;
    x0.z += acc[1].x;
    x0.w += acc[1].y;
    x1.x += acc[2].x;
    x1.y += acc[2].y;
    x1.z += acc[3].x;
    x1.w += acc[3].y;
    xp[0] = x0;
    xp[1] = x1;
  }
}

static Row quarter_geom(int64_t V, int R) {
  Row g;
  g.RD = 3 * R;
  g.spb = g.RD <= 256 ? std::max(1, 256 / g.RD) : 1;
  g.threads = (g.spb * g.RD + 31) / 32 * 32;
  g.grid = (int)std::max<int64_t>(1, std::min<int64_t>((V + g.spb - 1) / g.spb, 148 * 16));
  return g;
}

__global__ void xmy_bf16_kernel(const float2* __restrict__ X, const float2* __restrict__ Y, uint32_t* __restrict__ Z,
                                int64_t n) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    const float2 a = X[e], b = Y[e];
    Z[e] = f2_to_bf16w(a.x - b.x, a.y - b.y);
  }
}

// Y(r) = a[r] X(r) + b[r] Y(r)
template <class T>
__global__ void __launch_bounds__(1024) axpby_row_kernel(const double2* __restrict__ a,
                                                         const typename C2<T>::t* __restrict__ X,
                                                         const double2* __restrict__ b, typename C2<T>::t* __restrict__ Y,
                                                         int64_t V, int R, int dof, int spb) {
  const int RD = R * dof, t = threadIdx.x;
  if (t >= spb * RD) return;
  const int so = t / RD, i = t % RD, r = i / dof;
  const double2 ca = a[r], cb = b[r];
  for (int64_t s = (int64_t)blockIdx.x * spb + so; s < V; s += (int64_t)gridDim.x * spb) {
    const int64_t e = s * RD + i;
    const typename C2<T>::t x = X[e], y = Y[e];
    Y[e].x = (T)(ca.x * x.x - ca.y * x.y + cb.x * y.x - cb.y * y.y);
    Y[e].y = (T)(ca.x * x.y + ca.y * x.x + cb.x * y.y + cb.y * y.x);
  }
}

}  // namespace blas

// ---------------------------------------------------------------- host wrappers
gmg_status vec_multidot(const Vec& X0, int nx, int64_t xstride_elems, const Vec& Y, double2* out_dev, const int* mask,
                        cudaStream_t s) {
  GMG_CUDA(cudaMemsetAsync(out_dev, 0, sizeof(double2) * nx * Y.R, s));
  constexpr int JB = 4;
  if (Y.R * Y.dof <= 1024) {
    const blas::Row g = blas::row_geom(Y.V, Y.R, Y.dof);
    const size_t sm = sizeof(double) * 2 * JB * g.threads;
    if (sm > 48 * 1024) {
      GMG_CUDA(cudaFuncSetAttribute(blas::multidot_row_kernel<double, JB>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
      GMG_CUDA(cudaFuncSetAttribute(blas::multidot_row_kernel<float, JB>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    }
    // one resident wave of blocks: every block ends in nj * R global atomics on
    // the same nj * R addresses, so more blocks than fit at once only add
    // contention; and on short vectors (the coarse levels) no more blocks than
    // give each thread 32 sites, down to one per SM
    const int64_t by_len = std::max<int64_t>(148, Y.V / (32 * (int64_t)g.spb));
    const int grid = (int)std::min<int64_t>(std::min(g.grid, 148 * std::max(1, 2048 / g.threads)), by_len);
    for (int j0 = 0; j0 < nx; j0 += JB) {
      if (Y.prec == GMG_F64)
        blas::multidot_row_kernel<double, JB><<<grid, g.threads, sm, s>>>(
            (const double2*)X0.p, xstride_elems, j0, nx, (const double2*)Y.p, Y.V, Y.R, Y.dof, g.spb, out_dev, mask);
      else
        blas::multidot_row_kernel<float, JB><<<grid, g.threads, sm, s>>>(
            (const float2*)X0.p, xstride_elems, j0, nx, (const float2*)Y.p, Y.V, Y.R, Y.dof, g.spb, out_dev, mask);
      GMG_CUDA(cudaGetLastError());
    }
    return GMG_OK;
  }
  const int gx = (int)std::max<int64_t>(1, std::min<int64_t>((Y.V + 255) / 256, (148 * 8 + Y.R - 1) / Y.R));
  const dim3 grid(gx, Y.R);
  for (int j0 = 0; j0 < nx; j0 += JB) {
    if (Y.prec == GMG_F64)
      blas::multidot_kernel<double, JB><<<grid, 256, 0, s>>>((const double2*)X0.p, xstride_elems, j0, nx,
                                                             (const double2*)Y.p, Y.V, Y.R, Y.dof, out_dev, mask);
    else
      blas::multidot_kernel<float, JB><<<grid, 256, 0, s>>>((const float2*)X0.p, xstride_elems, j0, nx,
                                                            (const float2*)Y.p, Y.V, Y.R, Y.dof, out_dev, mask);
    GMG_CUDA(cudaGetLastError());
  }
  return GMG_OK;
}

gmg_status vec_multiaxpy(const double2* a_dev, const Vec& X0, int nx, int64_t xstride_elems, Vec& Y, cudaStream_t s,
                         double sgn) {
  if (Y.R * Y.dof <= 1024 && sizeof(double2) * (size_t)nx * Y.R <= 48 * 1024) {
    const blas::Row rg = blas::row_geom(Y.V, Y.R, Y.dof);
    const size_t sm = sizeof(double2) * (size_t)nx * Y.R;
    if (Y.prec == GMG_F64 && X0.prec == GMG_F64)
      blas::multiaxpy_row_kernel<double, double><<<rg.grid, rg.threads, sm, s>>>(
          a_dev, (const double2*)X0.p, xstride_elems, nx, (double2*)Y.p, Y.V, Y.R, Y.dof, rg.spb, sgn);
    else if (Y.prec == GMG_F64)
      blas::multiaxpy_row_kernel<float, double><<<rg.grid, rg.threads, sm, s>>>(
          a_dev, (const float2*)X0.p, xstride_elems, nx, (double2*)Y.p, Y.V, Y.R, Y.dof, rg.spb, sgn);
    else if (X0.prec == GMG_F32)
      blas::multiaxpy_row_kernel<float, float><<<rg.grid, rg.threads, sm, s>>>(
          a_dev, (const float2*)X0.p, xstride_elems, nx, (float2*)Y.p, Y.V, Y.R, Y.dof, rg.spb, sgn);
    else
      blas::multiaxpy_row_kernel<double, float><<<rg.grid, rg.threads, sm, s>>>(
          a_dev, (const double2*)X0.p, xstride_elems, nx, (float2*)Y.p, Y.V, Y.R, Y.dof, rg.spb, sgn);
    GMG_CUDA(cudaGetLastError());
    return GMG_OK;
  }
  const int g = blas::grid1(Y.elems());
  if (Y.prec == GMG_F64 && X0.prec == GMG_F64)
    blas::multiaxpy_kernel<double, double><<<g, 256, 0, s>>>(a_dev, (const double2*)X0.p, xstride_elems, nx,
                                                             (double2*)Y.p, Y.V, Y.R, Y.dof, sgn);
  else if (Y.prec == GMG_F64)
    blas::multiaxpy_kernel<float, double><<<g, 256, 0, s>>>(a_dev, (const float2*)X0.p, xstride_elems, nx,
                                                            (double2*)Y.p, Y.V, Y.R, Y.dof, sgn);
  else if (X0.prec == GMG_F32)
    blas::multiaxpy_kernel<float, float><<<g, 256, 0, s>>>(a_dev, (const float2*)X0.p, xstride_elems, nx,
                                                           (float2*)Y.p, Y.V, Y.R, Y.dof, sgn);
  else
    blas::multiaxpy_kernel<double, float><<<g, 256, 0, s>>>(a_dev, (const double2*)X0.p, xstride_elems, nx,
                                                            (float2*)Y.p, Y.V, Y.R, Y.dof, sgn);
  GMG_CUDA(cudaGetLastError());
  return GMG_OK;
}

gmg_status vec_axpby(const double2* a_dev, const Vec& X, const double2* b_dev, Vec& Y, cudaStream_t s) {
  if (Y.R * Y.dof <= 1024) {
    const blas::Row rg = blas::row_geom(Y.V, Y.R, Y.dof);
    if (Y.prec == GMG_F64)
      blas::axpby_row_kernel<double><<<rg.grid, rg.threads, 0, s>>>(a_dev, (const double2*)X.p, b_dev, (double2*)Y.p,
                                                                     Y.V, Y.R, Y.dof, rg.spb);
    else
      blas::axpby_row_kernel<float><<<rg.grid, rg.threads, 0, s>>>(a_dev, (const float2*)X.p, b_dev, (float2*)Y.p,
                                                                    Y.V, Y.R, Y.dof, rg.spb);
    GMG_CUDA(cudaGetLastError());
    return GMG_OK;
  }
  const int g = blas::grid1(Y.elems());
  if (Y.prec == GMG_F64)
    blas::axpby_kernel<double><<<g, 256, 0, s>>>(a_dev, (const double2*)X.p, b_dev, (double2*)Y.p, Y.V, Y.R, Y.dof);
  else
    blas::axpby_kernel<float><<<g, 256, 0, s>>>(a_dev, (const float2*)X.p, b_dev, (float2*)Y.p, Y.V, Y.R, Y.dof);
  GMG_CUDA(cudaGetLastError());
  return GMG_OK;
}

gmg_status vec_convert(const Vec& X, Vec& Y, cudaStream_t s) {
  GMG_CHECK(X.elems() == Y.elems(), GMG_ERR_SHAPE, "convert: size mismatch");
  const int64_t n = X.elems();
  const int g = blas::grid1(n);
  if (X.prec == Y.prec) {
    GMG_CUDA(cudaMemcpyAsync(Y.p, X.p, X.bytes(), cudaMemcpyDeviceToDevice, s));
    return GMG_OK;
  }
  if (X.prec == GMG_F64)
    blas::convert_kernel<double, float><<<g, 256, 0, s>>>((const double2*)X.p, (float2*)Y.p, n);
  else
    blas::convert_kernel<float, double><<<g, 256, 0, s>>>((const float2*)X.p, (double2*)Y.p, n);
  GMG_CUDA(cudaGetLastError());
  return GMG_OK;
}

namespace blas {

// dst[s][r'][a] = src[s][idx[r']][a]  (SCATTER: dst[s][idx[r']][a] = src[s][r'][a])
template <class T, bool SCATTER>
__global__ void permute_kernel(const typename C2<T>::t* __restrict__ src, typename C2<T>::t* __restrict__ dst,
                               const int* __restrict__ idx, int64_t V, int Rs, int Rd, int Rc, int dof) {
  const int64_t n = V * Rc * dof;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    const int a = (int)(e % dof);
    const int rc = (int)((e / dof) % Rc);
    const int64_t s = e / ((int64_t)dof * Rc);
    if (SCATTER) dst[(s * Rd + idx[rc]) * dof + a] = src[(s * Rs + rc) * dof + a];
    else dst[(s * Rd + rc) * dof + a] = src[(s * Rs + idx[rc]) * dof + a];
  }
}

// counter-based Gaussian: splitmix64 of (seed, element) -> Box-Muller
__device__ __forceinline__ uint64_t splitmix(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

template <class T>
__global__ void gaussian_kernel(typename C2<T>::t* __restrict__ X, int64_t n, uint64_t seed) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t h = splitmix(seed ^ splitmix((uint64_t)e));
    const double u1 = ((h >> 11) + 1.0) * (1.0 / 9007199254740993.0);  // (0, 1]
    const double u2 = (double)(splitmix(h) >> 11) * (1.0 / 9007199254740992.0);
    const double rad = sqrt(-log(u1));  // sqrt(-2 ln u1) * sqrt(1/2)
    double sn, cs;
    sincospi(2.0 * u2, &sn, &cs);
    X[e].x = (T)(rad * cs);
    X[e].y = (T)(rad * sn);
  }
}

// Y(r) = X(r) / sqrt(n[r].x)  (0 where n[r].x == 0); n holds <w, w> from a multidot
template <class T>
__global__ void scale_inv_norm_kernel(const double2* __restrict__ n, const typename C2<T>::t* __restrict__ X,
                                      typename C2<T>::t* __restrict__ Y, int64_t V, int R, int dof) {
  const int64_t tot = V * R * dof;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (RhsWalk w(blockIdx.x * (int64_t)blockDim.x + threadIdx.x, stride, R, dof); w.e < tot; w.next(stride)) {
    const int64_t e = w.e;
    const int r = w.r();
    const double nn = n[r].x;
    const double sc = nn > 0.0 ? rsqrt(nn) : 0.0;
    Y[e].x = (T)(sc * X[e].x);
    Y[e].y = (T)(sc * X[e].y);
  }
}

// minimal-residual step with per-RHS alpha = <Ar, r> / <Ar, Ar> read from the device
// (csg = -1: d1 holds the conjugate <r, Ar>): x += alpha r, r -= alpha Ar
template <class T>
__global__ void mr_update_kernel(const double2* __restrict__ d1, const double2* __restrict__ d2,
                                 typename C2<T>::t* __restrict__ x, typename C2<T>::t* __restrict__ r,
                                 const typename C2<T>::t* __restrict__ Ar, int64_t V, int R, int dof, bool update_r,
                                 double csg) {
  const int64_t tot = V * R * dof;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (RhsWalk w(blockIdx.x * (int64_t)blockDim.x + threadIdx.x, stride, R, dof); w.e < tot; w.next(stride)) {
    const int64_t e = w.e;
    const int k = w.r();
    const double den = d2[k].x;
    const double ar = den > 0.0 ? d1[k].x / den : 0.0, ai = den > 0.0 ? csg * d1[k].y / den : 0.0;
    const double rr = r[e].x, ri = r[e].y;
    x[e].x = (T)(x[e].x + ar * rr - ai * ri);
    x[e].y = (T)(x[e].y + ar * ri + ai * rr);
    if (update_r) {
      const double qr = Ar[e].x, qi = Ar[e].y;
      r[e].x = (T)(rr - (ar * qr - ai * qi));
      r[e].y = (T)(ri - (ar * qi + ai * qr));
    }
  }
}

// Y(r) = X(r) - Y(r)   (residual from b and A x)
template <class T>
__global__ void xmy_kernel(const typename C2<T>::t* __restrict__ X, typename C2<T>::t* __restrict__ Y, int64_t n) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    Y[e].x = X[e].x - Y[e].x;
    Y[e].y = X[e].y - Y[e].y;
  }
}

}  // namespace blas

gmg_status vec_scale_inv_norm(const double2* n_dev, const Vec& X, Vec& Y, cudaStream_t s) {
  if (X.prec != Y.prec) {
    GMG_CHECK(X.prec == GMG_F64 && Y.prec == GMG_F32 && Y.R * Y.dof <= 1024 && X.elems() == Y.elems(),
              GMG_ERR_UNSUPPORTED, "scale: mixed precision only FP64 -> FP32 with at most 1024 values per site");
    const blas::Row rg = blas::row_geom(Y.V, Y.R, Y.dof);
    blas::scale_inv_norm_row_kernel<float, double><<<rg.grid, rg.threads, 0, s>>>(
        n_dev, (const double2*)X.p, (float2*)Y.p, Y.V, Y.R, Y.dof, rg.spb);
    GMG_CUDA(cudaGetLastError());
    return GMG_OK;
  }
  if (Y.R * Y.dof <= 1024) {
    const blas::Row rg = blas::row_geom(Y.V, Y.R, Y.dof);
    if (Y.prec == GMG_F64)
      blas::scale_inv_norm_row_kernel<double><<<rg.grid, rg.threads, 0, s>>>(n_dev, (const double2*)X.p, (double2*)Y.p,
                                                                              Y.V, Y.R, Y.dof, rg.spb);
    else
      blas::scale_inv_norm_row_kernel<float><<<rg.grid, rg.threads, 0, s>>>(n_dev, (const float2*)X.p, (float2*)Y.p,
                                                                             Y.V, Y.R, Y.dof, rg.spb);
    GMG_CUDA(cudaGetLastError());
    return GMG_OK;
  }
  const int g = blas::grid1(Y.elems());
  if (Y.prec == GMG_F64)
    blas::scale_inv_norm_kernel<double><<<g, 256, 0, s>>>(n_dev, (const double2*)X.p, (double2*)Y.p, Y.V, Y.R, Y.dof);
  else
    blas::scale_inv_norm_kernel<float><<<g, 256, 0, s>>>(n_dev, (const float2*)X.p, (float2*)Y.p, Y.V, Y.R, Y.dof);
  GMG_CUDA(cudaGetLastError());
  return GMG_OK;
}

// Fused Gram-Schmidt sweep: Y += sgn * sum_j a_j X_j, then out = (mode 1)
// <X_j, Y> for j < nx, or (mode 2) <Y, Y>, both over the updated Y.  Falls back
// to separate passes where the fused kernel does not apply.
gmg_status vec_multiaxpy_dot(const double2* a_dev, const Vec& X0, int nx, int64_t xstride_elems, Vec& Y,
                             cudaStream_t s, double sgn, double2* out_dev, int mode) {
  const bool fused = nx <= blas::kAxDotMaxJ && X0.prec == Y.prec &&
                     Y.R * Y.dof <= (mode == 1 ? blas::kAxDot1Threads : blas::kAxDotThreads);
  if (!fused) {
    GMG_TRY(vec_multiaxpy(a_dev, X0, nx, xstride_elems, Y, s, sgn));
    return mode == 1 ? vec_multidot(X0, nx, xstride_elems, Y, out_dev, nullptr, s)
                     : vec_multidot(Y, 1, 0, Y, out_dev, nullptr, s);
  }
  GMG_CUDA(cudaMemsetAsync(out_dev, 0, sizeof(double2) * (mode == 1 ? nx : 1) * Y.R, s));
  const blas::Row g = blas::row_geom(Y.V, Y.R, Y.dof);
  const size_t sm = sizeof(double2) * blas::kAxDotMaxJ * Y.R + sizeof(double) * 8 * g.threads;
  const int grid = std::min(g.grid, 148 * std::max(1, 2048 / g.threads));
  auto launch = [&](auto kern, const auto* X, auto* Yp) -> gmg_status {
    if (sm > 48 * 1024) GMG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    kern<<<grid, g.threads, sm, s>>>(a_dev, X, xstride_elems, nx, Yp, Y.V, Y.R, Y.dof, g.spb, sgn, out_dev);
    GMG_CUDA(cudaGetLastError());
    return GMG_OK;
  };
  // mode 1 holds nx X values and 2 nx products per thread: one instantiation per nx
  auto run = [&](const auto* X, auto* Yp) -> gmg_status {
    typedef std::remove_const_t<std::remove_pointer_t<decltype(X)>> C;
    typedef std::conditional_t<std::is_same<C, double2>::value, double, float> Tb;
    if (mode == 2) return launch(blas::multiaxpy_dot_row_kernel<Tb, Tb, 2>, X, Yp);
    switch (nx) {
      case 1: return launch(blas::multiaxpy_dot_row_kernel<Tb, Tb, 1, 1>, X, Yp);
      case 2: return launch(blas::multiaxpy_dot_row_kernel<Tb, Tb, 1, 2>, X, Yp);
      case 3: return launch(blas::multiaxpy_dot_row_kernel<Tb, Tb, 1, 3>, X, Yp);
      case 4: return launch(blas::multiaxpy_dot_row_kernel<Tb, Tb, 1, 4>, X, Yp);
      case 5: return launch(blas::multiaxpy_dot_row_kernel<Tb, Tb, 1, 5>, X, Yp);
      case 6: return launch(blas::multiaxpy_dot_row_kernel<Tb, Tb, 1, 6>, X, Yp);
      case 7: return launch(blas::multiaxpy_dot_row_kernel<Tb, Tb, 1, 7>, X, Yp);
      case 8: return launch(blas::multiaxpy_dot_row_kernel<Tb, Tb, 1, 8>, X, Yp);
      case 9: return launch(blas::multiaxpy_dot_row_kernel<Tb, Tb, 1, 9>, X, Yp);
      default: return launch(blas::multiaxpy_dot_row_kernel<Tb, Tb, 1, 10>, X, Yp);
    }
  };
  if (Y.prec == GMG_F64) return run((const double2*)X0.p, (double2*)Y.p);
  return run((const float2*)X0.p, (float2*)Y.p);
}

gmg_status vec_mr_update(const double2* d1, const double2* d2, Vec& x, Vec& r, const Vec& Ar, cudaStream_t s,
                         bool update_r, bool conj_d1) {
  const double csg = conj_d1 ? -1.0 : 1.0;
  if (r.prec == GMG_BF16) {
    GMG_CHECK(x.prec == GMG_F32 && Ar.prec == GMG_BF16 && x.R * x.dof <= 1024 && !conj_d1, GMG_ERR_UNSUPPORTED,
              "mr update: BF16 residuals need an FP32 solution and at most 1024 values per site");
    const blas::Row rg = blas::row_geom(x.V, x.R, x.dof);
    blas::mr_update_bf16_row_kernel<<<rg.grid, rg.threads, 0, s>>>(d1, d2, (float2*)x.p, (uint32_t*)r.p,
                                                                  (const uint32_t*)Ar.p, x.V, x.R, x.dof, rg.spb,
                                                                  update_r);
    GMG_CUDA(cudaGetLastError());
    return GMG_OK;
  }
  if (x.R * x.dof <= 1024) {
    const blas::Row rg = blas::row_geom(x.V, x.R, x.dof);
    if (x.prec == GMG_F64)
      blas::mr_update_row_kernel<double><<<rg.grid, rg.threads, 0, s>>>(d1, d2, (double2*)x.p, (double2*)r.p,
                                                                         (const double2*)Ar.p, x.V, x.R, x.dof, rg.spb, update_r, csg);
    else
      blas::mr_update_row_kernel<float><<<rg.grid, rg.threads, 0, s>>>(d1, d2, (float2*)x.p, (float2*)r.p,
                                                                        (const float2*)Ar.p, x.V, x.R, x.dof, rg.spb, update_r, csg);
    GMG_CUDA(cudaGetLastError());
    return GMG_OK;
  }
  const int g = blas::grid1(x.elems());
  if (x.prec == GMG_F64)
    blas::mr_update_kernel<double><<<g, 256, 0, s>>>(d1, d2, (double2*)x.p, (double2*)r.p, (const double2*)Ar.p, x.V,
                                                     x.R, x.dof, update_r, csg);
  else
    blas::mr_update_kernel<float><<<g, 256, 0, s>>>(d1, d2, (float2*)x.p, (float2*)r.p, (const float2*)Ar.p, x.V, x.R,
                                                    x.dof, update_r, csg);
  GMG_CUDA(cudaGetLastError());
  return GMG_OK;
}

gmg_status vec_mr_resid_bf16(const double2* d1, const double2* d2, const Vec& r, const Vec& Ar, Vec& rn,
                             cudaStream_t s, bool blocked) {
  GMG_CHECK(r.prec == GMG_BF16 && Ar.prec == GMG_BF16 && rn.prec == GMG_BF16 && r.R * r.dof <= 1024 &&
                (!blocked || r.dof == 12),
            GMG_ERR_UNSUPPORTED, "mr residual: BF16 fields with at most 1024 values per site");
  if (blocked && 3 * r.R <= 256) {
    const blas::Row qg = blas::quarter_geom(r.V, r.R);
    blas::mr_resid_bf16_q_kernel<<<qg.grid, qg.threads, 0, s>>>(d1, d2, (const uint4*)r.p, (const uint4*)Ar.p,
                                                               (uint4*)rn.p, r.V, r.R, qg.spb);
    GMG_CUDA(cudaGetLastError());
    return GMG_OK;
  }
  const blas::Row rg = blas::row_geom(r.V, r.R, r.dof);
  blas::mr_resid_bf16_row_kernel<<<rg.grid, rg.threads, 0, s>>>(d1, d2, (const uint32_t*)r.p, (const uint32_t*)Ar.p,
                                                               (uint32_t*)rn.p, r.V, r.R, r.dof, rg.spb, blocked);
  GMG_CUDA(cudaGetLastError());
  return GMG_OK;
}

gmg_status vec_mr_xsum_bf16(const double2* d, int dstride, int K, const Vec& r0, int64_t rstride, Vec& x,
                            cudaStream_t s, bool blocked) {
  GMG_CHECK(r0.prec == GMG_BF16 && x.prec == GMG_F32 && K >= 1 && K <= kMrMaxSteps && x.R * x.dof <= 1024 &&
                (!blocked || x.dof == 12),
            GMG_ERR_UNSUPPORTED, "mr sum: BF16 residuals, an FP32 solution, 1 to 16 steps");
  if (blocked && 3 * x.R <= 256 && (((uintptr_t)x.p | (uintptr_t)r0.p) & 15) == 0 && rstride % 4 == 0) {
    const blas::Row qg = blas::quarter_geom(x.V, x.R);
    auto gq = [&](auto kern) {
      kern<<<qg.grid, qg.threads, 0, s>>>(d, dstride, (const uint4*)r0.p, rstride / 4, (float4*)x.p, x.V, x.R, qg.spb);
    };
    switch (K) {
      case 1: gq(blas::mr_xsum_bf16_q_kernel<1>); break;
      case 2: gq(blas::mr_xsum_bf16_q_kernel<2>); break;
      case 3: gq(blas::mr_xsum_bf16_q_kernel<3>); break;
      case 4: gq(blas::mr_xsum_bf16_q_kernel<4>); break;
      case 5: gq(blas::mr_xsum_bf16_q_kernel<5>); break;
      case 6: gq(blas::mr_xsum_bf16_q_kernel<6>); break;
      case 7: gq(blas::mr_xsum_bf16_q_kernel<7>); break;
      case 8: gq(blas::mr_xsum_bf16_q_kernel<8>); break;
      case 9: gq(blas::mr_xsum_bf16_q_kernel<9>); break;
      case 10: gq(blas::mr_xsum_bf16_q_kernel<10>); break;
      case 11: gq(blas::mr_xsum_bf16_q_kernel<11>); break;
      case 12: gq(blas::mr_xsum_bf16_q_kernel<12>); break;
      case 13: gq(blas::mr_xsum_bf16_q_kernel<13>); break;
      case 14: gq(blas::mr_xsum_bf16_q_kernel<14>); break;
      case 15: gq(blas::mr_xsum_bf16_q_kernel<15>); break;
      default: gq(blas::mr_xsum_bf16_q_kernel<16>); break;
    }
    GMG_CUDA(cudaGetLastError());
    return GMG_OK;
  }
  const blas::Row rg = blas::row_geom(x.V, x.R, x.dof);
  auto go = [&](auto kern) {
    kern<<<rg.grid, rg.threads, 0, s>>>(d, dstride, (const uint32_t*)r0.p, rstride, (float2*)x.p, x.V, x.R, x.dof,
                                        rg.spb, blocked);
  };
  switch (K) {
    case 1: go(blas::mr_xsum_bf16_row_kernel<1>); break;
    case 2: go(blas::mr_xsum_bf16_row_kernel<2>); break;
    case 3: go(blas::mr_xsum_bf16_row_kernel<3>); break;
    case 4: go(blas::mr_xsum_bf16_row_kernel<4>); break;
    case 5: go(blas::mr_xsum_bf16_row_kernel<5>); break;
    case 6: go(blas::mr_xsum_bf16_row_kernel<6>); break;
    case 7: go(blas::mr_xsum_bf16_row_kernel<7>); break;
    case 8: go(blas::mr_xsum_bf16_row_kernel<8>); break;
    case 9: go(blas::mr_xsum_bf16_row_kernel<9>); break;
    case 10: go(blas::mr_xsum_bf16_row_kernel<10>); break;
    case 11: go(blas::mr_xsum_bf16_row_kernel<11>); break;
    case 12: go(blas::mr_xsum_bf16_row_kernel<12>); break;
    case 13: go(blas::mr_xsum_bf16_row_kernel<13>); break;
    case 14: go(blas::mr_xsum_bf16_row_kernel<14>); break;
    case 15: go(blas::mr_xsum_bf16_row_kernel<15>); break;
    default: go(blas::mr_xsum_bf16_row_kernel<16>); break;
  }
  GMG_CUDA(cudaGetLastError());
  return GMG_OK;
}

gmg_status vec_xmy(const Vec& X, Vec& Y, cudaStream_t s) {
  const int64_t n = Y.elems();
  const int g = blas::grid1(n);
  if (Y.prec == GMG_F64) blas::xmy_kernel<double><<<g, 256, 0, s>>>((const double2*)X.p, (double2*)Y.p, n);
  else blas::xmy_kernel<float><<<g, 256, 0, s>>>((const float2*)X.p, (float2*)Y.p, n);
  GMG_CUDA(cudaGetLastError());
  return GMG_OK;
}

bool vec_dcgs_supported(const Vec& Y, int nv) {
  return (Y.prec == GMG_F64 || Y.prec == GMG_F32) && nv >= 0 && nv <= blas::kDcgsMaxNV && Y.dof % 2 == 0 &&
         Y.R * Y.dof / 2 <= blas::kDcgsThreads;
}

namespace {
// DCGS launch shape: R dof / 2 threads per site and the number of sites per
// CTA that keeps the most useful threads resident (the kernels hold many
// registers: their product accumulators or projection coefficients), one
// wave of CTAs.  smem_per_thread / smem_fixed: the kernel's dynamic shared memory.
template <class K>
blas::Row dcgs_geom(K kern, const Vec& B, size_t smem_per_thread, size_t smem_fixed, size_t* smem) {
  blas::Row g;
  g.RD = B.R * B.dof / 2;
  int best = -1;
  for (int spb = 1; spb * g.RD <= blas::kDcgsThreads; ++spb) {
    const int threads = (spb * g.RD + 31) / 32 * 32;
    const size_t sm = smem_per_thread * threads + smem_fixed;
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kern, threads, sm) != cudaSuccess) nb = 1;
    nb = std::max(nb, 1);
    if (nb * spb * g.RD > best) {
      best = nb * spb * g.RD;
      g.spb = spb;
      g.threads = threads;
      g.grid = (int)std::max<int64_t>(1, std::min<int64_t>((B.V + spb - 1) / spb, 148 * (int64_t)nb));
      *smem = sm;
    }
  }
  return g;
}
}  // namespace

gmg_status vec_dcgs_dots(const Vec& V0, int64_t vstride, int nv, const Vec& B, double2* out_dev, cudaStream_t s) {
  GMG_CHECK(vec_dcgs_supported(B, nv), GMG_ERR_UNSUPPORTED, "dcgs: unsupported shape");
  const int R = B.R;
  GMG_CUDA(cudaMemsetAsync(out_dev, 0, sizeof(double2) * (2 * nv + 3) * R, s));
  GMG_CHECK(V0.prec == B.prec, GMG_ERR_UNSUPPORTED, "dcgs: basis and new vector differ in precision");
  auto launch = [&](auto kern, auto* p) -> gmg_status {
    typedef std::remove_pointer_t<decltype(p)> CT;
    size_t sm = 0;
    const blas::Row g = dcgs_geom(kern, B, sizeof(double) * 8, 0, &sm);
    kern<<<g.grid, g.threads, sm, s>>>((const CT*)V0.p, vstride, (const CT*)B.p, B.V, B.R, B.dof, g.spb, out_dev);
    GMG_CUDA(cudaGetLastError());
    return GMG_OK;
  };
  auto run = [&](auto* p) -> gmg_status {
    typedef std::conditional_t<std::is_same<std::remove_pointer_t<decltype(p)>, float2>::value, float, double> T;
    switch (nv) {
      case 0: return launch(blas::dcgs_dots_row_kernel<0, T>, p);
      case 1: return launch(blas::dcgs_dots_row_kernel<1, T>, p);
      case 2: return launch(blas::dcgs_dots_row_kernel<2, T>, p);
      case 3: return launch(blas::dcgs_dots_row_kernel<3, T>, p);
      case 4: return launch(blas::dcgs_dots_row_kernel<4, T>, p);
      case 5: return launch(blas::dcgs_dots_row_kernel<5, T>, p);
      case 6: return launch(blas::dcgs_dots_row_kernel<6, T>, p);
      case 7: return launch(blas::dcgs_dots_row_kernel<7, T>, p);
      case 8: return launch(blas::dcgs_dots_row_kernel<8, T>, p);
      default: return launch(blas::dcgs_dots_row_kernel<9, T>, p);
    }
  };
  if (B.prec == GMG_F32) return run((float2*)nullptr);
  return run((double2*)nullptr);
}

gmg_status vec_dcgs_update(const double2* coef_dev, Vec& V0, int64_t vstride, int nv, const Vec& B, cudaStream_t s) {
  GMG_CHECK(vec_dcgs_supported(B, nv), GMG_ERR_UNSUPPORTED, "dcgs: unsupported shape");
  GMG_CHECK(V0.prec == B.prec, GMG_ERR_UNSUPPORTED, "dcgs: basis and new vector differ in precision");
  auto launch = [&](auto kern, auto* p) -> gmg_status {
    typedef std::remove_pointer_t<decltype(p)> CT;
    size_t sm = 0;
    const blas::Row g = dcgs_geom(kern, B, 0, sizeof(double2) * (2 * nv + 3) * B.R, &sm);
    kern<<<g.grid, g.threads, sm, s>>>(coef_dev, (CT*)V0.p, vstride, (const CT*)B.p, B.V, B.R, B.dof, g.spb);
    GMG_CUDA(cudaGetLastError());
    return GMG_OK;
  };
  auto run = [&](auto* p) -> gmg_status {
    typedef std::conditional_t<std::is_same<std::remove_pointer_t<decltype(p)>, float2>::value, float, double> T;
    switch (nv) {
      case 0: return launch(blas::dcgs_update_row_kernel<0, T>, p);
      case 1: return launch(blas::dcgs_update_row_kernel<1, T>, p);
      case 2: return launch(blas::dcgs_update_row_kernel<2, T>, p);
      case 3: return launch(blas::dcgs_update_row_kernel<3, T>, p);
      case 4: return launch(blas::dcgs_update_row_kernel<4, T>, p);
      case 5: return launch(blas::dcgs_update_row_kernel<5, T>, p);
      case 6: return launch(blas::dcgs_update_row_kernel<6, T>, p);
      case 7: return launch(blas::dcgs_update_row_kernel<7, T>, p);
      case 8: return launch(blas::dcgs_update_row_kernel<8, T>, p);
      default: return launch(blas::dcgs_update_row_kernel<9, T>, p);
    }
  };
  if (B.prec == GMG_F32) return run((float2*)nullptr);
  return run((double2*)nullptr);
}

gmg_status vec_xmy_bf16_blocked(const Vec& X, const Vec& Y, Vec& Z, cudaStream_t s) {
  GMG_CHECK(X.prec == GMG_F32 && Y.prec == GMG_F32 && Z.prec == GMG_BF16 && X.dof == 12 && X.R * 12 <= 1024,
            GMG_ERR_UNSUPPORTED, "xmy (site-blocked BF16): FP32 spin-colour inputs");
  const blas::Row rg = blas::row_geom(X.V, X.R, 12);
  blas::xmy_bf16_blocked_row_kernel<<<rg.grid, rg.threads, 0, s>>>((const float2*)X.p, (const float2*)Y.p,
                                                                  (uint32_t*)Z.p, X.V, X.R, rg.spb);
  GMG_CUDA(cudaGetLastError());
  return GMG_OK;
}

gmg_status vec_xmy_bf16(const Vec& X, const Vec& Y, Vec& Z, cudaStream_t s) {
  GMG_CHECK(X.prec == GMG_F32 && Y.prec == GMG_F32 && Z.prec == GMG_BF16, GMG_ERR_UNSUPPORTED,
            "xmy to BF16: FP32 operands and a BF16 result");
  const int64_t n = Z.elems();
  blas::xmy_bf16_kernel<<<blas::grid1(n), 256, 0, s>>>((const float2*)X.p, (const float2*)Y.p, (uint32_t*)Z.p, n);
  GMG_CUDA(cudaGetLastError());
  return GMG_OK;
}

gmg_status vec_gather(const Vec& src, const int* idx, Vec& dst, cudaStream_t s) {
  const int64_t n = dst.elems();
  const int g = blas::grid1(n);
  if (src.prec == GMG_F64)
    blas::permute_kernel<double, false><<<g, 256, 0, s>>>((const double2*)src.p, (double2*)dst.p, idx, dst.V, src.R,
                                                          dst.R, dst.R, dst.dof);
  else
    blas::permute_kernel<float, false><<<g, 256, 0, s>>>((const float2*)src.p, (float2*)dst.p, idx, dst.V, src.R,
                                                         dst.R, dst.R, dst.dof);
  GMG_CUDA(cudaGetLastError());
  return GMG_OK;
}

gmg_status vec_scatter(const Vec& src, const int* idx, Vec& dst, cudaStream_t s) {
  const int64_t n = src.elems();
  const int g = blas::grid1(n);
  if (src.prec == GMG_F64)
    blas::permute_kernel<double, true><<<g, 256, 0, s>>>((const double2*)src.p, (double2*)dst.p, idx, src.V, src.R,
                                                         dst.R, src.R, src.dof);
  else
    blas::permute_kernel<float, true><<<g, 256, 0, s>>>((const float2*)src.p, (float2*)dst.p, idx, src.V, src.R,
                                                        dst.R, src.R, src.dof);
  GMG_CUDA(cudaGetLastError());
  return GMG_OK;
}

gmg_status vec_gaussian(Vec& X, uint64_t seed, cudaStream_t s) {
  const int64_t n = X.elems();
  const int g = blas::grid1(n);
  if (X.prec == GMG_F64) blas::gaussian_kernel<double><<<g, 256, 0, s>>>((double2*)X.p, n, seed);
  else blas::gaussian_kernel<float><<<g, 256, 0, s>>>((float2*)X.p, n, seed);
  GMG_CUDA(cudaGetLastError());
  return GMG_OK;
}

gmg_status vec_chiral_double(const Vec& X, double* basis_dev, cudaStream_t s, double factor) {
  const int64_t n = X.elems();
  const int g = blas::grid1(n);
  if (X.prec == GMG_F64)
    blas::chiral_double_kernel<double>
        <<<g, 256, 0, s>>>((const double2*)X.p, (double2*)basis_dev, X.V, X.R, X.dof, factor);
  else
    blas::chiral_double_kernel<float>
        <<<g, 256, 0, s>>>((const float2*)X.p, (double2*)basis_dev, X.V, X.R, X.dof, factor);
  GMG_CUDA(cudaGetLastError());
  return GMG_OK;
}

// ---------------------------------------------------------------------------
// Gram matrix across the RHS columns of a field and a triangular recombination
// of the columns (global orthonormalisation of a set of lattice vectors kept
// as the RHS of one field)
// ---------------------------------------------------------------------------
namespace blas {
template <class T>
__global__ void gram_rhs_kernel(const typename C2<T>::t* __restrict__ X, int64_t V, int R, int dof,
                                double2* __restrict__ G) {
  const int a = threadIdx.x / R, b = threadIdx.x % R;  // blockDim = R * R
  double gr = 0.0, gi = 0.0;
  for (int64_t s = blockIdx.x; s < V; s += gridDim.x) {
    const typename C2<T>::t* xa = X + (s * R + a) * dof;
    const typename C2<T>::t* xb = X + (s * R + b) * dof;
    for (int k = 0; k < dof; ++k) {  // conj(xa) xb
      const double ar = xa[k].x, ai = xa[k].y, br = xb[k].x, bi = xb[k].y;
      gr += ar * br + ai * bi;
      gi += ar * bi - ai * br;
    }
  }
  atomicAdd(&G[a * R + b].x, gr);
  atomicAdd(&G[a * R + b].y, gi);
}

// X[s][a][k] <- sum_{b <= a} T[a * R + b] X[s][b][k]   (R <= 32)
template <class T>
__global__ void tri_apply_kernel(const double2* __restrict__ Tm, typename C2<T>::t* __restrict__ X, int64_t V, int R,
                                 int dof) {
  const int64_t n = V * dof;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t s = e / dof;
    const int k = (int)(e % dof);
    double xr[32], xi[32];
    for (int b = 0; b < R; ++b) {
      xr[b] = X[(s * R + b) * dof + k].x;
      xi[b] = X[(s * R + b) * dof + k].y;
    }
    for (int a = 0; a < R; ++a) {  // inputs are held in registers
      double yr = 0.0, yi = 0.0;
      for (int b = 0; b <= a; ++b) {
        const double2 t = Tm[a * R + b];
        yr += t.x * xr[b] - t.y * xi[b];
        yi += t.x * xi[b] + t.y * xr[b];
      }
      typename C2<T>::t o;
      o.x = yr;
      o.y = yi;
      X[(s * R + a) * dof + k] = o;
    }
  }
}
}  // namespace blas

gmg_status vec_gram(const Vec& X, double2* G_dev, cudaStream_t s) {
  GMG_CHECK(X.R >= 1 && X.R <= 32, GMG_ERR_UNSUPPORTED, "vec_gram: at most 32 vectors");
  GMG_CUDA(cudaMemsetAsync(G_dev, 0, sizeof(double2) * X.R * X.R, s));
  const int g = (int)std::min<int64_t>(X.V, 148 * 8);
  if (X.prec == GMG_F64)
    blas::gram_rhs_kernel<double><<<g, X.R * X.R, 0, s>>>((const double2*)X.p, X.V, X.R, X.dof, G_dev);
  else
    blas::gram_rhs_kernel<float><<<g, X.R * X.R, 0, s>>>((const float2*)X.p, X.V, X.R, X.dof, G_dev);
  GMG_CUDA(cudaGetLastError());
  return GMG_OK;
}

gmg_status vec_tri_apply(const double2* T_dev, Vec& X, cudaStream_t s) {
  GMG_CHECK(X.R >= 1 && X.R <= 32, GMG_ERR_UNSUPPORTED, "vec_tri_apply: at most 32 vectors");
  const int g = blas::grid1(X.V * X.dof);
  if (X.prec == GMG_F64)
    blas::tri_apply_kernel<double><<<g, 256, 0, s>>>(T_dev, (double2*)X.p, X.V, X.R, X.dof);
  else
    blas::tri_apply_kernel<float><<<g, 256, 0, s>>>(T_dev, (float2*)X.p, X.V, X.R, X.dof);
  GMG_CUDA(cudaGetLastError());
  return GMG_OK;
}

// ---------------------------------------------------------------------------
// BiCGStab building blocks with per-RHS scalars kept on the device
// (sc layout per RHS r: sc[0*R+r] rho, [1] alpha, [2] omega, [3] beta)
// ---------------------------------------------------------------------------
namespace blas {
__device__ __forceinline__ double2 zdiv(double2 a, double2 b) {
  const double n = b.x * b.x + b.y * b.y;
  if (!(n > 0.0)) return make_double2(0.0, 0.0);
  return make_double2((a.x * b.x + a.y * b.y) / n, (a.y * b.x - a.x * b.y) / n);
}
__device__ __forceinline__ double2 zmul2(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// rho_new = <r0, r>: beta = (rho_new / rho) (alpha / omega), rho = rho_new
__global__ void bicg_beta_kernel(const double2* __restrict__ rho_new, double2* __restrict__ sc, int R) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= R) return;
  const double2 rho = sc[r], alpha = sc[R + r], omega = sc[2 * R + r];
  sc[3 * R + r] = zmul2(zdiv(rho_new[r], rho), zdiv(alpha, omega));
  sc[r] = rho_new[r];
}
// alpha = rho / <r0, v>
__global__ void bicg_alpha_kernel(const double2* __restrict__ r0v, double2* __restrict__ sc, int R) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r < R) sc[R + r] = zdiv(sc[r], r0v[r]);
}
// omega = <t, s> / <t, t>
__global__ void bicg_omega_kernel(const double2* __restrict__ ts, const double2* __restrict__ tt, double2* __restrict__ sc,
                                  int R) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r < R) sc[2 * R + r] = zdiv(ts[r], tt[r]);
}

// p = r + beta (p - omega v)
template <class T>
__global__ void bicg_p_kernel(typename C2<T>::t* __restrict__ p, const typename C2<T>::t* __restrict__ r,
                              const typename C2<T>::t* __restrict__ v, const double2* __restrict__ sc, int64_t V, int R,
                              int dof) {
  const int64_t n = V * R * dof;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (RhsWalk w(blockIdx.x * (int64_t)blockDim.x + threadIdx.x, stride, R, dof); w.e < n; w.next(stride)) {
    const int64_t e = w.e;
    const int k = w.r();
    const double2 om = sc[2 * R + k], be = sc[3 * R + k];
    const double2 pv = make_double2(p[e].x, p[e].y), vv = make_double2(v[e].x, v[e].y);
    const double2 ov = zmul2(om, vv);
    const double2 q = zmul2(be, make_double2(pv.x - ov.x, pv.y - ov.y));
    p[e].x = (T)(r[e].x + q.x);
    p[e].y = (T)(r[e].y + q.y);
  }
}
// s = r - alpha v   (written into r's buffer s)
template <class T>
__global__ void bicg_s_kernel(typename C2<T>::t* __restrict__ s_, const typename C2<T>::t* __restrict__ r,
                              const typename C2<T>::t* __restrict__ v, const double2* __restrict__ sc, int64_t V, int R,
                              int dof) {
  const int64_t n = V * R * dof;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (RhsWalk w(blockIdx.x * (int64_t)blockDim.x + threadIdx.x, stride, R, dof); w.e < n; w.next(stride)) {
    const int64_t e = w.e;
    const int k = w.r();
    const double2 av = zmul2(sc[R + k], make_double2(v[e].x, v[e].y));
    s_[e].x = (T)(r[e].x - av.x);
    s_[e].y = (T)(r[e].y - av.y);
  }
}
// x += alpha p + omega s;  r = s - omega t
template <class T>
__global__ void bicg_xr_kernel(typename C2<T>::t* __restrict__ x, typename C2<T>::t* __restrict__ r,
                               const typename C2<T>::t* __restrict__ p, const typename C2<T>::t* __restrict__ s_,
                               const typename C2<T>::t* __restrict__ t, const double2* __restrict__ sc, int64_t V, int R,
                               int dof) {
  const int64_t n = V * R * dof;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (RhsWalk w(blockIdx.x * (int64_t)blockDim.x + threadIdx.x, stride, R, dof); w.e < n; w.next(stride)) {
    const int64_t e = w.e;
    const int k = w.r();
    const double2 al = sc[R + k], om = sc[2 * R + k];
    const double2 sv = make_double2(s_[e].x, s_[e].y);
    const double2 ap = zmul2(al, make_double2(p[e].x, p[e].y)), os = zmul2(om, sv);
    const double2 ot = zmul2(om, make_double2(t[e].x, t[e].y));
    x[e].x = (T)(x[e].x + ap.x + os.x);
    x[e].y = (T)(x[e].y + ap.y + os.y);
    r[e].x = (T)(sv.x - ot.x);
    r[e].y = (T)(sv.y - ot.y);
  }
}
}  // namespace blas

gmg_status bicg_scalar(int which, const double2* a, const double2* b, double2* sc, int R, cudaStream_t s) {
  const int g = (R + 127) / 128;
  if (which == 0) blas::bicg_beta_kernel<<<g, 128, 0, s>>>(a, sc, R);
  else if (which == 1) blas::bicg_alpha_kernel<<<g, 128, 0, s>>>(a, sc, R);
  else blas::bicg_omega_kernel<<<g, 128, 0, s>>>(a, b, sc, R);
  GMG_CUDA(cudaGetLastError());
  return GMG_OK;
}

gmg_status bicg_vec(int which, Vec& a, const Vec& b, const Vec& c, const Vec& d, const Vec& e, const double2* sc,
                    cudaStream_t s) {
  const int g = blas::grid1(a.elems());
  const bool f64 = a.prec == GMG_F64;
  if (which == 0) {  // p = r + beta (p - omega v): a = p, b = r, c = v
    if (f64) blas::bicg_p_kernel<double><<<g, 256, 0, s>>>((double2*)a.p, (const double2*)b.p, (const double2*)c.p, sc, a.V, a.R, a.dof);
    else blas::bicg_p_kernel<float><<<g, 256, 0, s>>>((float2*)a.p, (const float2*)b.p, (const float2*)c.p, sc, a.V, a.R, a.dof);
  } else if (which == 1) {  // s = r - alpha v: a = s, b = r, c = v
    if (f64) blas::bicg_s_kernel<double><<<g, 256, 0, s>>>((double2*)a.p, (const double2*)b.p, (const double2*)c.p, sc, a.V, a.R, a.dof);
    else blas::bicg_s_kernel<float><<<g, 256, 0, s>>>((float2*)a.p, (const float2*)b.p, (const float2*)c.p, sc, a.V, a.R, a.dof);
  } else {  // x += alpha p + omega s; r = s - omega t: a = x, b = r (written), c = p, d = s, e = t
    Vec& r = const_cast<Vec&>(b);
    if (f64)
      blas::bicg_xr_kernel<double><<<g, 256, 0, s>>>((double2*)a.p, (double2*)r.p, (const double2*)c.p, (const double2*)d.p,
                                                     (const double2*)e.p, sc, a.V, a.R, a.dof);
    else
      blas::bicg_xr_kernel<float><<<g, 256, 0, s>>>((float2*)a.p, (float2*)r.p, (const float2*)c.p, (const float2*)d.p,
                                                    (const float2*)e.p, sc, a.V, a.R, a.dof);
  }
  GMG_CUDA(cudaGetLastError());
  return GMG_OK;
}

}  // namespace gmg

extern "C" gmg_status gmg_chiral_double(int64_t V, int dof, int nvec, gmg_prec prec, const void* vecs, double factor,
                                        double* basis, gmg_stream stream) {
  using namespace gmg;
  GMG_CHECK(vecs && basis, GMG_ERR_ARGUMENT, "gmg_chiral_double: null argument");
  GMG_CHECK(V >= 1 && dof >= 2 && dof % 2 == 0 && nvec >= 1 && nvec <= 4096, GMG_ERR_ARGUMENT,
            "gmg_chiral_double: V >= 1, an even dof >= 2 and 1 <= nvec <= 4096 required");
  GMG_CHECK(prec == GMG_F64 || prec == GMG_F32, GMG_ERR_ARGUMENT, "gmg_chiral_double: vectors must be F64 or F32");
  Vec X;
  X.p = const_cast<void*>(vecs);
  X.V = V;
  X.R = nvec;
  X.dof = dof;
  X.prec = prec;
  return vec_chiral_double(X, basis, S(stream), factor);
}

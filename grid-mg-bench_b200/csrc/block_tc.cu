// block_tc.cu -- block projection and promotion on the 5th-generation tensor cores
// (BF16 hi+lo split).  Promotion is described above promote_tc_kernel.
//
// Restates blockLutedInnerProduct (include/CoarsenedMatrixUpstreamImprovedDirsaveLut.h:70-121,
// multi-RHS ...LutMRHS.h:70-120), the restriction ProjectToSubspace of the K-cycle, as one
// complex GEMM per block c:
//
//     C_c[r][i] = sum_k conj(V_c[i][k]) F_c[k][r]          K = sites per block * dof
//
// decomposed into one real MMA per K-step with interleaved basis rows (2i = Re v_i, 2i+1 = Im v_i):
//
//     D (2N x 2R) += [Re V; Im V] (2N x K) . [Re F | Im F] (K x 2R)
//     C_r = D[2i][r] + D[2i+1][R+r],   C_i = D[2i][R+r] - D[2i+1][r]
//
// Both operands are split into BF16 hi + lo parts (x = hi + lo, lo = bf16(x - hi)); three
// products hi.hi + hi.lo + lo.hi accumulate in FP32 in tensor memory, which keeps the
// result at about FP32 accuracy while reading the basis at BF16 cost per part.
//
// Kernel (one or two persistent CTAs per SM, blocks c = blockIdx.x, +gridDim.x, ...):
//   warp 0      producer: one bulk copy of the basis hi and lo tiles per stage
//               (the packed basis is stage-contiguous in HBM)
//   warp 1      TMEM allocation + MMA issue (one thread): 3 MMAs per K-step
//   warps 2-9   converters: read the FP32 fine vector of the stage's sites (bulk-copied
//               into the stage by the producer when its rows are 16-byte aligned), split
//               into hi/lo BF16 and store the B tiles in the canonical K-major
//               core-matrix layout, then fence.proxy.async + mbarrier arrive
//   warps 10-13 epilogue: tcgen05.ld, lane-pair (re, im) recombination, FP32 output
// All mbarrier waits are bounded; on time-out the kernel records an error code,
// drains its copies and MMAs, frees TMEM and returns.
#include <algorithm>

#include "gmg_internal.cuh"

namespace gmg {
namespace ptc {

constexpr int kWarps = 14;
constexpr int kThreads = kWarps * 32;
constexpr int kConvThreads = 256;
constexpr int kEpiThreads = 128;
constexpr int kAcc = 2;
constexpr long long kTimeoutCycles = 4000000000LL;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, volatile int* abort_flag) {
  if (mbar_try_wait(bar, parity)) return true;
  const long long t0 = clock64();
  while (true) {
    if (mbar_try_wait(bar, parity)) return true;
    if (*abort_flag) return false;
    if (clock64() - t0 > kTimeoutCycles) return false;
  }
}
__device__ __forceinline__ bool mbar_drain(uint64_t* bar, uint32_t parity) {
  const long long t0 = clock64();
  while (!mbar_try_wait(bar, parity))
    if (clock64() - t0 > kTimeoutCycles) return false;
  return true;
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ uint64_t make_desc(const void* smem, uint32_t lbo, uint32_t sbo) {
  uint64_t d = (smem_u32(smem) >> 4) & 0x3FFF;
  d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
  d |= (uint64_t)1 << 46;  // sm_100 descriptor version; no swizzle
  return d;
}
__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(acc)
      : "memory");
}
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tmem_ld16x2(uint32_t ta, uint32_t tb, float* va, float* vb) {
  uint32_t a[16], b[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
      "%14, %15}, [%16];"
      : "=r"(a[0]), "=r"(a[1]), "=r"(a[2]), "=r"(a[3]), "=r"(a[4]), "=r"(a[5]), "=r"(a[6]), "=r"(a[7]),
        "=r"(a[8]), "=r"(a[9]), "=r"(a[10]), "=r"(a[11]), "=r"(a[12]), "=r"(a[13]), "=r"(a[14]), "=r"(a[15])
      : "r"(ta));
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
      "%14, %15}, [%16];"
      : "=r"(b[0]), "=r"(b[1]), "=r"(b[2]), "=r"(b[3]), "=r"(b[4]), "=r"(b[5]), "=r"(b[6]), "=r"(b[7]),
        "=r"(b[8]), "=r"(b[9]), "=r"(b[10]), "=r"(b[11]), "=r"(b[12]), "=r"(b[13]), "=r"(b[14]), "=r"(b[15])
      : "r"(tb));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) {
    va[i] = __uint_as_float(a[i]);
    vb[i] = __uint_as_float(b[i]);
  }
}

// K-steps of one stage as straight-line code: three MMAs (hi.hi, hi.lo, lo.hi) per
// 16-deep K-step.  Issuing tcgen05.mma from rolled loops with data-dependent
// control flow between the instructions measured several times slower per MMA.
template <int KSTEPS>
__device__ __forceinline__ void issue_hilo(uint32_t dt, uint64_t ah, uint64_t al, uint64_t bh, uint64_t bl,
                                           uint32_t a_ks, uint32_t b_ks, uint32_t idesc, bool first) {
#pragma unroll
  for (int k = 0; k < KSTEPS; ++k) {
    mma_bf16(dt, ah + k * a_ks, bh + k * b_ks, idesc, (first && k == 0) ? 0u : 1u);
    mma_bf16(dt, ah + k * a_ks, bl + k * b_ks, idesc, 1u);
    mma_bf16(dt, al + k * a_ks, bh + k * b_ks, idesc, 1u);
  }
}

__device__ __forceinline__ void issue_hilo_n(int ksteps, uint32_t dt, uint64_t ah, uint64_t al, uint64_t bh,
                                             uint64_t bl, uint32_t a_ks, uint32_t b_ks, uint32_t idesc, bool first) {
  switch (ksteps) {
    case 1: issue_hilo<1>(dt, ah, al, bh, bl, a_ks, b_ks, idesc, first); break;
    case 2: issue_hilo<2>(dt, ah, al, bh, bl, a_ks, b_ks, idesc, first); break;
    case 3: issue_hilo<3>(dt, ah, al, bh, bl, a_ks, b_ks, idesc, first); break;
    case 4: issue_hilo<4>(dt, ah, al, bh, bl, a_ks, b_ks, idesc, first); break;
    case 5: issue_hilo<5>(dt, ah, al, bh, bl, a_ks, b_ks, idesc, first); break;
    case 6: issue_hilo<6>(dt, ah, al, bh, bl, a_ks, b_ks, idesc, first); break;
    case 7: issue_hilo<7>(dt, ah, al, bh, bl, a_ks, b_ks, idesc, first); break;
    case 8: issue_hilo<8>(dt, ah, al, bh, bl, a_ks, b_ks, idesc, first); break;
    default: {
      int k = 0;
      for (; k + 8 <= ksteps; k += 8)
        issue_hilo<8>(dt, ah + k * a_ks, al + k * a_ks, bh + k * b_ks, bl + k * b_ks, a_ks, b_ks, idesc,
                      first && k == 0);
      for (; k < ksteps; ++k)
        issue_hilo<1>(dt, ah + k * a_ks, al + k * a_ks, bh + k * b_ks, bl + k * b_ks, a_ks, b_ks, idesc, false);
    }
  }
}

__device__ __forceinline__ uint32_t bf16_pair(float a, float b) {
  return (uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(a)) |
         ((uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(b)) << 16);
}
__device__ __forceinline__ float bf16_round(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }
// hi = round-to-nearest BF16 of (a, b) packed in one word (low half: a), and
// the lo parts a - hi_a, b - hi_b packed the same way; the BF16 -> FP32 of hi
// is a 16-bit shift
__device__ __forceinline__ void bf16_hilo_pair(float a, float b, uint32_t& hi, uint32_t& lo) {
  const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
  hi = *reinterpret_cast<const uint32_t*>(&h);
  const float ha = __uint_as_float(hi << 16), hb = __uint_as_float(hi & 0xffff0000u);
  const __nv_bfloat162 l = __floats2bfloat162_rn(a - ha, b - hb);
  lo = *reinterpret_cast<const uint32_t*>(&l);
}

struct Params {
  const uint16_t* ahi;      // packed basis, hi part: [Vc][Kp/8][Mp][8]
  const uint16_t* alo;      // lo part
  const float2* fine;       // [Vf][nrhs][dof] FP32
  const int32_t* blk_sites; // [Vc][bv]
  float2* coarse;           // [Vc][nrhs][N] FP32
  int* err;
  int Vc, N, dof, bv, nrhs, R, Rp, Kp, Mp, KS, sps, stages, aligned16;
  int raw;  // 1: the producer bulk-copies each site's FP32 rows into the stage (16-byte aligned rows)
};

template <int CTAS>  // CTAs per SM the register budget allows (1 or 2)
__global__ void __launch_bounds__(kThreads, CTAS) project_tc_kernel(const Params P) {
  extern __shared__ __align__(1024) unsigned char smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int kc_stage = P.KS / 8;                               // K-chunks per stage
  const uint32_t a_bytes = (uint32_t)kc_stage * P.Mp * 16;     // one of hi / lo
  const uint32_t b_bytes = (uint32_t)kc_stage * 2 * P.Rp * 16; // one of hi / lo
  const uint32_t site_bytes = (uint32_t)P.nrhs * P.dof * 8;      // one fine site, all RHS, FP32
  const uint32_t raw_bytes = P.raw ? (uint32_t)P.sps * site_bytes : 0u;
  const uint32_t stage_bytes = 2 * a_bytes + 2 * b_bytes + raw_bytes;
  const int spb = P.Kp / P.KS;  // stages per block

  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + (size_t)P.stages * stage_bytes);
  uint64_t* full = bars;
  uint64_t* empty = full + P.stages;
  uint64_t* rawb = empty + P.stages;  // [stages] raw site rows landed (raw mode)
  uint64_t* tfull = rawb + P.stages;
  uint64_t* tempty = tfull + kAcc;
  uint64_t* drain = tempty + kAcc;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(drain + 1);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);
  int* site_tab = reinterpret_cast<int*>(tmem_slot + 4);  // [bv] fine sites of the producer's block (raw mode)

  const uint32_t acc_cols = 2 * P.Rp;
  uint32_t ncols = 32;
  while (ncols < kAcc * acc_cols) ncols <<= 1;

  // zero the B tiles once: padding rows (r >= R) and padding K stay zero
  for (size_t k = threadIdx.x; k < (size_t)P.stages * stage_bytes / 16; k += blockDim.x)
    reinterpret_cast<uint4*>(smem)[k] = make_uint4(0, 0, 0, 0);
  if (threadIdx.x == 0) {
    for (int s = 0; s < P.stages; ++s) {
      mbar_init(&full[s], 1 + kConvThreads);
      mbar_init(&empty[s], 1);
      mbar_init(&rawb[s], 1);
    }
    for (int a = 0; a < kAcc; ++a) {
      mbar_init(&tfull[a], 1);
      mbar_init(&tempty[a], kEpiThreads);
    }
    mbar_init(drain, 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // zeroed tiles visible to the tensor core
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tmem_base = *tmem_slot;
  const int nblk = (P.Vc - (int)blockIdx.x + (int)gridDim.x - 1) / (int)gridDim.x;
  const int64_t nseq = (int64_t)nblk * spb;  // stage-sequence numbers of this CTA

  if (warp == 0) {
    // ---------------------------------------------------------------- producer: basis tiles
    // (+ the fine site rows in raw mode).  At the start of each block the warp
    // loads the block's site table into shared memory in parallel, so the issuing
    // lane never waits on a dependent global load between copies.
    int64_t last = -1;
    bool stop = false;
    for (int bi = 0; bi < nblk && !stop; ++bi) {
      const int c = blockIdx.x + bi * gridDim.x;
      if (P.raw) {
        __syncwarp();
        for (int k = lane; k < P.bv; k += 32) site_tab[k] = P.blk_sites[(size_t)c * P.bv + k];
        __syncwarp();
      }
      if (lane == 0) {
        for (int ks = 0; ks < spb; ++ks) {
          const int64_t n = (int64_t)bi * spb + ks;
          const int stage = (int)(n % P.stages);
          const uint32_t phase = (uint32_t)((n / P.stages) & 1);
          if (!mbar_wait(&empty[stage], phase ^ 1, abort_flag)) {
            atomicCAS(P.err, 0, 1);
            *abort_flag = 1;
            stop = true;
            break;
          }
          unsigned char* st = smem + (size_t)stage * stage_bytes;
          const size_t off = ((size_t)c * (P.Kp / 8) + (size_t)ks * kc_stage) * P.Mp * 8;  // halves
          mbar_expect_tx(&full[stage], 2 * a_bytes);
          bulk_g2s(st, P.ahi + off, a_bytes, &full[stage]);
          bulk_g2s(st + a_bytes, P.alo + off, a_bytes, &full[stage]);
          if (P.raw) {
            // the stage's fine sites: one contiguous [nrhs][dof] FP32 row block each
            const int s0 = ks * P.sps;
            const int nsv = min(P.sps, P.bv - s0);
            unsigned char* rw = st + 2 * a_bytes + 2 * b_bytes;
            mbar_expect_tx(&rawb[stage], (uint32_t)nsv * site_bytes);
            for (int sl = 0; sl < nsv; ++sl)
              bulk_g2s(rw + (size_t)sl * site_bytes,
                       reinterpret_cast<const unsigned char*>(P.fine) + (size_t)site_tab[s0 + sl] * site_bytes,
                       site_bytes, &rawb[stage]);
          }
          last = n;
        }
      }
      stop = __shfl_sync(0xffffffffu, stop, 0);
    }
    if (lane == 0) {
      for (int64_t n = last; n >= 0 && n > last - P.stages; --n) {
        mbar_drain(&full[n % P.stages], (uint32_t)((n / P.stages) & 1));
        if (P.raw) mbar_drain(&rawb[n % P.stages], (uint32_t)((n / P.stages) & 1));
      }
    }
  } else if (warp == 1) {
    // ---------------------------------------------------------------- MMA issue
    if (lane == 0) {
      const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(2 * P.Rp) >> 3) << 17 |
                             ((uint32_t)P.Mp >> 4) << 24;
      bool ok = true;
      int64_t n = 0;
      for (int bi = 0; bi < nblk && ok; ++bi) {
        const int acc = bi % kAcc;
        const uint32_t aph = (uint32_t)(bi / kAcc) & 1;
        if (!mbar_wait(&tempty[acc], aph ^ 1, abort_flag)) { ok = false; break; }
        fence_after();
        const uint32_t dt = tmem_base + acc * acc_cols;
        for (int ks = 0; ks < spb; ++ks, ++n) {
          const int stage = (int)(n % P.stages);
          const uint32_t phase = (uint32_t)((n / P.stages) & 1);
          if (!mbar_wait(&full[stage], phase, abort_flag)) { ok = false; break; }
          fence_after();
          unsigned char* st = smem + (size_t)stage * stage_bytes;
          unsigned char* ah = st;
          unsigned char* al = st + a_bytes;
          unsigned char* bh = st + 2 * a_bytes;
          unsigned char* bl = bh + b_bytes;
          const uint32_t la = (uint32_t)P.Mp * 16, lb = (uint32_t)(2 * P.Rp) * 16;
          issue_hilo_n(kc_stage / 2, dt, make_desc(ah, la, 128), make_desc(al, la, 128), make_desc(bh, lb, 128),
                       make_desc(bl, lb, 128), 2 * P.Mp, 4 * P.Rp, idesc, ks == 0);
          mma_commit(&empty[stage]);
        }
        if (!ok) break;
        mma_commit(&tfull[acc]);
      }
      if (!ok) {
        atomicCAS(P.err, 0, 2);
        *abort_flag = 1;
      }
      mma_commit(drain);
      mbar_drain(drain, 0);
    }
  } else if (warp < 10) {
    // ---------------------------------------------------------------- converters: B tiles
    // Each thread takes (site, rhs) records and splits the record's dof FP32
    // complex values (dof even) into BF16 hi / lo pairs of the K-major B tiles.
    // Raw mode reads the records from the stage's bulk-copied site rows; the
    // direct mode loads them from global memory.
    const int t = threadIdx.x - 64;  // 0..255
    const int hd = P.dof / 2;        // complex pairs per (site, rhs) record
    const int items = P.sps * P.R * hd;
    // per-item step of kConvThreads items in (a2, r, sl) digits
    const int da2 = kConvThreads % hd, drec = kConvThreads / hd;
    const int dr = drec % P.R, dsl = drec / P.R;
    for (int64_t n = 0; n < nseq; ++n) {
      const int stage = (int)(n % P.stages);
      const uint32_t phase = (uint32_t)((n / P.stages) & 1);
      const bool ok = P.raw ? mbar_wait(&rawb[stage], phase, abort_flag)
                            : mbar_wait(&empty[stage], phase ^ 1, abort_flag);
      if (!ok) {
        atomicCAS(P.err, 0, 3);
        *abort_flag = 1;
        break;
      }
      const int c = blockIdx.x + (int)(n / spb) * gridDim.x;
      const int ks = (int)(n % spb);
      unsigned char* st = smem + (size_t)stage * stage_bytes;
      uint32_t* bh = reinterpret_cast<uint32_t*>(st + 2 * a_bytes);
      uint32_t* bl = reinterpret_cast<uint32_t*>(st + 2 * a_bytes + b_bytes);
      const unsigned char* rw = st + 2 * a_bytes + 2 * b_bytes;
      // item = ((sl * R) + r) * hd + a2: consecutive threads read consecutive 16-byte pairs;
      // (a2, r, sl) advance by carries instead of divisions per item
      int a2 = t % hd, rec0 = t / hd;
      int r = rec0 % P.R, sl = rec0 / P.R;
      for (int it = t; it < items; it += kConvThreads) {
        const int sb = ks * P.sps + sl;  // in-block site
        const int a = 2 * a2;
        float2 x0 = make_float2(0.f, 0.f), x1 = make_float2(0.f, 0.f);
        if (sb < P.bv) {  // else K padding of the block's last stage: zero
          if (P.raw) {
            const float4 v = *reinterpret_cast<const float4*>(rw + (size_t)sl * site_bytes + ((size_t)r * P.dof + a) * 8);
            x0 = make_float2(v.x, v.y);
            x1 = make_float2(v.z, v.w);
          } else {
            const float2* src = P.fine + ((size_t)P.blk_sites[(size_t)c * P.bv + sb] * P.nrhs + r) * P.dof + a;
            if (P.aligned16) {
              const float4 v = *reinterpret_cast<const float4*>(src);
              x0 = make_float2(v.x, v.y);
              x1 = make_float2(v.z, v.w);
            } else {
              x0 = src[0];
              x1 = src[1];
            }
          }
        }
        const int k = sl * P.dof + a;  // even: k, k+1 share a 16-byte core-matrix row
        const int chunk = k >> 3, j = k & 7;
        const size_t rre = ((size_t)chunk * 2 * P.Rp + r) * 4 + (j >> 1);  // 32-bit words
        const size_t rim = ((size_t)chunk * 2 * P.Rp + P.Rp + r) * 4 + (j >> 1);
        uint32_t hre, lre, him, lim;
        bf16_hilo_pair(x0.x, x1.x, hre, lre);
        bf16_hilo_pair(x0.y, x1.y, him, lim);
        bh[rre] = hre;
        bh[rim] = him;
        bl[rre] = lre;
        bl[rim] = lim;
        a2 += da2;
        r += dr;
        if (a2 >= hd) {
          a2 -= hd;
          ++r;
        }
        sl += dsl;
        if (r >= P.R) {
          r -= P.R;
          ++sl;
        }
      }
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      mbar_arrive(&full[stage]);
    }
  } else {
    // ---------------------------------------------------------------- epilogue (warps 10-13)
    const int q = warp & 3;
    const int rows_per_warp = P.Mp / 4;
    const int row = q * rows_per_warp + lane;
    const int i = row >> 1;
    const bool odd = row & 1;
    const bool valid = lane < rows_per_warp && row < 2 * P.N;
    for (int bi = 0; bi < nblk; ++bi) {
      const int c = blockIdx.x + bi * gridDim.x;
      const int acc = bi % kAcc;
      const uint32_t aph = (uint32_t)(bi / kAcc) & 1;
      const bool waited = mbar_wait(&tfull[acc], aph, abort_flag);
      if (!__all_sync(0xffffffffu, waited)) {
        if (!waited) atomicCAS(P.err, 0, 4);
        *abort_flag = 1;
        break;
      }
      fence_after();
      const uint32_t ta = tmem_base + ((uint32_t)(32 * q) << 16) + acc * acc_cols;
      float2* orow = P.coarse + (size_t)c * P.nrhs * P.N + i;
      for (int c0 = 0; c0 < P.Rp; c0 += 16) {
        float va[16], vb[16];
        tmem_ld16x2(ta + c0, ta + P.Rp + c0, va, vb);
        float pa[8], pb[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          pa[j] = __shfl_xor_sync(0xffffffffu, odd ? va[j] : va[8 + j], 1);
          pb[j] = __shfl_xor_sync(0xffffffffu, odd ? vb[j] : vb[8 + j], 1);
        }
        if (valid) {
#pragma unroll
          for (int j = 0; j < 8; ++j) {
            const int r = c0 + (odd ? 8 : 0) + j;
            if (r < P.R) {
              const float re = odd ? pa[j] + vb[8 + j] : va[j] + pb[j];
              const float im = odd ? pb[j] - va[8 + j] : vb[j] - pa[j];
              orow[(size_t)r * P.N] = make_float2(re, im);
            }
          }
        }
      }
      fence_before();
      mbar_arrive(&tempty[acc]);
    }
  }
  fence_before();
  __syncthreads();
  if (warp == 1) {
    fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_base), "r"(ncols) : "memory");
  }
}

// ---------------------------------------------------------------------------------
// Promotion: F_c[k][r] = sum_i V_c[i][k] C_c[i][r]  (blockLutedAxpy, ...Lut.h:122-170)
//
//     D (K x 2R) = A (K x 2N) . B (2N x 2R),  A[k][2i] = Re v_i(k), A[k][2i+1] = Im v_i(k)
//     B[2i][r] = Re C[i][r],  B[2i+1][r] = -Im C[i][r],  B[2i][R+r] = Im C[i][r],  B[2i+1][R+r] = Re C[i][r]
//     Re F = D[k][r],  Im F = D[k][R+r]
//
// A is the projection's packed basis read MN-major (its 8-dof x 8-row core matrices are
// contiguous: SBO = one K-chunk of Mp rows, LBO = 8 rows); M tiles of 128 fine dofs.
// B (2N x 2R, hi / lo) is built in shared memory once per block from the FP32 coarse
// vector.  Warp roles: 0 producer (basis tiles, one bulk copy each of hi / lo per
// M tile), 1 MMA issue, 2-5 B builders (once per block) and epilogue (FP32 output).
// ---------------------------------------------------------------------------------
struct PParams {
  const uint16_t* ahi;
  const uint16_t* alo;
  const float2* coarse;      // [Vc][nrhs][N]
  const int32_t* blk_sites;  // [Vc][bv]
  float2* fine;              // [Vf][nrhs][dof]
  int* err;
  int Vc, N, dof, bv, nrhs, R, Rp, K, Kp, Mp, K2, stages;  // K2 = 2N rounded up to 16
};

constexpr int kPWarps = 6;
constexpr int kPThreads = kPWarps * 32;
constexpr int kTileM = 128;

template <int CTAS>
__global__ void __launch_bounds__(kPThreads, CTAS) promote_tc_kernel(const PParams P) {
  extern __shared__ __align__(1024) unsigned char smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int ctile = kTileM / 8;                         // K-chunks (8 fine dofs) per M tile
  const uint32_t a_bytes = (uint32_t)ctile * P.Mp * 16;  // one of hi / lo
  const uint32_t stage_bytes = 2 * a_bytes;
  const int tpb = (P.Kp + kTileM - 1) / kTileM;         // M tiles per block
  const uint32_t b_bytes = (uint32_t)(P.K2 / 8) * 2 * P.Rp * 16;  // [K2/8 K-chunks][2Rp rows][8]
  unsigned char* bbuf = smem + (size_t)P.stages * stage_bytes;       // 2 blocks x (hi, lo)
  uint64_t* bars = reinterpret_cast<uint64_t*>(bbuf + 4 * (size_t)b_bytes);
  uint64_t* full = bars;
  uint64_t* empty = full + P.stages;
  uint64_t* tfull = empty + P.stages;   // [2] accumulator ready
  uint64_t* tempty = tfull + 2;         // [2] accumulator drained (128 epilogue threads)
  uint64_t* bfull = tempty + 2;         // [2] B of a block built (128 threads)
  uint64_t* bempty = bfull + 2;         // [2] B no longer read (MMA commit)
  uint64_t* drain = bempty + 2;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(drain + 1);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

  const uint32_t acc_cols = 2 * P.Rp;
  uint32_t ncols = 32;
  while (ncols < 2 * acc_cols) ncols <<= 1;
  if (threadIdx.x == 0) {
    for (int s = 0; s < P.stages; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int a = 0; a < 2; ++a) {
      mbar_init(&tfull[a], 1);
      mbar_init(&tempty[a], 128);
      mbar_init(&bfull[a], 128);
      mbar_init(&bempty[a], 1);
    }
    mbar_init(drain, 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tmem_base = *tmem_slot;
  const int nblk = (P.Vc - (int)blockIdx.x + (int)gridDim.x - 1) / (int)gridDim.x;
  const int64_t ntile = (int64_t)nblk * tpb;

  if (warp == 0) {
    if (lane == 0) {
      int64_t last = -1;
      for (int64_t n = 0; n < ntile; ++n) {
        const int stage = (int)(n % P.stages);
        const uint32_t phase = (uint32_t)((n / P.stages) & 1);
        if (!mbar_wait(&empty[stage], phase ^ 1, abort_flag)) {
          atomicCAS(P.err, 0, 11);
          *abort_flag = 1;
          break;
        }
        const int c = blockIdx.x + (int)(n / tpb) * gridDim.x;
        const int t = (int)(n % tpb);
        const int nch = min(ctile, P.Kp / 8 - t * ctile);
        const size_t off = ((size_t)c * (P.Kp / 8) + (size_t)t * ctile) * P.Mp * 8;
        unsigned char* st = smem + (size_t)stage * stage_bytes;
        mbar_expect_tx(&full[stage], 2u * nch * P.Mp * 16);
        bulk_g2s(st, P.ahi + off, nch * P.Mp * 16, &full[stage]);
        bulk_g2s(st + a_bytes, P.alo + off, nch * P.Mp * 16, &full[stage]);
        last = n;
      }
      for (int64_t n = last; n >= 0 && n > last - P.stages; --n)
        mbar_drain(&full[n % P.stages], (uint32_t)((n / P.stages) & 1));
    }
  } else if (warp == 1) {
    if (lane == 0) {
      const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | (1u << 15) /* A MN-major */ |
                             ((uint32_t)(2 * P.Rp) >> 3) << 17 | ((uint32_t)kTileM >> 4) << 24;
      bool ok = true;
      int64_t n = 0;
      for (int bi = 0; bi < nblk && ok; ++bi) {
        const int bsel = bi & 1;
        if (!mbar_wait(&bfull[bsel], (uint32_t)(bi >> 1) & 1, abort_flag)) { ok = false; break; }
        fence_after();
        unsigned char* bh = bbuf + (size_t)bsel * 2 * b_bytes;
        unsigned char* bl = bh + b_bytes;
        for (int t = 0; t < tpb; ++t, ++n) {
          const int acc = (int)(n & 1);
          const uint32_t aph = (uint32_t)(n >> 1) & 1;
          if (!mbar_wait(&tempty[acc], aph ^ 1, abort_flag)) { ok = false; break; }
          const int stage = (int)(n % P.stages);
          if (!mbar_wait(&full[stage], (uint32_t)((n / P.stages) & 1), abort_flag)) { ok = false; break; }
          fence_after();
          unsigned char* ah = smem + (size_t)stage * stage_bytes;
          unsigned char* al = ah + a_bytes;
          const uint32_t dt = tmem_base + acc * acc_cols;
          // A: MN-major, 8-dof groups P.Mp*16 bytes apart (SBO), 8-row groups 128 bytes apart (LBO);
          // B: K-major [K2/8 chunks][2Rp rows][8]
          issue_hilo_n(P.K2 / 16, dt, make_desc(ah, 128, (uint32_t)P.Mp * 16), make_desc(al, 128, (uint32_t)P.Mp * 16),
                       make_desc(bh, (uint32_t)(2 * P.Rp) * 16, 128), make_desc(bl, (uint32_t)(2 * P.Rp) * 16, 128),
                       2 * 128 / 16, 2 * 2 * P.Rp, idesc, true);
          mma_commit(&empty[stage]);
          mma_commit(&tfull[acc]);
        }
        if (!ok) break;
        mma_commit(&bempty[bsel]);
      }
      if (!ok) {
        atomicCAS(P.err, 0, 12);
        *abort_flag = 1;
      }
      mma_commit(drain);
      mbar_drain(drain, 0);
    }
  } else {
    // warps 2-5: build B for block bi + 1 while the MMAs of block bi run, then
    // drain the accumulators of block bi's M tiles
    const int t128 = threadIdx.x - 64;  // 0..127
    const int q = warp & 3;             // TMEM sub-partition: rows 32q..32q+31 of the M = 128 tile
    const int kpairs = P.K2 / 2;        // K rows (2i, 2i+1) of B, zero beyond i = N
    // B[2i + part][n'] (K-major: row n' = output column, 8-element K chunks), hi and lo
    auto build_b = [&](int bi) -> bool {
      const int c = blockIdx.x + bi * gridDim.x;
      const int bsel = bi & 1;
      const bool w1 = mbar_wait(&bempty[bsel], ((uint32_t)(bi >> 1) & 1) ^ 1, abort_flag);
      if (!__all_sync(0xffffffffu, w1)) {
        if (!w1) atomicCAS(P.err, 0, 13);
        *abort_flag = 1;
        return false;
      }
      uint32_t* bh = reinterpret_cast<uint32_t*>(bbuf + (size_t)bsel * 2 * b_bytes);
      uint32_t* bl = reinterpret_cast<uint32_t*>(bbuf + (size_t)bsel * 2 * b_bytes + b_bytes);
      for (int e = t128; e < 2 * P.Rp * kpairs; e += 128) {
        const int col = e / kpairs, i = e % kpairs;  // output column (r or Rp + r), basis index
        const int r = col < P.Rp ? col : col - P.Rp;
        float2 cv = make_float2(0.f, 0.f);
        if (r < P.R && i < P.N) cv = P.coarse[((size_t)c * P.nrhs + r) * P.N + i];
        // K entries 2i (Re v_i) and 2i+1 (Im v_i): (Re C, -Im C) for Re F, (Im C, Re C) for Im F
        const float k0 = col < P.Rp ? cv.x : cv.y;
        const float k1 = col < P.Rp ? -cv.y : cv.x;
        const float h0 = bf16_round(k0), h1 = bf16_round(k1);
        const size_t word = ((size_t)(2 * i / 8) * 2 * P.Rp + col) * 4 + ((2 * i) & 7) / 2;
        bh[word] = bf16_pair(h0, h1);
        bl[word] = bf16_pair(k0 - h0, k1 - h1);
      }
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      mbar_arrive(&bfull[bsel]);
      return true;
    };
    int64_t n = 0;
    bool stop = nblk > 0 && !build_b(0);
    for (int bi = 0; bi < nblk && !stop; ++bi) {
      const int c = blockIdx.x + bi * gridDim.x;
      if (bi + 1 < nblk && !build_b(bi + 1)) {
        stop = true;
        break;
      }
      for (int t = 0; t < tpb; ++t, ++n) {
        const int acc = (int)(n & 1);
        const uint32_t aph = (uint32_t)(n >> 1) & 1;
        const bool waited = mbar_wait(&tfull[acc], aph, abort_flag);
        if (!__all_sync(0xffffffffu, waited)) {
          if (!waited) atomicCAS(P.err, 0, 14);
          *abort_flag = 1;
          stop = true;
          break;
        }
        fence_after();
        const int k = t * kTileM + q * 32 + lane;  // fine dof within the block
        const bool valid = k < P.K;
        const int sb = k / P.dof, a = k % P.dof;
        const int sf = valid ? P.blk_sites[(size_t)c * P.bv + sb] : 0;
        const uint32_t ta = tmem_base + ((uint32_t)(32 * q) << 16) + acc * acc_cols;
        for (int c0 = 0; c0 < P.Rp; c0 += 16) {
          float vr[16], vi[16];
          tmem_ld16x2(ta + c0, ta + P.Rp + c0, vr, vi);
          if (valid) {
#pragma unroll
            for (int j = 0; j < 16; ++j) {
              const int r = c0 + j;
              if (r < P.R) P.fine[((size_t)sf * P.nrhs + r) * P.dof + a] = make_float2(vr[j], vi[j]);
            }
          }
        }
        fence_before();
        mbar_arrive(&tempty[acc]);
      }
    }
  }
  fence_before();
  __syncthreads();
  if (warp == 1) {
    fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_base), "r"(ncols) : "memory");
  }
}

// basis_blk [c][i][k] (FP64) -> hi / lo [c][Kp/8][Mp][8] BF16, rows 2i = Re v_i, 2i+1 = Im v_i
__global__ void pack_basis_kernel(const double2* __restrict__ B, uint4* __restrict__ hi, uint4* __restrict__ lo,
                                  int64_t Vc, int N, int K, int Kp, int Mp) {
  const int64_t total = Vc * (Kp / 8) * Mp;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int m = (int)(e % Mp);
    const int ch = (int)((e / Mp) % (Kp / 8));
    const int64_t c = e / ((int64_t)Mp * (Kp / 8));
    float h[8], l[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int k = ch * 8 + j;
      float v = 0.f;
      if (m < 2 * N && k < K) {
        const double2 z = B[(c * N + (m >> 1)) * K + k];
        v = (float)((m & 1) ? z.y : z.x);
      }
      h[j] = bf16_round(v);
      l[j] = v - h[j];
    }
    hi[e] = make_uint4(bf16_pair(h[0], h[1]), bf16_pair(h[2], h[3]), bf16_pair(h[4], h[5]), bf16_pair(h[6], h[7]));
    lo[e] = make_uint4(bf16_pair(l[0], l[1]), bf16_pair(l[2], l[3]), bf16_pair(l[4], l[5]), bf16_pair(l[6], l[7]));
  }
}

static int gcd(int a, int b) { return b ? gcd(b, a % b) : a; }

}  // namespace ptc

// Geometry of the tensor-core projection for this aggregation.
struct TcProjGeom {
  int K, Kp, Mp, KS, sps;
};

static TcProjGeom tc_geom(const gmg_agg* h) {
  TcProjGeom g;
  g.K = h->bv * h->dof;
  g.sps = 16 / ptc::gcd(h->dof, 16);  // sites per stage so that a stage is a whole number of K-steps
  if (h->dof * g.sps < 48 && (48 % (h->dof * g.sps)) == 0) g.sps *= 48 / (h->dof * g.sps);
  g.KS = g.sps * h->dof;
  g.Kp = (g.K + g.KS - 1) / g.KS * g.KS;
  g.Mp = 2 * h->N <= 64 ? 64 : 128;
  return g;
}

gmg_status agg_prepare_tc(gmg_agg* h, cudaStream_t s) {
  if (h->basis_tc_ok) return GMG_OK;
  GMG_CHECK(2 * h->N <= 128, GMG_ERR_UNSUPPORTED, "tensor-core projection needs nbasis <= 64");
  const TcProjGeom g = tc_geom(h);
  const int64_t Vc = h->cdims.vol();
  const size_t bytes = (size_t)Vc * (g.Kp / 8) * g.Mp * 16;
  GMG_TRY(h->basis_tc_hi.alloc(bytes));
  GMG_TRY(h->basis_tc_lo.alloc(bytes));
  const int64_t total = Vc * (g.Kp / 8) * g.Mp;
  ptc::pack_basis_kernel<<<(int)std::min<int64_t>((total + 255) / 256, 148 * 64), 256, 0, s>>>(
      h->basis_blk.as<double2>(), h->basis_tc_hi.as<uint4>(), h->basis_tc_lo.as<uint4>(), Vc, h->N, g.K, g.Kp, g.Mp);
  GMG_CUDA(cudaGetLastError());
  h->basis_tc_ok = true;
  return GMG_OK;
}

gmg_status agg_project_tc(gmg_agg* h, int nrhs, const float* fine, float* coarse, cudaStream_t s) {
  GMG_CHECK(nrhs <= 128, GMG_ERR_UNSUPPORTED, "tensor-core projection: at most 128 RHS");
  GMG_CHECK(h->dof % 2 == 0, GMG_ERR_UNSUPPORTED, "tensor-core projection: site dof must be even");
  GMG_TRY(agg_prepare_tc(h, s));
  const TcProjGeom g = tc_geom(h);
  const int Rp = (nrhs + 15) / 16 * 16;
  const uint32_t a_bytes = (uint32_t)(g.KS / 8) * g.Mp * 16;
  const uint32_t b_bytes = (uint32_t)(g.KS / 8) * 2 * Rp * 16;
  const size_t fixed = (3 * 16 + 2 * ptc::kAcc + 1) * 8 + 16 + (size_t)h->bv * 4;
  // raw mode: the fine site rows are bulk-copied into the stage (16-byte aligned rows)
  const uint32_t site_bytes = (uint32_t)nrhs * h->dof * 8;
  const bool aligned = (reinterpret_cast<uintptr_t>(fine) & 15) == 0 && site_bytes % 16 == 0;
  const uint32_t raw_stage = (uint32_t)g.sps * site_bytes;
  // two CTAs per SM (twice the converter and MMA warps) when both TMEM
  // accumulators fit the SM's 512 columns and each CTA keeps 3 stages in half
  // the shared memory; else one CTA with all of it
  uint32_t ncols = 32;
  while (ncols < ptc::kAcc * 2 * (uint32_t)Rp) ncols <<= 1;
  int ctas = 1, raw = 0, stages = 0;
  uint32_t stage_bytes = 0;
  for (int c2 : {2, 1}) {
    if (c2 == 2 && 2 * ncols > 512) continue;
    const size_t cap = c2 == 2 ? 233472 / 2 - 1024 : 227 * 1024;
    raw = aligned && (2 * a_bytes + 2 * b_bytes + raw_stage) * 2 + fixed <= cap ? 1 : 0;
    stage_bytes = 2 * a_bytes + 2 * b_bytes + (raw ? raw_stage : 0u);
    stages = (int)std::min<size_t>(16, (cap - fixed) / stage_bytes);
    ctas = c2;
    if (c2 == 1 || stages >= 3) break;
  }
  GMG_CHECK(stages >= 2, GMG_ERR_UNSUPPORTED, "tensor-core projection: stage does not fit shared memory");
  const size_t smem = (size_t)stages * stage_bytes + (size_t)(3 * stages + 2 * ptc::kAcc + 1) * 8 + 16 + (size_t)h->bv * 4;
  auto kern = ctas == 2 ? ptc::project_tc_kernel<2> : ptc::project_tc_kernel<1>;
  GMG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  if (!h->dev_err.p) {
    GMG_TRY(h->dev_err.alloc(256));
    GMG_CUDA(cudaMemsetAsync(h->dev_err.p, 0, 256, s));
  }
  int dev = 0, nsm = 148;
  GMG_CUDA(cudaGetDevice(&dev));
  GMG_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  ptc::Params P;
  P.ahi = h->basis_tc_hi.as<uint16_t>();
  P.alo = h->basis_tc_lo.as<uint16_t>();
  P.fine = reinterpret_cast<const float2*>(fine);
  P.blk_sites = h->blk_sites.as<int32_t>();
  P.coarse = reinterpret_cast<float2*>(coarse);
  P.err = h->dev_err.as<int>();
  P.Vc = (int)h->cdims.vol();
  P.N = h->N;
  P.dof = h->dof;
  P.bv = h->bv;
  P.nrhs = nrhs;
  P.R = nrhs;
  P.Rp = Rp;
  P.Kp = g.Kp;
  P.Mp = g.Mp;
  P.KS = g.KS;
  P.sps = g.sps;
  P.stages = stages;
  P.aligned16 = ((reinterpret_cast<uintptr_t>(fine) & 15) == 0 && (h->dof % 2) == 0) ? 1 : 0;
  P.raw = raw;

  {
    KernelTimer kt("project_tc", s);
    kern<<<std::min(P.Vc, nsm * ctas), ptc::kThreads, smem, s>>>(P);
  }
  GMG_CUDA(cudaGetLastError());
  return GMG_OK;
}

gmg_status agg_promote_tc(gmg_agg* h, int nrhs, const float* coarse, float* fine, cudaStream_t s) {
  GMG_CHECK(nrhs <= 128, GMG_ERR_UNSUPPORTED, "tensor-core promotion: at most 128 RHS");
  GMG_TRY(agg_prepare_tc(h, s));
  const TcProjGeom g = tc_geom(h);
  const int Rp = (nrhs + 15) / 16 * 16;
  const int K2 = (2 * h->N + 15) / 16 * 16;  // <= Mp: the packed basis rows beyond 2N are zero
  const uint32_t a_bytes = (uint32_t)(ptc::kTileM / 8) * g.Mp * 16;
  const uint32_t b_bytes = (uint32_t)(K2 / 8) * 2 * Rp * 16;
  const size_t fixed = 4 * (size_t)b_bytes + (2 * 16 + 10 + 1) * 8 + 16;
  GMG_CHECK(fixed < 227 * 1024, GMG_ERR_UNSUPPORTED, "tensor-core promotion: coarse tile does not fit");
  // two CTAs per SM when both TMEM accumulators fit and each keeps 2 stages in
  // half the shared memory; else one CTA with all of it
  uint32_t ncols = 32;
  while (ncols < 2 * 2 * (uint32_t)Rp) ncols <<= 1;
  int ctas = 1, stages = 0;
  for (int c2 : {2, 1}) {
    if (c2 == 2 && 2 * ncols > 512) continue;
    const size_t cap = c2 == 2 ? 233472 / 2 - 1024 : 227 * 1024;
    if (fixed >= cap) continue;
    stages = (int)std::min<size_t>(16, (cap - fixed) / (2 * a_bytes));
    ctas = c2;
    if (c2 == 1 || stages >= 2) break;
  }
  GMG_CHECK(stages >= 2, GMG_ERR_UNSUPPORTED, "tensor-core promotion: stage does not fit shared memory");
  const size_t smem = (size_t)stages * 2 * a_bytes + 4 * (size_t)b_bytes + (size_t)(2 * stages + 10 + 1) * 8 + 16;
  auto kern = ctas == 2 ? ptc::promote_tc_kernel<2> : ptc::promote_tc_kernel<1>;
  GMG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  if (!h->dev_err.p) {
    GMG_TRY(h->dev_err.alloc(256));
    GMG_CUDA(cudaMemsetAsync(h->dev_err.p, 0, 256, s));
  }
  int dev = 0, nsm = 148;
  GMG_CUDA(cudaGetDevice(&dev));
  GMG_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  ptc::PParams P;
  P.ahi = h->basis_tc_hi.as<uint16_t>();
  P.alo = h->basis_tc_lo.as<uint16_t>();
  P.coarse = reinterpret_cast<const float2*>(coarse);
  P.blk_sites = h->blk_sites.as<int32_t>();
  P.fine = reinterpret_cast<float2*>(fine);
  P.err = h->dev_err.as<int>();
  P.Vc = (int)h->cdims.vol();
  P.N = h->N;
  P.dof = h->dof;
  P.bv = h->bv;
  P.nrhs = nrhs;
  P.R = nrhs;
  P.Rp = Rp;
  P.K = g.K;
  P.Kp = g.Kp;
  P.Mp = g.Mp;
  P.K2 = K2;
  P.stages = stages;

  {
    KernelTimer kt("promote_tc", s);
    kern<<<std::min(P.Vc, nsm * ctas), ptc::kPThreads, smem, s>>>(P);
  }
  GMG_CUDA(cudaGetLastError());
  return GMG_OK;
}

}  // namespace gmg

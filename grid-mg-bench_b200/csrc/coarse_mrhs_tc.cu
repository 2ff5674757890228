// coarse_mrhs_tc.cu -- multi-RHS coarse stencil on the 5th-generation tensor cores.
//
// Restates the multi-RHS coarse operator M / Mdag / Mdir / Mdiag
// (include/CoarsenedMatrixUpstreamImprovedDirsaveLutMRHS.h:736-947) as, per
// coarse site x, a sum over the 9 stencil points of complex products
//
//     out(x)[r][b] = sum_p sum_bb A_p(x)[b][bb] in(nbr_p(x))[r][bb]
//
// decomposed into one real MMA per point and K-step, with the link rows
// interleaved (row 2b = Re A[b][.], row 2b+1 = Im A[b][.]):
//
//     D (2N x 2R) += [Re A; Im A] (2N x N)  .  [Xr^T | Xi^T] (N x 2R)
//     out_r = D[2b][r] - D[2b+1][R+r],   out_i = D[2b][R+r] + D[2b+1][r]
//
// so the links are read once in their compact (re, im) form and every
// operand is a straight copy from HBM.  BF16 or FP16 operands, FP32
// accumulation in tensor memory (TMEM), tcgen05.mma issued by one thread.
//
// Kernel structure (one persistent CTA per SM, 11 warps):
//   warps 0, 10  producers: stage-sequence numbers alternate between them; one
//                stage = 1-4 stencil points of one site: one bulk copy of
//                the points' contiguous link tiles and one per neighbour tile
//                (cp.async.bulk + mbarrier transaction counts)
//   warp 1       TMEM allocator + MMA issuer (one elected thread); accumulates
//                the 9 points of a site into one of up to 4 TMEM buffers
//   warps 2-9    epilogue, two warps per TMEM sub-partition: tcgen05.ld the
//                accumulator, recombine (re, im) with one lane-pair shuffle,
//                apply G5C for Mdag, write FP32 output
// Every mbarrier wait is bounded in time: on time-out the kernel records an
// error code, stops issuing work, drains its own copies and MMAs, frees TMEM
// and returns.
//
// Global layouts (prepared once per link set / per apply):
//   links  [V][9][Ks][Mr][8]   halves, Ks = ceil(N/8) K-chunks of Mr = 2N
//          rows (rounded up to 8), interleaved as above, zero-padded beyond 2N
//          and N (the MMA's M = 64 / 128 rows and whole K-steps are read
//          across the tile boundaries, see link_geometry)
//   packed [V][Kc][2Rp][8]     halves, Kc = ceil16(N)/8: rows n < Rp = Re
//          in[r=n][.], Rp <= n < 2Rp = Im in[r=n-Rp][.]  (Rp = R rounded up
//          to 16), zero beyond N and R
// Both are the canonical no-swizzle K-major core-matrix layout
// (8 rows x 16 B per core matrix): SBO = 128 B, LBO = rows * 16 B.
#include <algorithm>
#include <mutex>

#include "gmg_internal.cuh"

namespace gmg {

namespace tc {

constexpr int kWarps = 11;  // producer, MMA issuer, 8 epilogue warps (two per TMEM sub-partition), producer
constexpr int kThreads = kWarps * 32;
constexpr int kAccBufs = 4;  // TMEM accumulator buffers (fewer when 2*Rp columns do not fit 4 times)
constexpr int kEpiThreads = 256;
constexpr long long kTimeoutCycles = 4000000000LL;  // ~2 s at 2 GHz

enum : int { ERR_NONE = 0, ERR_TIMEOUT_PRODUCER = 1, ERR_TIMEOUT_MMA = 2, ERR_TIMEOUT_EPILOGUE = 3 };

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

// bounded wait: false after kTimeoutCycles or when another role aborted
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, volatile int* abort_flag) {
  if (mbar_try_wait(bar, parity)) return true;
  const long long t0 = clock64();
  while (true) {
    if (mbar_try_wait(bar, parity)) return true;
    if (*abort_flag) return false;
    if (clock64() - t0 > kTimeoutCycles) return false;
  }
}

// wait without the abort short-cut (used to drain our own copies / MMAs)
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
  const uint64_t a = (smem_u32(smem) >> 4) & 0x3FFF;
  uint64_t d = a;
  d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
  d |= (uint64_t)1 << 46;  // descriptor version for sm_100
  // base offset 0, lbo mode 0, layout type 0 = SWIZZLE_NONE
  return d;
}

__device__ __forceinline__ void mma_f16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                        uint32_t accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float* v) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
      "%14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
        "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]),
        "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]),
        "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void named_bar(int id, int nthreads) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
}

// named barrier that also ORs a predicate over the participating threads
__device__ __forceinline__ bool named_bar_or(int id, int nthreads, bool pred) {
  uint32_t r;
  asm volatile(
      "{\n .reg .pred p, q;\n setp.ne.u32 p, %1, 0;\n bar.red.or.pred q, %2, %3, p;\n selp.u32 %0, 1, 0, q;\n}\n"
      : "=r"(r)
      : "r"((uint32_t)pred), "r"(id), "r"(nthreads)
      : "memory");
  return r != 0;
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
      "%14, %15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
        "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// two 16-column TMEM loads (real-part and imaginary-part columns), one wait
__device__ __forceinline__ void tmem_ld16x2(uint32_t ta, uint32_t tb, float* va, float* vb) {
  uint32_t a[16], b[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
      "%14, %15}, [%16];"
      : "=r"(a[0]), "=r"(a[1]), "=r"(a[2]), "=r"(a[3]), "=r"(a[4]), "=r"(a[5]), "=r"(a[6]), "=r"(a[7]),
        "=r"(a[8]), "=r"(a[9]), "=r"(a[10]), "=r"(a[11]), "=r"(a[12]), "=r"(a[13]), "=r"(a[14]),
        "=r"(a[15])
      : "r"(ta));
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
      "%14, %15}, [%16];"
      : "=r"(b[0]), "=r"(b[1]), "=r"(b[2]), "=r"(b[3]), "=r"(b[4]), "=r"(b[5]), "=r"(b[6]), "=r"(b[7]),
        "=r"(b[8]), "=r"(b[9]), "=r"(b[10]), "=r"(b[11]), "=r"(b[12]), "=r"(b[13]), "=r"(b[14]),
        "=r"(b[15])
      : "r"(tb));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) {
    va[i] = __uint_as_float(a[i]);
    vb[i] = __uint_as_float(b[i]);
  }
}

struct Params {
  const uint16_t* links;   // [V][9][Ks][Mr][8]
  const uint16_t* packed;  // [V][Kc][2Rp][8]
  const int32_t* nbr;      // [9][V]: input index of point p's neighbour of output index o
  const int32_t* site_map; // [V] link site of output index o (null: o itself)
  const int32_t* active;   // nullable
  float2* out;             // [V][nrhs][N]
  int* err;                // device error word
  int V, N, nrhs, R, Rp, Kc, Mp, p0, p1, g5, stages, kind, pps;
  int Ks, Mr;              // stored link tile: Ks K-chunks of Mr rows (see link_geometry)
};

// The MMAs of one stage as straight-line code: PPS points x KH K-steps.  Issuing
// tcgen05.mma from rolled loops with data-dependent control flow between the
// instructions measured several times slower per MMA than unrolled sequences.
template <int PPS, int KH>
__device__ __forceinline__ void issue_stage(uint32_t dt, uint64_t ad, uint64_t bd, uint32_t a_pt, uint32_t b_pt,
                                            uint32_t a_ks, uint32_t b_ks, uint32_t idesc, bool first) {
#pragma unroll
  for (int pp = 0; pp < PPS; ++pp)
#pragma unroll
    for (int ks = 0; ks < KH; ++ks)
      mma_f16(dt, ad + pp * a_pt + ks * a_ks, bd + pp * b_pt + ks * b_ks, idesc, (first && pp == 0 && ks == 0) ? 0u : 1u);
}

template <int PPS>
__device__ __forceinline__ void issue_stage_kh(int kh, uint32_t dt, uint64_t ad, uint64_t bd, uint32_t a_pt,
                                               uint32_t b_pt, uint32_t a_ks, uint32_t b_ks, uint32_t idesc, bool first) {
  switch (kh) {
    case 1: issue_stage<PPS, 1>(dt, ad, bd, a_pt, b_pt, a_ks, b_ks, idesc, first); break;
    case 2: issue_stage<PPS, 2>(dt, ad, bd, a_pt, b_pt, a_ks, b_ks, idesc, first); break;
    case 3: issue_stage<PPS, 3>(dt, ad, bd, a_pt, b_pt, a_ks, b_ks, idesc, first); break;
    default: issue_stage<PPS, 4>(dt, ad, bd, a_pt, b_pt, a_ks, b_ks, idesc, first); break;
  }
}


// Shared memory: `stages` stages of pps link tiles followed by pps neighbour
// tiles, then the mbarriers, the TMEM address, the abort flag and the
// producer's neighbour-index table.
template <int CTAS>  // CTAs per SM the register budget allows (1 or 2)
__global__ void __launch_bounds__(kThreads, CTAS) coarse_mrhs_tc_kernel(const Params P) {
  extern __shared__ __align__(1024) unsigned char smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t link_bytes = (uint32_t)P.Ks * P.Mr * 16;     // one stencil point of one site
  const uint32_t vec_bytes = (uint32_t)P.Kc * 2 * P.Rp * 16;  // one neighbour tile
  const int pps = P.pps;                                      // stencil points per stage
  const uint32_t stage_bytes = (uint32_t)pps * (link_bytes + vec_bytes);
  const int ngroups = (P.p1 - P.p0) / pps;                    // pps divides the point count

  unsigned char* stage_base = smem;
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + (size_t)P.stages * stage_bytes);
  uint64_t* full = bars;
  uint64_t* empty = full + P.stages;
  uint64_t* tfull = empty + P.stages;
  uint64_t* tempty = tfull + kAccBufs;
  uint64_t* drain = tempty + kAccBufs;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(drain + 1);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);
  int* nbr_s = reinterpret_cast<int*>(tmem_slot + 4);  // [2][32][9] neighbour indices of the two producers
  int* lsite_s = nbr_s + 2 * 32 * 9;                   // [2][32] link sites of the two producers

  const uint32_t acc_cols = 2 * P.Rp;
  const int nacc = (int)min((uint32_t)kAccBufs, 512u / acc_cols);  // >= 2 since Rp <= 128
  uint32_t ncols_alloc = 32;
  while (ncols_alloc < nacc * acc_cols) ncols_alloc <<= 1;

  if (threadIdx.x == 0) {
    for (int s = 0; s < P.stages; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int a = 0; a < kAccBufs; ++a) {
      mbar_init(&tfull[a], 1);
      mbar_init(&tempty[a], kEpiThreads);
    }
    mbar_init(drain, 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(ncols_alloc)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tmem_base = *tmem_slot;

  // sites of this CTA: blockIdx.x, blockIdx.x + gridDim.x, ...
  const int nsites = (P.V - (int)blockIdx.x + (int)gridDim.x - 1) / (int)gridDim.x;

  if (warp == 0 || warp == kWarps - 1) {
    // ------------------------------------------------------------ producers
    // Two producer warps fill alternate stages: stage-sequence number n (one
    // per group of pps points of one site, in the order the MMA issuer
    // consumes them) goes to producer n % 2, stage n % stages (stages is even).
    // Each warp stages the neighbour indices of 32 sites at a time in its own
    // shared-memory table (one parallel load), so its issuing lane never waits
    // on a dependent global load between two stages.  One stage = one bulk copy
    // of the pps (contiguous) link tiles and one per neighbour tile.
    const int pid = warp == 0 ? 0 : 1;
    int* my_nbr = nbr_s + pid * 32 * 9;
    int* my_lsite = lsite_s + pid * 32;
    int64_t last = -1;
    bool stop = false;
    // the first `stages` sequence numbers fill stages that have never been used:
    // their link tiles (which do not depend on the pack) are requested before
    // the wait on the pack grid, and only their neighbour tiles after it
    const int64_t npre = min((int64_t)P.stages, (int64_t)nsites * ngroups);
    for (int i0 = 0; i0 < nsites && !stop; i0 += 32) {
      const int cnt = min(32, nsites - i0);
      __syncwarp();
      if (lane < cnt) {
        const int site = blockIdx.x + (i0 + lane) * gridDim.x;
#pragma unroll
        for (int p = 0; p < 9; ++p) my_nbr[lane * 9 + p] = __ldg(&P.nbr[(size_t)p * P.V + site]);
        my_lsite[lane] = P.site_map ? __ldg(&P.site_map[site]) : site;
      }
      if (i0 == 0) {
        __syncwarp();
        if (lane == 0) {
          // npre <= stages <= 32 and ngroups >= 1, so these sites are in this first table
          for (int64_t n = pid; n < npre; n += 2) {
            const int j = (int)(n / ngroups), g = (int)(n % ngroups);
            const int stage = (int)n;
            const int pf = P.p0 + g * pps;
            mbar_expect_tx(&full[stage], stage_bytes);
            bulk_g2s(stage_base + (size_t)stage * stage_bytes,
                     P.links + ((size_t)my_lsite[j] * 9 + pf) * (link_bytes / 2), pps * link_bytes, &full[stage]);
          }
        }
        // launched as a programmatic dependent of the vector pack: everything
        // above overlaps the pack's tail; the packed vectors are read only
        // after the pack grid has completed (a no-op for a plain launch)
        asm volatile("griddepcontrol.wait;" ::: "memory");
      }
      __syncwarp();
      if (lane == 0) {
        for (int j = 0; j < cnt && !stop; ++j) {
          const int lsite = my_lsite[j];
          for (int g = 0; g < ngroups; ++g) {
            const int64_t n = (int64_t)(i0 + j) * ngroups + g;
            if ((int)(n & 1) != pid) continue;
            const int stage = (int)(n % P.stages);
            const uint32_t phase = (uint32_t)((n / P.stages) & 1);
            unsigned char* st = stage_base + (size_t)stage * stage_bytes;
            const int pf = P.p0 + g * pps;
            if (n >= npre) {
              if (!mbar_wait(&empty[stage], phase ^ 1, abort_flag)) {
                atomicCAS(P.err, 0, ERR_TIMEOUT_PRODUCER);
                *abort_flag = 1;
                stop = true;
                break;
              }
              mbar_expect_tx(&full[stage], stage_bytes);
              bulk_g2s(st, P.links + ((size_t)lsite * 9 + pf) * (link_bytes / 2), pps * link_bytes, &full[stage]);
            }
            for (int pp = 0; pp < pps; ++pp) {
              const int nb = my_nbr[j * 9 + pf + pp];
              bulk_g2s(st + pps * link_bytes + pp * vec_bytes, P.packed + (size_t)nb * (vec_bytes / 2), vec_bytes,
                       &full[stage]);
            }
            last = n;
          }
        }
      }
      stop = __shfl_sync(0xffffffffu, stop, 0);
    }
    if (lane == 0) {
      // drain: wait for this producer's copies of the last `stages` sequence numbers to land
      for (int64_t n = last; n >= 0 && n > last - P.stages; --n) {
        if ((int)(n & 1) != pid) continue;
        mbar_drain(&full[n % P.stages], (uint32_t)((n / P.stages) & 1));
      }
    }
  } else if (warp == 1) {
    // ------------------------------------------------------------ MMA issuer
    if (lane == 0) {
      const uint32_t idesc = (1u << 4)                            // D format F32
                             | ((uint32_t)P.kind << 7)            // A format (0 F16, 1 BF16)
                             | ((uint32_t)P.kind << 10)           // B format
                             | ((uint32_t)(2 * P.Rp) >> 3) << 17  // N
                             | ((uint32_t)P.Mp >> 4) << 24;       // M
      // Descriptors advance by adding 16-byte units to their start-address field.
      const uint64_t adesc0 = make_desc(stage_base, (uint32_t)P.Mr * 16, 128);
      const uint64_t bdesc0 = make_desc(stage_base + (size_t)pps * link_bytes, (uint32_t)(2 * P.Rp) * 16, 128);
      const uint32_t st_units = stage_bytes >> 4, a_pt = link_bytes >> 4, b_pt = vec_bytes >> 4;
      const uint32_t a_ks = 2 * P.Mr, b_ks = 4 * P.Rp;  // two 16-byte K-chunks per MMA
      const int kh = P.Kc / 2;
      int stage = 0;
      uint32_t phase = 0, st_off = 0;
      bool ok = true;
      for (int i = 0; i < nsites && ok; ++i) {
        const int acc = i % nacc;
        const uint32_t aphase = (uint32_t)(i / nacc) & 1;
        if (!mbar_wait(&tempty[acc], aphase ^ 1, abort_flag)) { ok = false; break; }
        fence_after();
        const uint32_t dt = tmem_base + acc * acc_cols;
        for (int g = 0; g < ngroups; ++g) {
          if (!mbar_wait(&full[stage], phase, abort_flag)) { ok = false; break; }
          fence_after();
          switch (pps) {
            case 4: issue_stage_kh<4>(kh, dt, adesc0 + st_off, bdesc0 + st_off, a_pt, b_pt, a_ks, b_ks, idesc, g == 0); break;
            case 3: issue_stage_kh<3>(kh, dt, adesc0 + st_off, bdesc0 + st_off, a_pt, b_pt, a_ks, b_ks, idesc, g == 0); break;
            case 2: issue_stage_kh<2>(kh, dt, adesc0 + st_off, bdesc0 + st_off, a_pt, b_pt, a_ks, b_ks, idesc, g == 0); break;
            default: issue_stage_kh<1>(kh, dt, adesc0 + st_off, bdesc0 + st_off, a_pt, b_pt, a_ks, b_ks, idesc, g == 0);
          }
          mma_commit(&empty[stage]);
          if (++stage == P.stages) {
            stage = 0;
            phase ^= 1;
            st_off = 0;
          } else {
            st_off += st_units;
          }
        }
        if (!ok) break;
        mma_commit(&tfull[acc]);
      }
      if (!ok) {
        atomicCAS(P.err, 0, ERR_TIMEOUT_MMA);
        *abort_flag = 1;
      }
      // drain our own MMAs before TMEM is freed
      mma_commit(drain);
      mbar_drain(drain, 0);
    }
  } else {
    // ------------------------------------------------------------ epilogue (warps 2..9)
    // Link rows are interleaved (2b = Re A[b], 2b+1 = Im A[b]), so accumulator
    // rows 2b and 2b+1 sit in neighbouring lanes of one warp and the complex
    // recombination is one lane-pair exchange:
    //   out_r = D[2b][r] - D[2b+1][Rp+r],   out_i = D[2b][Rp+r] + D[2b+1][r]
    // The even lane writes r in [c, c+8) of every 16-column chunk, the odd lane [c+8, c+16).
    // Two warps share each TMEM sub-partition and take alternate 16-column chunks.
    const int q = warp & 3;              // TMEM sub-partition of this warp
    const int half = (warp - 2) >> 2;    // 0 or 1: which alternate chunks
    const int rows_per_warp = P.Mp / 4;  // 16 (M=64) or 32 (M=128)
    const int row = q * rows_per_warp + lane;
    const int b = row >> 1;
    const bool odd = row & 1;
    const bool valid = lane < rows_per_warp && row < 2 * P.N;
    const float sg = (P.g5 && b >= P.N / 2) ? -1.f : 1.f;
    for (int i = 0; i < nsites; ++i) {
      const int site = blockIdx.x + i * gridDim.x;
      const int acc = i % nacc;
      const uint32_t aphase = (uint32_t)(i / nacc) & 1;
      const bool waited = mbar_wait(&tfull[acc], aphase, abort_flag);
      if (!__all_sync(0xffffffffu, waited)) {  // the warp leaves together
        if (!waited) atomicCAS(P.err, 0, ERR_TIMEOUT_EPILOGUE);
        *abort_flag = 1;
        break;
      }
      fence_after();
      const uint32_t ta = tmem_base + ((uint32_t)(32 * q) << 16) + acc * acc_cols;
      float2* orow = P.out + (size_t)site * P.nrhs * P.N + b;
      for (int c = 16 * half; c < P.Rp; c += 32) {
        float vr[16], vi[16];
        tmem_ld16x2(ta + c, ta + P.Rp + c, vr, vi);
        float pr[8], pi[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          pr[j] = __shfl_xor_sync(0xffffffffu, odd ? vr[j] : vr[8 + j], 1);
          pi[j] = __shfl_xor_sync(0xffffffffu, odd ? vi[j] : vi[8 + j], 1);
        }
        if (valid) {
#pragma unroll
          for (int j = 0; j < 8; ++j) {
            const int r = c + (odd ? 8 : 0) + j;
            if (r < P.R) {
              const float re = odd ? pr[j] - vi[8 + j] : vr[j] - pi[j];
              const float im = odd ? pi[j] + vr[8 + j] : vi[j] + pr[j];
              const int slot = P.active ? __ldg(&P.active[r]) : r;
              orow[(size_t)slot * P.N] = make_float2(sg * re, sg * im);
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
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_base), "r"(ncols_alloc)
                 : "memory");
  }
}

// ---------------------------------------------------------------- packers
__device__ __forceinline__ uint16_t to_half_bits(float x, int kind) {
  if (kind == GMG_BF16) return __bfloat16_as_ushort(__float2bfloat16_rn(x));
  return __half_as_ushort(__float2half_rn(x));
}
// (a, b) rounded to the 16-bit kind with one paired conversion; a in the low half
__device__ __forceinline__ uint32_t to_half_pair(float a, float b, int kind) {
  if (kind == GMG_BF16) {
    const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<const uint32_t*>(&h);
  }
  const __half2 h = __floats2half2_rn(a, b);
  return *reinterpret_cast<const uint32_t*>(&h);
}

// links (exchange layout, FP64) -> [V][9][Ks][Mr][8] halves (Kc, Mp: the chunk and row counts stored)
__global__ void pack_links_kernel(const double2* __restrict__ A, uint4* __restrict__ dst, int V, int N, int Kc,
                                  int Mp, int kind) {
  const int64_t total = (int64_t)V * 9 * Kc * Mp;  // one 16-byte row each
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int m = (int)(e % Mp);
    const int kc = (int)((e / Mp) % Kc);
    const int p = (int)((e / ((int64_t)Mp * Kc)) % 9);
    const int64_t s = e / ((int64_t)Mp * Kc * 9);
    uint16_t h[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int bb = kc * 8 + j;
      float v = 0.f;
      if (m < 2 * N && bb < N) {  // interleaved rows: 2b = Re A[b][.], 2b+1 = Im A[b][.]
        const double2 a = A[(((int64_t)p * V + s) * N + (m >> 1)) * N + bb];
        v = (float)((m & 1) ? a.y : a.x);
      }
      h[j] = to_half_bits(v, kind);
    }
    uint4 o;
    o.x = h[0] | ((uint32_t)h[1] << 16);
    o.y = h[2] | ((uint32_t)h[3] << 16);
    o.z = h[4] | ((uint32_t)h[5] << 16);
    o.w = h[6] | ((uint32_t)h[7] << 16);
    dst[e] = o;
  }
}

// vectors (FP32 [V][nrhs][N]) -> [V][Kc][2Rp][8] halves, G5C applied on input.
// One thread per (site, K-chunk, rhs), K chunk fastest: the Kc threads of one
// (site, RHS) read its row of N complex numbers contiguously (a warp reads 2 KB
// in one run) and each writes the real-part row r and the imaginary-part row
// Rp + r of its chunk, so a warp's writes are whole 128-byte runs.  Indices are
// 32-bit with the chunk count a compile-time constant: one 32-bit division per
// item (64-bit divisions, expanded in software, had made the kernel
// instruction-bound).
// vectors (FP32 [V][nrhs][N]) -> [V][Kc][2Rp][8] halves, G5C applied on input.
// One thread per (site, K-chunk, rhs), K chunk fastest: the Kc threads of one
// (site, RHS) read its row of N complex numbers contiguously (a warp reads 2 KB
// in one run) and each writes the real-part row r and the imaginary-part row
// Rp + r of its chunk, so a warp's writes are whole 128-byte runs.  Indices are
// 32-bit with the chunk count a compile-time constant: one 32-bit division per
// item (64-bit divisions, expanded in software, had made the kernel
// instruction-bound).  Two items per thread, both loaded before either is
// stored, measured slower (14.3 against 12.4 us on 8^4 x 32 x 32).
template <int KC>
__global__ void __launch_bounds__(256) pack_vec_kernel(const float2* __restrict__ in, uint4* __restrict__ dst,
                                                       const int32_t* __restrict__ active, int V, int N, int nrhs,
                                                       int R, int Rp, int kind, int g5, int aligned16) {
  // the stencil launched after this kernel may start its prologue now (it
  // waits for this grid's completion before reading the packed vectors)
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  const uint32_t per_site = (uint32_t)KC * Rp;
  const uint32_t total = (uint32_t)V * per_site;
  for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < total; e += gridDim.x * blockDim.x) {
    const uint32_t s = e / per_site;
    const uint32_t rem = e - s * per_site;
    const int kc = (int)(rem % KC);
    const int r = (int)(rem / KC);
    uint32_t pr[4], pi[4];
    if (r < R) {
      const int slot = active ? __ldg(&active[r]) : r;
      const float2* src = in + ((size_t)s * nrhs + slot) * N + kc * 8;
      float2 x[8];
      if (aligned16 && (N & 1) == 0 && kc * 8 + 8 <= N) {
        // `in` is 16-byte aligned (checked on the host), N and 8*kc are even, and the
        // chunk lies inside the row (the last chunk of N = 24, 40, ... is partial)
        const float4* s4 = reinterpret_cast<const float4*>(src);
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const float4 v = __ldg(s4 + j);
          x[2 * j] = make_float2(v.x, v.y);
          x[2 * j + 1] = make_float2(v.z, v.w);
        }
      } else {
#pragma unroll
        for (int j = 0; j < 8; ++j) x[j] = (kc * 8 + j < N) ? src[j] : make_float2(0.f, 0.f);
      }
      float re[8], im[8];
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const int bb = kc * 8 + j;
        re[j] = 0.f;
        im[j] = 0.f;
        if (bb < N) {
          re[j] = x[j].x;
          im[j] = x[j].y;
          if (g5 && bb >= N / 2) { re[j] = -re[j]; im[j] = -im[j]; }
        }
      }
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        pr[j] = to_half_pair(re[2 * j], re[2 * j + 1], kind);
        pi[j] = to_half_pair(im[2 * j], im[2 * j + 1], kind);
      }
    } else {
#pragma unroll
      for (int j = 0; j < 4; ++j) pr[j] = pi[j] = 0;
    }
    uint4* row = dst + ((size_t)s * KC + kc) * 2 * Rp;
    row[r] = make_uint4(pr[0], pr[1], pr[2], pr[3]);
    row[Rp + r] = make_uint4(pi[0], pi[1], pi[2], pi[3]);
  }
}

// The same packing with coalesced loads, for all RHS (no active list), N a
// multiple of 8 and a 16-byte aligned input.  A warp takes 256 consecutive
// complex numbers of the input (2 KB): load j of lane l is the 16 bytes at
// complex 64 j + 2 l, so each load instruction of the warp reads 512
// contiguous bytes.  A 4 x 4 transpose inside each quad of lanes (two
// shuffle stages) then gives lane k of quad q the 8 consecutive complex
// numbers 64 k + 8 q .. + 7: one packed chunk, which it converts and stores
// as the generic kernel does.  Rows r >= nrhs of the padded RHS dimension and
// the chunks kc >= N / 8 (b >= N) are written as zeros by a second loop.
template <int KC>
__global__ void __launch_bounds__(256) pack_vec_coalesced_kernel(const float4* __restrict__ in,
                                                                 uint4* __restrict__ dst, int V, int N, int nrhs,
                                                                 int Rp, int kind, int g5) {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  const uint32_t total = (uint32_t)V * (uint32_t)nrhs * (uint32_t)N;  // complex numbers, < 2^31
  const int lane = threadIdx.x & 31, k = lane & 3, q = lane >> 2;
  const uint32_t nwarps = gridDim.x * (blockDim.x >> 5);
  for (uint32_t base = (blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) * 256u; base < total;
       base += nwarps * 256u) {
    float4 x[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const uint32_t c = base + 64u * j + 2u * lane;
      x[j] = c < total ? __ldg(in + (c >> 1)) : make_float4(0.f, 0.f, 0.f, 0.f);
    }
    // transpose (register j, lane k) within the quad: x[m] <- lane m's x[k]
#pragma unroll
    for (int b = 2; b >= 1; b >>= 1) {
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        if (j & b) continue;
        const bool hi = (k & b) != 0;
        const float4 send = hi ? x[j] : x[j ^ b];
        float4 got;
        got.x = __shfl_xor_sync(0xffffffffu, send.x, b);
        got.y = __shfl_xor_sync(0xffffffffu, send.y, b);
        got.z = __shfl_xor_sync(0xffffffffu, send.z, b);
        got.w = __shfl_xor_sync(0xffffffffu, send.w, b);
        if (hi)
          x[j] = got;
        else
          x[j ^ b] = got;
      }
    }
    const uint32_t c0 = base + 64u * k + 8u * q;
    if (c0 < total) {
      const uint32_t row = c0 / (uint32_t)N;  // site * nrhs + r
      const int b0 = (int)(c0 - row * (uint32_t)N);
      const uint32_t s = row / (uint32_t)nrhs;
      const int r = (int)(row - s * (uint32_t)nrhs);
      float re[8], im[8];
#pragma unroll
      for (int m = 0; m < 4; ++m) {
        re[2 * m] = x[m].x;
        im[2 * m] = x[m].y;
        re[2 * m + 1] = x[m].z;
        im[2 * m + 1] = x[m].w;
      }
      if (g5) {
#pragma unroll
        for (int i = 0; i < 8; ++i)
          if (b0 + i >= N / 2) {
            re[i] = -re[i];
            im[i] = -im[i];
          }
      }
      uint32_t pr[4], pi[4];
#pragma unroll
      for (int m = 0; m < 4; ++m) {
        pr[m] = to_half_pair(re[2 * m], re[2 * m + 1], kind);
        pi[m] = to_half_pair(im[2 * m], im[2 * m + 1], kind);
      }
      uint4* rowp = dst + ((size_t)s * KC + (b0 >> 3)) * 2 * Rp;
      rowp[r] = make_uint4(pr[0], pr[1], pr[2], pr[3]);
      rowp[Rp + r] = make_uint4(pi[0], pi[1], pi[2], pi[3]);
    }
  }
  // zeros: padded rows r in [nrhs, Rp) of every chunk, and chunks kc >= N / 8 of rows r < nrhs
  const int kfull = N / 8, npad = Rp - nrhs;
  const uint32_t per_site = (uint32_t)KC * npad + (uint32_t)(KC - kfull) * nrhs;
  const uint32_t zitems = (uint32_t)V * per_site;
  const uint4 z = make_uint4(0u, 0u, 0u, 0u);
  for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < zitems; e += gridDim.x * blockDim.x) {
    const uint32_t s = e / per_site;
    const int rem = (int)(e - s * per_site);
    int kc, r;
    if (rem < KC * npad) {
      kc = rem / npad;
      r = nrhs + (rem - kc * npad);
    } else {
      const int t = rem - KC * npad;
      kc = kfull + t / nrhs;
      r = t - (kc - kfull) * nrhs;
    }
    uint4* rowp = dst + ((size_t)s * KC + kc) * 2 * Rp;
    rowp[r] = z;
    rowp[Rp + r] = z;
  }
}

inline int round_up(int x, int m) { return (x + m - 1) / m * m; }

// pack the vectors of one apply (G5C on input when g5).  (Two variants did not
// beat this one on the 8^4 x 32 x 32 apply, 15.5 us: one thread per 16 input
// bytes with 4-byte stores, 23 us; two chunks per thread with all eight loads
// issued first, 15.7 us.)
inline gmg_status launch_pack(const float* in, uint4* packed, const int32_t* active, int V, int N, int nrhs,
                              int R, int Rp, int Kc, int kind, bool g5, cudaStream_t s) {
  const int64_t rows = (int64_t)V * Kc * Rp;
  GMG_CHECK(rows < ((int64_t)1 << 31), GMG_ERR_UNSUPPORTED,
            "tensor-core coarse stencil: coarse volume x packed RHS rows exceeds 2^31");
  const int grid = (int)std::min<int64_t>((rows + 255) / 256, 148 * 64);
  const float2* src = reinterpret_cast<const float2*>(in);
  const int a16 = (reinterpret_cast<uintptr_t>(in) & 15) == 0 ? 1 : 0;
  const int64_t total = (int64_t)V * nrhs * N;
  if (!active && R == nrhs && N % 8 == 0 && a16 && total < ((int64_t)1 << 31)) {
    // one warp per 256 input complex numbers, 8 warps per CTA
    const int cgrid = (int)std::min<int64_t>((total + 2047) / 2048, 148 * 32);
    const float4* s4 = reinterpret_cast<const float4*>(in);
    switch (Kc) {
      case 2: pack_vec_coalesced_kernel<2><<<cgrid, 256, 0, s>>>(s4, packed, V, N, nrhs, Rp, kind, g5); break;
      case 4: pack_vec_coalesced_kernel<4><<<cgrid, 256, 0, s>>>(s4, packed, V, N, nrhs, Rp, kind, g5); break;
      case 6: pack_vec_coalesced_kernel<6><<<cgrid, 256, 0, s>>>(s4, packed, V, N, nrhs, Rp, kind, g5); break;
      default: pack_vec_coalesced_kernel<8><<<cgrid, 256, 0, s>>>(s4, packed, V, N, nrhs, Rp, kind, g5); break;
    }
    GMG_CUDA(cudaGetLastError());
    return GMG_OK;
  }
  switch (Kc) {  // Kc = ceil16(N) / 8: 2, 4, 6 or 8 for N <= 64
    case 2: pack_vec_kernel<2><<<grid, 256, 0, s>>>(src, packed, active, V, N, nrhs, R, Rp, kind, g5, a16); break;
    case 4: pack_vec_kernel<4><<<grid, 256, 0, s>>>(src, packed, active, V, N, nrhs, R, Rp, kind, g5, a16); break;
    case 6: pack_vec_kernel<6><<<grid, 256, 0, s>>>(src, packed, active, V, N, nrhs, R, Rp, kind, g5, a16); break;
    default: pack_vec_kernel<8><<<grid, 256, 0, s>>>(src, packed, active, V, N, nrhs, R, Rp, kind, g5, a16); break;
  }
  GMG_CUDA(cudaGetLastError());
  return GMG_OK;
}

// The stored link tile of one stencil point: Ks = ceil(N / 8) K-chunks of
// Mr = 2N rows rounded up to a core-matrix group of 8, i.e. without the MMA's
// padding to a whole K-step (16) and to M = 64 / 128 rows.  The MMA still reads
// whole K-steps and M rows at the chunk stride Mr * 16: its extra rows land on
// the next chunk (only accumulator rows >= 2N, never read, see them) and its
// extra K-chunk on the next point's tile or the stage's vector tiles (finite
// values, multiplied by the zero K-padding of the packed vectors).  At
// nbasis 24 a point's tile is 2304 bytes instead of 4096, at nbasis 40 6400
// instead of 12288; at nbasis 32 nothing changes.
inline void link_geometry(int N, int* Ks, int* Mr) {
  *Ks = (N + 7) / 8;
  *Mr = round_up(2 * N, 8);
}

}  // namespace tc

gmg_status coarse_prepare_tc(gmg_coarse* h, int kind, cudaStream_t s) {
  const int N = h->N;
  GMG_CHECK(2 * N <= 128, GMG_ERR_UNSUPPORTED, "tensor-core coarse stencil needs nbasis <= 64");
  int Ks, Mr;
  tc::link_geometry(N, &Ks, &Mr);
  const int V = (int)h->dims.vol();
  const size_t bytes = (size_t)V * 9 * Ks * Mr * 16;
  GMG_TRY(h->links_h.buf.alloc(bytes));
  const int64_t rows = (int64_t)V * 9 * Ks * Mr;
  tc::pack_links_kernel<<<(int)std::min<int64_t>((rows + 255) / 256, 148 * 64), 256, 0, s>>>(
      h->links_ref.as<double2>(), h->links_h.buf.as<uint4>(), V, N, Ks, Mr, kind);
  GMG_CUDA(cudaGetLastError());
  h->links_h.kind = kind;
  return GMG_OK;
}

namespace tc {

constexpr int kMaxAttrDevices = 64;
constexpr size_t kFlushBytes = (size_t)192 << 20;  // the shape tuner's L2 flush (L2: 126 MB)

// Launch shape of the stencil: CTAs per SM (1 or 2), stencil points per stage
// and the stage count that fills the shared memory of one CTA.
struct Shape {
  int ctas = 0, pps = 0, stages = 0;
  uint32_t stage_bytes = 0;
  size_t smem = 0;
};

// barriers (<= 2*32+9), TMEM slot + flag, neighbour and link-site tables of the two producers
constexpr size_t kTables = 2 * 32 * 9 * 4 + 2 * 32 * 4;
constexpr size_t kFixed = 80 * 8 + 16 + kTables;

// the shape (ctas, pps) when it fits: TMEM accumulators of all CTAs of an SM in
// its 512 columns, at least 2 stages (an even count: two producers)
static bool make_shape(int ctas, int pps, int npts, uint32_t per_point, uint32_t ncols, Shape* out) {
  if (npts % pps) return false;
  if ((uint32_t)ctas * ncols > 512) return false;
  const size_t cap = ctas == 2 ? 233472 / 2 - 1024 : 227 * 1024;
  const uint32_t stage_bytes = (uint32_t)pps * per_point;
  const int stages = (int)std::min<size_t>(32, (cap - kFixed) / stage_bytes) & ~1;
  if (stages < 2) return false;
  out->ctas = ctas;
  out->pps = pps;
  out->stages = stages;
  out->stage_bytes = stage_bytes;
  out->smem = (size_t)stages * stage_bytes + (size_t)(2 * stages + 2 * kAccBufs + 1) * 8 + 16 + kTables;
  return true;
}

// Launch configuration shared by gmg_coarse_apply and gmg_coarse_apply_noalloc.
// V output sites; site_map (nullable): link site of each output index; nbr [9][V]: input index per point.
// The shape is autotuned: the first call of a handle for a key (nbasis, padded
// RHS count, output volume, point count, operand kind, site map or not) times
// every shape that fits (one warm-up and two timed launches each, CUDA events
// on the caller's stream) and keeps the fastest; calls while the stream is
// being captured, and calls with `timed` false (the allocation-free entry),
// use the kept shape or, before there is one, the largest points-per-stage with
// 4 stages at two CTAs per SM.
static gmg_status launch_stencil(gmg_coarse* h, const uint4* packed, int V, const int32_t* site_map,
                                 const int32_t* nbr, int p0, int p1, bool g5, int kind, int nrhs,
                                 float* out, const int32_t* active, int R, bool timed, cudaStream_t s) {
  const int N = h->N;
  const int Rp = round_up(R, 16);
  const int Kc = round_up(N, 16) / 8;
  const int Mp = 2 * N <= 64 ? 64 : 128;
  int Ks, Mr;
  link_geometry(N, &Ks, &Mr);
  // the MMA's reads beyond a point's stored tile stay inside the stage: the
  // last K-step of the last point reaches at most this far past the link tiles
  const uint32_t over = (uint32_t)(Kc - 1) * Mr * 16 + (uint32_t)Mp * 16 - (uint32_t)Ks * Mr * 16;
  GMG_CHECK(over <= (uint32_t)Kc * 2 * Rp * 16, GMG_ERR_UNSUPPORTED, "tensor-core coarse stencil: link tile geometry");
  const uint32_t per_point = (uint32_t)Ks * Mr * 16 + (uint32_t)Kc * 2 * Rp * 16;
  const int npts = p1 - p0;
  const uint32_t acc_cols = 2 * (uint32_t)Rp;
  const uint32_t nacc = std::min<uint32_t>(kAccBufs, 512u / acc_cols);
  uint32_t ncols = 32;
  while (ncols < nacc * acc_cols) ncols <<= 1;

  int dev = 0;
  GMG_CUDA(cudaGetDevice(&dev));
  static int nsm_of[kMaxAttrDevices] = {0};
  static size_t smem_of[kMaxAttrDevices][2] = {{0}};
  GMG_CHECK(dev < kMaxAttrDevices, GMG_ERR_UNSUPPORTED, "tensor-core coarse stencil: device index too large");
  static std::mutex attr_mu;  // handles used from different host threads share these tables
  int nsm = 0;
  {
    std::lock_guard<std::mutex> g(attr_mu);
    if (!nsm_of[dev]) GMG_CUDA(cudaDeviceGetAttribute(&nsm_of[dev], cudaDevAttrMultiProcessorCount, dev));
    nsm = nsm_of[dev];
  }

  Params P;
  P.links = h->links_h.buf.as<uint16_t>();
  P.packed = reinterpret_cast<const uint16_t*>(packed);
  P.nbr = nbr;
  P.site_map = site_map;
  P.active = active;
  P.out = reinterpret_cast<float2*>(out);
  P.err = h->dev_err.as<int>();
  P.V = V;
  P.N = N;
  P.nrhs = nrhs;
  P.R = R;
  P.Rp = Rp;
  P.Kc = Kc;
  P.Mp = Mp;
  P.Ks = Ks;
  P.Mr = Mr;
  P.p0 = p0;
  P.p1 = p1;
  P.g5 = g5 ? 1 : 0;
  P.kind = kind == GMG_BF16 ? 1 : 0;

  // one launch of shape sh (the shared-memory attribute of each instantiation
  // only grows, so it is set again only for a larger request)
  auto launch = [&](const Shape& sh) -> gmg_status {
    auto kern = sh.ctas == 2 ? coarse_mrhs_tc_kernel<2> : coarse_mrhs_tc_kernel<1>;
    {
      std::lock_guard<std::mutex> g(attr_mu);
      if (smem_of[dev][sh.ctas - 1] < sh.smem) {
        GMG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh.smem));
        smem_of[dev][sh.ctas - 1] = sh.smem;
      }
    }
    Params Q = P;
    Q.stages = sh.stages;
    Q.pps = sh.pps;
    // programmatic dependent launch on the pack that precedes every stencil
    // launch (not inside a stream capture: captured cycles keep plain edges)
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    GMG_CUDA(cudaStreamIsCapturing(s, &cs));
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(std::min(V, nsm * sh.ctas));
    cfg.blockDim = dim3(kThreads);
    cfg.dynamicSmemBytes = sh.smem;
    cfg.stream = s;
    cfg.attrs = attr;
    cfg.numAttrs = cs == cudaStreamCaptureStatusNone ? 1 : 0;
    GMG_CUDA(cudaLaunchKernelEx(&cfg, kern, Q));
    return GMG_OK;
  };

  const uint64_t key = (uint64_t)N | ((uint64_t)Rp << 8) | ((uint64_t)npts << 16) | ((uint64_t)P.kind << 20) |
                       ((uint64_t)(site_map != nullptr) << 21) | ((uint64_t)V << 24);
  Shape sh;
  bool have = h->tc_force && make_shape(h->tc_force >> 8, h->tc_force & 0xff, npts, per_point, ncols, &sh);
  auto it = h->tc_shape.find(key);
  if (!have)
    have = it != h->tc_shape.end() && make_shape(it->second >> 8, it->second & 0xff, npts, per_point, ncols, &sh);
  if (!have) {
    // candidates: every (ctas, pps) that fits, the heuristic choice first
    Shape cand[8];
    int ncand = 0;
    for (int c2 : {2, 1})
      for (int pp : {4, 3, 2, 1}) {
        Shape t;
        if (make_shape(c2, pp, npts, per_point, ncols, &t) && (pp == 1 || t.stages >= 4)) cand[ncand++] = t;
      }
    GMG_CHECK(ncand > 0, GMG_ERR_UNSUPPORTED, "tensor-core coarse stencil: tile does not fit shared memory");
    sh = cand[0];
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    GMG_CUDA(cudaStreamIsCapturing(s, &cap));
    if (timed && cap == cudaStreamCaptureStatusNone && ncand > 1) {
      cudaEvent_t e0, e1;
      GMG_CUDA(cudaEventCreate(&e0));
      const cudaError_t ce = cudaEventCreate(&e1);
      if (ce != cudaSuccess) {
        cudaEventDestroy(e0);
        return cuda_fail(ce, "cudaEventCreate");
      }
      float best = 1e30f;
      gmg_status st = GMG_OK;
      // a failed event call leaves the timing unknown: the heuristic shape
      // is used for this call and nothing is stored for the key
      bool timing_ok = true;
      // each timed launch starts from a cold L2 (a write of a buffer larger
      // than L2 before it, outside the timed span): back-to-back launches on
      // the same operands would keep a small level's links L2-resident, which
      // they are not inside a solve, and favoured the wrong shape there
      void* flush = nullptr;
      size_t flush_bytes = 0;
      {
        static std::mutex fmu;
        static void* fbuf[kMaxAttrDevices] = {};
        std::lock_guard<std::mutex> g(fmu);
        if (dev < kMaxAttrDevices) {
          if (!fbuf[dev] && cudaMalloc(&fbuf[dev], kFlushBytes) != cudaSuccess) {
            fbuf[dev] = nullptr;
            (void)cudaGetLastError();
          }
          flush = fbuf[dev];
          flush_bytes = flush ? kFlushBytes : 0;
        }
      }
      for (int ci = 0; ci < ncand && timing_ok; ++ci) {
        const Shape& c = cand[ci];
        st = launch(c);  // warm-up
        if (st != GMG_OK) break;
        float total = 0.f;
        for (int k = 0; k < 2 && st == GMG_OK && timing_ok; ++k) {
          if (flush) timing_ok = cudaMemsetAsync(flush, k, flush_bytes, s) == cudaSuccess;
          timing_ok = timing_ok && cudaEventRecord(e0, s) == cudaSuccess;
          st = launch(c);
          if (st != GMG_OK) break;
          float ms = 0.f;
          timing_ok = timing_ok && cudaEventRecord(e1, s) == cudaSuccess &&
                      cudaEventSynchronize(e1) == cudaSuccess && cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess;
          total += ms;
        }
        if (st != GMG_OK) break;
        if (timing_ok && total < best) {
          best = total;
          sh = c;
        }
      }
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
      GMG_TRY(st);
      if (timing_ok) {
        h->tc_shape[key] = ((uint32_t)sh.ctas << 8) | (uint32_t)sh.pps;
      } else {
        (void)cudaGetLastError();  // reset the error state the failed event call left behind
        sh = cand[0];
      }
    }
  }
  if (timed) {
    KernelTimer kt("coarse_mrhs_tc", s);
    return launch(sh);
  }
  return launch(sh);
}

// the tuned shape of a key, for reports: ctas << 8 | pps, or 0 when not tuned
static uint32_t tuned_shape(gmg_coarse* h, int R, int npts, int kind) {
  const uint64_t key = (uint64_t)h->N | ((uint64_t)round_up(R, 16) << 8) | ((uint64_t)npts << 16) |
                       ((uint64_t)(kind == GMG_BF16 ? 1 : 0) << 20) | ((uint64_t)h->dims.vol() << 24);
  auto it = h->tc_shape.find(key);
  return it == h->tc_shape.end() ? 0u : it->second;
}

}  // namespace tc

gmg_status coarse_apply_tc(gmg_coarse* h, int p0, int p1, bool g5, int kind, int nrhs, const float* in,
                           float* out, const int32_t* active, int n_active, cudaStream_t s) {
  const int N = h->N;
  const int R = active ? n_active : nrhs;
  if (R == 0) return GMG_OK;
  GMG_CHECK(R <= 128, GMG_ERR_UNSUPPORTED, "tensor-core coarse stencil supports at most 128 active RHS");
  const int Rp = tc::round_up(R, 16);
  const int Kc = tc::round_up(N, 16) / 8;
  const int V = (int)h->dims.vol();
  // scratch: packed vectors
  const size_t packed_bytes = (size_t)V * Kc * 2 * Rp * 16;
  GMG_TRY(h->scratch.alloc(packed_bytes));
  uint4* packed = h->scratch.as<uint4>();
  {
    KernelTimer kt("pack_vec", s);
    GMG_TRY(tc::launch_pack(in, packed, active, V, N, nrhs, R, Rp, Kc, kind, g5, s));
  }
  return tc::launch_stencil(h, packed, V, nullptr, h->nbr.as<int32_t>(), p0, p1, g5, kind, nrhs, out, active, R,
                            true, s);
}

gmg_status coarse_apply_tc_ex(gmg_coarse* h, int V, int V_in, const int32_t* site_map, const int32_t* nbr, int p0,
                              int p1, bool g5, int kind, int nrhs, const float* in, float* out,
                              const int32_t* active, int n_active, cudaStream_t s) {
  const int N = h->N;
  const int R = active ? n_active : nrhs;
  if (R == 0) return GMG_OK;
  GMG_CHECK(R <= 128, GMG_ERR_UNSUPPORTED, "tensor-core coarse stencil supports at most 128 active RHS");
  const int Rp = tc::round_up(R, 16);
  const int Kc = tc::round_up(N, 16) / 8;
  GMG_TRY(h->scratch.alloc((size_t)V_in * Kc * 2 * Rp * 16));
  uint4* packed = h->scratch.as<uint4>();
  GMG_TRY(tc::launch_pack(in, packed, active, V_in, N, nrhs, R, Rp, Kc, kind, g5, s));
  return tc::launch_stencil(h, packed, V, site_map, nbr, p0, p1, g5, kind, nrhs, out, active, R, true, s);
}

}  // namespace gmg

// ---------------------------------------------------------------------------
// Allocation-free variant of the tensor-core multi-RHS apply.
//
// gmg_coarse_apply packs the right-hand sides into a per-handle device buffer
// that it grows with cudaMalloc on demand.  Some callers cannot let a library
// allocate at that point: a solver loop that must not stall the device (the
// CUDA runtime may synchronise inside cudaMalloc / cudaFree), or an
// application whose device memory is handed out entirely by its own pool
// allocator.  gmg_coarse_apply_noalloc runs the same two kernels (pack, then
// the tcgen05 stencil) with the packed right-hand sides in the fixed array
// below instead, so it calls no cudaMalloc, cudaFree or other allocating
// routine.
//
// The array is kNoAllocScratchBytes (16 MiB) of global memory on every GPU
// that loads this library, held until the process exits.  That is exactly
// the packed size of the 8^4 lattice / nbasis 32 / 32 RHS workload.  Larger
// requests are rejected with GMG_ERR_UNSUPPORTED.  Every call shares the
// array: the pack kernel rewrites every byte the stencil kernel reads (zero
// padding included), so no clearing is needed between calls.  Calls that
// overlap on the GPU (different streams, or different host threads) race on
// the array and must be serialised by the caller.
// ---------------------------------------------------------------------------
namespace gmg {
namespace tc {

constexpr size_t kNoAllocScratchBytes = size_t(16) << 20;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// Device address of g_noalloc_scratch on the current device.  In host code the
// symbol itself is only a host-side stand-in, so its device address is looked
// up with that device current.  The lookup is repeated on every call rather
// than cached: after a cudaDeviceReset (or any other re-creation of the
// primary context) the module is loaded again and a cached address would point
// into freed memory.  Once the module is loaded the lookup allocates nothing;
// the first lookup on a device may load it, which is when the array is
// committed.
static gmg_status noalloc_scratch(void** p) {
  void* ptr = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
  if (e != cudaSuccess || ptr == nullptr) return cuda_fail(e, "cudaGetSymbolAddress(g_noalloc_scratch)");
  *p = ptr;
  return GMG_OK;
}

}  // namespace tc
}  // namespace gmg

extern "C" gmg_status gmg_coarse_set_shape(gmg_coarse* h, int ctas, int points_per_stage) {
  GMG_CHECK(h != nullptr, GMG_ERR_ARGUMENT, "gmg_coarse_set_shape: null handle");
  GMG_CHECK((ctas == 0 && points_per_stage == 0) ||
                ((ctas == 1 || ctas == 2) && points_per_stage >= 1 && points_per_stage <= 4),
            GMG_ERR_ARGUMENT, "gmg_coarse_set_shape: ctas must be 1 or 2, points per stage 1 to 4 (0, 0: autotune)");
  h->tc_force = ((uint32_t)ctas << 8) | (uint32_t)points_per_stage;
  return GMG_OK;
}

extern "C" gmg_status gmg_coarse_tuned_shape(gmg_coarse* h, int nrhs, int npoints, gmg_prec compute, int* ctas,
                                             int* points_per_stage) {
  GMG_CHECK(h && ctas && points_per_stage, GMG_ERR_ARGUMENT, "gmg_coarse_tuned_shape: null argument");
  const uint32_t v = gmg::tc::tuned_shape(h, nrhs, npoints, (int)compute);
  *ctas = (int)(v >> 8);
  *points_per_stage = (int)(v & 0xff);
  return GMG_OK;
}

extern "C" gmg_status gmg_coarse_apply_noalloc(gmg_coarse* h, gmg_op op, int point, gmg_prec compute, int nrhs,
                                               const float* in, float* out, const int32_t* active, int n_active,
                                               gmg_stream stream) {
  using namespace gmg;
  GMG_CHECK(h != nullptr, GMG_ERR_ARGUMENT, "gmg_coarse_apply_noalloc: null handle");
  GMG_CHECK(in && out && in != out, GMG_ERR_ARGUMENT, "gmg_coarse_apply_noalloc: null or aliased vectors");
  GMG_CHECK(h->links_set, GMG_ERR_STATE, "gmg_coarse_apply_noalloc: links not set");
  GMG_CHECK(compute == GMG_BF16 || compute == GMG_F16, GMG_ERR_UNSUPPORTED,
            "gmg_coarse_apply_noalloc: only the BF16 / F16 tensor-core forms have an allocation-free variant");
  GMG_CHECK(h->links_h.kind == compute, GMG_ERR_STATE,
            "gmg_coarse_apply_noalloc: call gmg_coarse_prepare for this precision first (it allocates)");
  GMG_CHECK(nrhs >= 1 && nrhs <= 1024, GMG_ERR_ARGUMENT, "gmg_coarse_apply_noalloc: nrhs out of range");
  if (active) GMG_CHECK(n_active >= 0 && n_active <= nrhs, GMG_ERR_ARGUMENT, "gmg_coarse_apply_noalloc: bad n_active");
  int p0 = 0, p1 = 9;
  bool g5 = false;
  switch (op) {
    case GMG_OP_M: break;
    case GMG_OP_MDAG: g5 = !h->hermitian; break;
    case GMG_OP_MDIAG: p0 = 8; p1 = 9; break;
    case GMG_OP_MDIR:
      GMG_CHECK(point >= 0 && point < 9, GMG_ERR_ARGUMENT, "gmg_coarse_apply_noalloc: point out of range");
      p0 = point; p1 = point + 1;
      break;
    default: return fail(GMG_ERR_ARGUMENT, "gmg_coarse_apply_noalloc: bad op");
  }
  const int N = h->N;
  const int R = active ? n_active : nrhs;
  if (R == 0) return GMG_OK;
  GMG_CHECK(R <= 128, GMG_ERR_UNSUPPORTED, "gmg_coarse_apply_noalloc: at most 128 active RHS");
  const int Rp = tc::round_up(R, 16);
  const int Kc = tc::round_up(N, 16) / 8;
  const int V = (int)h->dims.vol();
  const size_t packed_bytes = (size_t)V * Kc * 2 * Rp * 16;
  if (packed_bytes > tc::kNoAllocScratchBytes)
    return fail(GMG_ERR_UNSUPPORTED,
                "gmg_coarse_apply_noalloc: packed right-hand sides need " + std::to_string(packed_bytes) +
                    " bytes, more than the 16 MiB static scratch; use gmg_coarse_apply");
  void* scratch = nullptr;
  GMG_TRY(tc::noalloc_scratch(&scratch));
  cudaStream_t s = S(stream);
  uint4* packed = reinterpret_cast<uint4*>(scratch);
  GMG_TRY(tc::launch_pack(static_cast<const float*>(in), packed, active, V, N, nrhs, R, Rp, Kc, compute, g5, s));
  return tc::launch_stencil(h, packed, V, nullptr, h->nbr.as<int32_t>(), p0, p1, g5, compute, nrhs, out, active, R,
                            false, s);
}

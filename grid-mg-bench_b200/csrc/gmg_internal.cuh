// gmg_internal.cuh -- shared declarations of the libgmg_b200 implementation.
#pragma once

#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <stdint.h>

#include <map>
#include <string>
#include <vector>

#include "../../include/gmg.h"

namespace gmg {

// ---------------------------------------------------------------------------
// error handling: every C entry point returns a status; the message of the
// last failure is kept per host thread.
// ---------------------------------------------------------------------------
void set_error(const std::string& msg);
const char* last_error_cstr();
gmg_status fail(gmg_status st, const std::string& msg);
gmg_status cuda_fail(cudaError_t e, const char* what);

#define GMG_CUDA(call)                                     \
  do {                                                     \
    cudaError_t e_ = (call);                               \
    if (e_ != cudaSuccess) return ::gmg::cuda_fail(e_, #call); \
  } while (0)

#define GMG_CHECK(cond, st, msg)              \
  do {                                        \
    if (!(cond)) return ::gmg::fail(st, msg); \
  } while (0)

#define GMG_TRY(call)                   \
  do {                                  \
    gmg_status st_ = (call);            \
    if (st_ != GMG_OK) return st_;      \
  } while (0)

inline cudaStream_t S(gmg_stream s) { return reinterpret_cast<cudaStream_t>(s); }

// Live timing of one kernel launch (see prof.cu); a no-op unless enabled.
class KernelTimer {
 public:
  KernelTimer(const char* name, cudaStream_t s);
  ~KernelTimer();

 private:
  const char* name_;
  cudaStream_t s_;
  cudaEvent_t a_ = nullptr, b_ = nullptr;
  bool active_ = false;
};

// ---------------------------------------------------------------------------
// lattice helpers
// ---------------------------------------------------------------------------
struct Dims {
  int d[4];
  int64_t vol() const { return (int64_t)d[0] * d[1] * d[2] * d[3]; }
};

gmg_status check_dims(const int* dims, const char* what);

// device buffer owned by a handle
struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  gmg_status alloc(size_t n);
  void free();
  ~DevBuf() { free(); }
  template <class T> T* as() const { return reinterpret_cast<T*>(p); }
};

// ---------------------------------------------------------------------------
// handles
// ---------------------------------------------------------------------------
struct LinksF16 {  // tensor-core link copy (see coarse_mrhs_tc.cu for the layout)
  DevBuf buf;
  int kind = -1;  // GMG_BF16 or GMG_F16, -1 = not built
};

}  // namespace gmg

struct gmg_coarse {
  gmg::Dims dims;
  int N = 0;
  int hermitian = 0;
  bool links_set = false;
  gmg::DevBuf nbr;         // int32 [9][V]
  gmg::DevBuf links_ref;   // complex<double> [9][V][N][N] (exchange layout)
  gmg::DevBuf links_d;     // complex<double> [V][9][N][N] (site-major, SIMT kernels)
  gmg::DevBuf links_f;     // complex<float>  [V][9][N][N]
  bool links_f_ok = false;
  gmg::LinksF16 links_h;
  gmg::DevBuf scratch;     // per-handle temporary: packed tensor-core vectors
  gmg::DevBuf dev_err;     // int: first error code a kernel of this handle recorded
  std::map<uint64_t, uint32_t> tc_shape;  // autotuned tensor-core stencil shape per key (ctas << 8 | pps)
  uint32_t tc_force = 0;                  // forced shape (ctas << 8 | pps), 0: autotuned
  // red-black operator (coarse_rb.cu)
  gmg::DevBuf self_inv;    // complex<double> [V][N][N]: inverse of the self-stencil link
  gmg::DevBuf self_inv_f;  // complex<float> copy
  bool self_inv_ok = false, self_inv_f_ok = false;
  gmg::DevBuf rb_site;     // int32 [2][V/2]: full site of half index h of parity q
  gmg::DevBuf rb_nbr;      // int32 [2][9][V/2]: half index (other / same parity) of point p's neighbour
  bool rb_ok = false;
};

struct gmg_agg {
  gmg::Dims fdims, cdims;
  int b[4] = {0, 0, 0, 0};
  int bv = 0;       // fine sites per block
  int dof = 0;      // complex dof per fine site
  int N = 0;
  bool basis_set = false;
  gmg::DevBuf blk_sites;  // int32 [Vc][bv]: fine site of in-block index (lexicographic)
  gmg::DevBuf basis_blk;  // complex<double> [Vc][N][bv*dof]   (block-major copy)
  gmg::DevBuf basis_blk_f;  // complex<float> same layout
  bool basis_f_ok = false;
  gmg::DevBuf basis_tc_hi, basis_tc_lo;  // BF16 hi / lo tensor-core packing (block_tc.cu)
  bool basis_tc_ok = false;
  gmg::DevBuf scratch;
  gmg::DevBuf ortho_ws;  // orthonormalisation workspace (ortho.cu): status, per-block flags, Cholesky factors
  gmg::DevBuf dev_err;  // int: error code recorded by the tensor-core kernels
  // CoarsenOperator workspace over the Wilson-clover operator (coarsen.cu),
  // kept between calls: fine fields of one batch of cw_nb basis vectors, the
  // projection output, per direction the fine sites of the backward faces
  // (global, cw_face) and their in-block indices (cw_sel), and per site the
  // hops (bit p) whose neighbour lies in a block of the other parity (cw_hskip)
  gmg::DevBuf cw_phi, cw_w, cw_proj, cw_face, cw_sel, cw_hskip;
  int cw_nb = 0;
  int cw_max_batch = 0;  // cap on basis vectors per CoarsenOperator batch (0: from free memory)
  int cw_nface[4] = {0, 0, 0, 0}, cw_nsel[4] = {0, 0, 0, 0};
};

struct gmg_wilson {
  gmg::Dims dims;
  double mass = 0, csw = 0;
  int apbc = 0;
  bool gauge_set = false;
  gmg::DevBuf gauge;      // complex<double> [V][4][3][3]
  gmg::DevBuf gauge_f;    // complex<float>
  gmg::DevBuf clover;     // complex<double> [V][2][6][6]
  gmg::DevBuf clover_f;
  gmg::DevBuf nbr;        // int32 [9][V]
  // hop links [V][8][3][3] (p < 4: U_mu(x), p >= 4: U_mu(x - mu)^dagger) for
  // the tile, staged and face-hop kernels
  gmg::DevBuf hop, hop_f;
  // plans of the pipelined staged kernel, by z block of the tile order: the
  // neighbour records each 4-site tile reads, tiles in processing order
  struct PipePlan {
    gmg::DevBuf buf;
    int smax = 0;         // most slots any tile uses; 0: the lattice has no plan
  };
  std::map<int, PipePlan> pplans;
  gmg::DevBuf dev_err;    // device error word of the staged kernel
  std::map<int, int> sel_pick;  // coarsening self term per nrhs: 0 pipelined staged kernel, 1 tile kernel
  int wforce = -1;                  // forced kernel variant (gmg_wilson_kernel), -1: autotuned
  std::map<uint64_t, int> wtune;    // autotuned variant per (precision, products, op class, nrhs class)
};

namespace gmg {

// neighbour table (device) for a lattice
gmg_status build_neighbors(const Dims& d, DevBuf& nbr, cudaStream_t s);
void host_neighbors(const Dims& d, int32_t* nbr);

// coarse stencil kernels (coarse_stencil.cu)
gmg_status coarse_links_to_site_major(gmg_coarse* h, cudaStream_t s);
gmg_status coarse_prepare_f32(gmg_coarse* h, cudaStream_t s);
gmg_status coarse_apply_simt(gmg_coarse* h, int p0, int p1, bool g5, int compute, int vec_prec,
                             int nrhs, const void* in, void* out, const int32_t* active,
                             int n_active, cudaStream_t s);
// src 0: stencil links, 1: self-link inverse; V / site_map / nbr: output geometry; dag: conjugate-transposed links
gmg_status coarse_apply_simt_ex(gmg_coarse* h, int src, int V, const int32_t* site_map, const int32_t* nbr,
                                bool dag, int p0, int p1, bool g5, int compute, int vec_prec, int nrhs,
                                const void* in, void* out, const int32_t* active, int n_active, cudaStream_t s);
gmg_status coarse_construct_remaining(gmg_coarse* h, cudaStream_t s);

// tensor-core multi-RHS stencil (coarse_mrhs_tc.cu)
gmg_status coarse_prepare_tc(gmg_coarse* h, int kind, cudaStream_t s);
gmg_status coarse_apply_tc(gmg_coarse* h, int p0, int p1, bool g5, int kind, int nrhs,
                           const float* in, float* out, const int32_t* active, int n_active,
                           cudaStream_t s);
// the same on a sub-geometry: V output sites, site_map (nullable) -> link site, nbr [9][V] -> input index,
// V_in input sites
gmg_status coarse_apply_tc_ex(gmg_coarse* h, int V, int V_in, const int32_t* site_map, const int32_t* nbr, int p0,
                              int p1, bool g5, int kind, int nrhs, const float* in, float* out,
                              const int32_t* active, int n_active, cudaStream_t s);

// aggregation kernels (block_ops.cu)
gmg_status agg_build_tables(gmg_agg* h, cudaStream_t s);
gmg_status agg_basis_to_blocked(gmg_agg* h, const double* basis_dev, cudaStream_t s);
gmg_status agg_basis_from_blocked(gmg_agg* h, double* basis_dev, cudaStream_t s);
gmg_status agg_project(gmg_agg* h, int compute, int vec_prec, int nrhs, const void* fine,
                       void* coarse, const int32_t* mask_blk, cudaStream_t s);
gmg_status agg_promote(gmg_agg* h, int compute, int vec_prec, int nrhs, const void* coarse,
                       void* fine, cudaStream_t s);
// block orthonormalisation and its check (ortho.cu)
gmg_status agg_orthonormalise(gmg_agg* h, int passes, cudaStream_t s);
gmg_status agg_check_orthogonal(gmg_agg* h, double* max_err, cudaStream_t s);
gmg_status agg_prepare_f32(gmg_agg* h, cudaStream_t s);
// tensor-core projection / promotion (block_tc.cu): FP32 vectors, BF16 hi+lo operands
gmg_status agg_prepare_tc(gmg_agg* h, cudaStream_t s);
gmg_status agg_project_tc(gmg_agg* h, int nrhs, const float* fine, float* coarse, cudaStream_t s);
gmg_status agg_promote_tc(gmg_agg* h, int nrhs, const float* coarse, float* fine, cudaStream_t s);

// fine Wilson-clover (wilson.cu)
gmg_status wilson_build_clover(gmg_wilson* h, cudaStream_t s);
gmg_status wilson_apply_face(gmg_wilson* h, int p, int nrhs, const double* in, double* out, const int32_t* sel,
                             int nsel, cudaStream_t s);
gmg_status wilson_apply_sel(gmg_wilson* h, int op, int dir, int disp, int nrhs, const double* in, double* out,
                            const int32_t* sel, int nsel, const uint8_t* hskip, cudaStream_t s);
gmg_status wilson_apply(gmg_wilson* h, int op, int dir, int disp, int vec_prec, int nrhs,
                        const void* in, void* out, cudaStream_t s);
gmg_status wilson_apply_mr(gmg_wilson* h, int vec_prec, int nrhs, const void* in, void* out, double2* d1,
                           double2* d2, cudaStream_t s);
gmg_status wilson_apply_f32_in(gmg_wilson* h, int op, int nrhs, const float* in, double* out, cudaStream_t s);
// BF16 fields [V][nrhs][12] words, or with `blocked` the site-blocked layout
// [V][3][nrhs][4] (the 16-byte quarters of one site's records back to back)
gmg_status wilson_apply_mr_bf16(gmg_wilson* h, int nrhs, const uint32_t* in, uint32_t* out, double2* d1, double2* d2,
                                cudaStream_t s, bool blocked = false);
// r = b - M x, FP64 fields (32-byte aligned)
gmg_status wilson_residual_f64(gmg_wilson* h, int nrhs, const double* b, const double* x, double* r,
                               cudaStream_t s);
// out = bf16(b - M x), site-blocked BF16 out, FP32 b and x (32-byte aligned)
gmg_status wilson_residual_bf16(gmg_wilson* h, int nrhs, const float* b, const float* x, uint32_t* out,
                                cudaStream_t s);

// coarse-operator construction (coarsen.cu)
gmg_status coarsen_wilson(gmg_coarse* out, gmg_agg* agg, gmg_wilson* fine, cudaStream_t s);
gmg_status coarsen_coarse(gmg_coarse* out, gmg_agg* agg, gmg_coarse* fine, cudaStream_t s);

}  // namespace gmg

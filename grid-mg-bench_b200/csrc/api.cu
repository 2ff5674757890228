// api.cu -- the extern "C" entry points declared in include/gmg.h.
//
// Host-side validation happens here (Grid's conformable()/assert checks become
// status codes); the work is dispatched to the kernels of the other files.
#include <cstring>
#include <new>

#include "gmg_internal.cuh"

using namespace gmg;

namespace {

gmg_status copy_in(void* dst, const void* src, size_t bytes, int on_device, cudaStream_t s) {
  GMG_CHECK(src != nullptr, GMG_ERR_ARGUMENT, "null input pointer");
  GMG_CUDA(cudaMemcpyAsync(dst, src, bytes, on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, s));
  if (!on_device) GMG_CUDA(cudaStreamSynchronize(s));  // caller may free its host buffer on return
  return GMG_OK;
}

gmg_status copy_out(void* dst, const void* src, size_t bytes, int on_device, cudaStream_t s) {
  GMG_CHECK(dst != nullptr, GMG_ERR_ARGUMENT, "null output pointer");
  GMG_CUDA(cudaMemcpyAsync(dst, src, bytes, on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, s));
  if (!on_device) GMG_CUDA(cudaStreamSynchronize(s));
  return GMG_OK;
}

bool vec_prec_ok(int p) { return p == GMG_F64 || p == GMG_F32; }

}  // namespace

extern "C" {

const char* gmg_last_error(void) { return last_error_cstr(); }

const char* gmg_version(void) { return "gmg_b200 1.0 (sm_100a)"; }

int gmg_point_from_dir_disp(int ndim, int dirs_faster, int dir, int disp) {
  if (!(disp == -1 || disp == 0 || disp == 1)) return -1;
  const int acts = ndim >= 5 ? 4 : ndim;
  const int base = ndim == 5 ? 1 : 0;
  if (dir == 0 && disp == 0) return 2 * acts;
  if (disp == 0) return -1;
  if (dir - base < 0 || dir - base >= acts) return -1;
  if (dirs_faster) return (1 - disp) / 2 * acts + dir - base;
  return 2 * (dir - base) + (1 - disp) / 2;
}

gmg_status gmg_lut_build(const int fine_dims[4], const int coarse_dims[4], int mask_kind, int32_t* lut,
                         int32_t* sizes, int32_t* reverse) {
  GMG_TRY(check_dims(fine_dims, "gmg_lut_build"));
  GMG_TRY(check_dims(coarse_dims, "gmg_lut_build"));
  GMG_CHECK(lut && sizes, GMG_ERR_ARGUMENT, "gmg_lut_build: null output");
  GMG_CHECK(mask_kind == -1 || (mask_kind >= 0 && mask_kind < 8) || mask_kind == 9 || mask_kind == 10,
            GMG_ERR_ARGUMENT, "gmg_lut_build: bad mask kind");
  int b[4];
  for (int d = 0; d < 4; ++d) {
    GMG_CHECK(fine_dims[d] % coarse_dims[d] == 0, GMG_ERR_SHAPE, "gmg_lut_build: coarse does not divide fine");
    b[d] = fine_dims[d] / coarse_dims[d];
  }
  const int bv = b[0] * b[1] * b[2] * b[3];
  Dims cd{{coarse_dims[0], coarse_dims[1], coarse_dims[2], coarse_dims[3]}};
  Dims fd{{fine_dims[0], fine_dims[1], fine_dims[2], fine_dims[3]}};
  for (int64_t sc = 0; sc < cd.vol(); ++sc) {
    int cc[4];
    int64_t q = sc;
    for (int d = 0; d < 4; ++d) { cc[d] = (int)(q % cd.d[d]); q /= cd.d[d]; }
    int count = 0;
    for (int sb = 0; sb < bv; ++sb) {
      int cb[4], cf[4], r = sb;
      for (int d = 0; d < 4; ++d) { cb[d] = r % b[d]; r /= b[d]; }
      int bcb = 0;
      for (int d = 0; d < 4; ++d) { cf[d] = cc[d] * b[d] + cb[d]; bcb += cf[d] / b[d]; }
      int64_t sf = 0;
      for (int d = 3; d >= 0; --d) sf = sf * fd.d[d] + cf[d];
      bool keep = true;
      if (mask_kind >= 0 && mask_kind < 8) {
        const int dir = mask_kind % 4;
        const int rr = cf[dir] % b[dir];
        keep = mask_kind < 4 ? (rr == b[dir] - 1) : (rr == 0);
      } else if (mask_kind == 9) {
        keep = bcb % 2 == 0;
      } else if (mask_kind == 10) {
        keep = bcb % 2 == 1;
      }
      if (keep) lut[sc * bv + count++] = (int32_t)sf;
      if (reverse) reverse[sf] = (int32_t)sc;
    }
    sizes[sc] = count;
    for (int k = count; k < bv; ++k) lut[sc * bv + k] = -1;
  }
  return GMG_OK;
}

// ------------------------------------------------------------------ coarse --
gmg_status gmg_coarse_create(const int dims[4], int nbasis, int hermitian, gmg_coarse** h) {
  GMG_CHECK(h != nullptr, GMG_ERR_ARGUMENT, "gmg_coarse_create: null handle pointer");
  *h = nullptr;
  GMG_TRY(check_dims(dims, "gmg_coarse_create"));
  GMG_CHECK(nbasis >= 2 && nbasis <= 128 && nbasis % 2 == 0, GMG_ERR_ARGUMENT,
            "gmg_coarse_create: nbasis must be even and in [2, 128]");
  gmg_coarse* c = new (std::nothrow) gmg_coarse();
  GMG_CHECK(c != nullptr, GMG_ERR_NOMEM, "gmg_coarse_create: host allocation failed");
  memcpy(c->dims.d, dims, sizeof(c->dims.d));
  c->N = nbasis;
  c->hermitian = hermitian ? 1 : 0;
  gmg_status st = build_neighbors(c->dims, c->nbr, 0);
  if (st == GMG_OK) st = c->links_ref.alloc(sizeof(double2) * 9 * c->dims.vol() * nbasis * nbasis);
  if (st == GMG_OK) st = c->dev_err.alloc(256);
  if (st == GMG_OK && cudaMemset(c->dev_err.p, 0, 256) != cudaSuccess) st = fail(GMG_ERR_CUDA, "cudaMemset");
  if (st != GMG_OK) {
    delete c;
    return st;
  }
  *h = c;
  return GMG_OK;
}

gmg_status gmg_coarse_destroy(gmg_coarse* h) {
  if (h) {
    cudaDeviceSynchronize();
    delete h;
  }
  return GMG_OK;
}

gmg_status gmg_coarse_set_links(gmg_coarse* h, const double* links, int on_device, gmg_stream s) {
  GMG_CHECK(h != nullptr, GMG_ERR_ARGUMENT, "gmg_coarse_set_links: null handle");
  const size_t bytes = sizeof(double2) * 9 * h->dims.vol() * h->N * h->N;
  GMG_TRY(copy_in(h->links_ref.p, links, bytes, on_device, S(s)));
  GMG_TRY(coarse_links_to_site_major(h, S(s)));
  h->links_set = true;
  h->self_inv_ok = h->self_inv_f_ok = false;
  if (h->links_f_ok) GMG_TRY(coarse_prepare_f32(h, S(s)));
  if (h->links_h.kind >= 0) GMG_TRY(coarse_prepare_tc(h, h->links_h.kind, S(s)));
  return GMG_OK;
}

gmg_status gmg_coarse_get_links(gmg_coarse* h, double* links, int on_device, gmg_stream s) {
  GMG_CHECK(h != nullptr, GMG_ERR_ARGUMENT, "gmg_coarse_get_links: null handle");
  GMG_CHECK(h->links_set, GMG_ERR_STATE, "gmg_coarse_get_links: links not set");
  const size_t bytes = sizeof(double2) * 9 * h->dims.vol() * h->N * h->N;
  return copy_out(links, h->links_ref.p, bytes, on_device, S(s));
}

gmg_status gmg_coarse_links_device(gmg_coarse* h, double** links) {
  GMG_CHECK(h && links, GMG_ERR_ARGUMENT, "gmg_coarse_links_device: null argument");
  *links = h->links_ref.as<double>();
  return GMG_OK;
}

gmg_status gmg_coarse_prepare(gmg_coarse* h, gmg_prec compute, gmg_stream s) {
  GMG_CHECK(h != nullptr, GMG_ERR_ARGUMENT, "gmg_coarse_prepare: null handle");
  GMG_CHECK(h->links_set, GMG_ERR_STATE, "gmg_coarse_prepare: links not set");
  switch (compute) {
    case GMG_F64: return GMG_OK;
    case GMG_F32: return coarse_prepare_f32(h, S(s));
    case GMG_BF16:
    case GMG_F16: return coarse_prepare_tc(h, compute, S(s));
    default: return fail(GMG_ERR_ARGUMENT, "gmg_coarse_prepare: bad precision");
  }
}

static gmg_status coarse_apply_points(gmg_coarse* h, int p0, int p1, bool g5, gmg_prec compute,
                                      gmg_prec vec_prec, int nrhs, const void* in, void* out,
                                      const int32_t* active, int n_active, cudaStream_t s) {
  if (compute == GMG_BF16 || compute == GMG_F16) {
    GMG_CHECK(vec_prec == GMG_F32, GMG_ERR_UNSUPPORTED, "tensor-core coarse apply takes F32 vectors");
    GMG_CHECK(h->links_h.kind == compute, GMG_ERR_STATE,
              "tensor-core links not prepared for this precision (gmg_coarse_prepare)");
    return coarse_apply_tc(h, p0, p1, g5, compute, nrhs, (const float*)in, (float*)out, active, n_active, s);
  }
  return coarse_apply_simt(h, p0, p1, g5, compute, vec_prec, nrhs, in, out, active, n_active, s);
}

gmg_status gmg_coarse_apply(gmg_coarse* h, gmg_op op, int point, gmg_prec compute, gmg_prec vec_prec,
                            int nrhs, const void* in, void* out, const int32_t* active, int n_active,
                            gmg_stream s) {
  GMG_CHECK(h != nullptr, GMG_ERR_ARGUMENT, "gmg_coarse_apply: null handle");
  GMG_CHECK(in && out, GMG_ERR_ARGUMENT, "gmg_coarse_apply: null vector");
  GMG_CHECK(in != out, GMG_ERR_ARGUMENT, "gmg_coarse_apply: in and out must not alias");
  GMG_CHECK(h->links_set, GMG_ERR_STATE, "gmg_coarse_apply: links not set");
  GMG_CHECK(nrhs >= 1 && nrhs <= 1024, GMG_ERR_ARGUMENT, "gmg_coarse_apply: nrhs out of range");
  GMG_CHECK(vec_prec_ok(vec_prec), GMG_ERR_ARGUMENT, "gmg_coarse_apply: vectors must be F64 or F32");
  if (active) GMG_CHECK(n_active >= 0 && n_active <= nrhs, GMG_ERR_ARGUMENT, "gmg_coarse_apply: bad n_active");
  int p0 = 0, p1 = 9;
  bool g5 = false;
  switch (op) {
    case GMG_OP_M: break;
    case GMG_OP_MDAG: g5 = !h->hermitian; break;
    case GMG_OP_MDIAG: p0 = 8; p1 = 9; break;
    case GMG_OP_MDIR:
      GMG_CHECK(point >= 0 && point < 9, GMG_ERR_ARGUMENT, "gmg_coarse_apply: point out of range");
      p0 = point; p1 = point + 1;
      break;
    default: return fail(GMG_ERR_ARGUMENT, "gmg_coarse_apply: bad op");
  }
  return coarse_apply_points(h, p0, p1, g5, compute, vec_prec, nrhs, in, out, active, n_active, S(s));
}

gmg_status gmg_coarse_mdir_all(gmg_coarse* h, gmg_prec compute, gmg_prec vec_prec, int nrhs,
                               const void* in, void* const* out8, gmg_stream s) {
  GMG_CHECK(h && in && out8, GMG_ERR_ARGUMENT, "gmg_coarse_mdir_all: null argument");
  GMG_CHECK(h->links_set, GMG_ERR_STATE, "gmg_coarse_mdir_all: links not set");
  GMG_CHECK(vec_prec_ok(vec_prec), GMG_ERR_ARGUMENT, "gmg_coarse_mdir_all: vectors must be F64 or F32");
  for (int p = 0; p < 8; ++p) {
    GMG_CHECK(out8[p] != nullptr && out8[p] != in, GMG_ERR_ARGUMENT, "gmg_coarse_mdir_all: bad output");
    GMG_TRY(coarse_apply_points(h, p, p + 1, false, compute, vec_prec, nrhs, in, out8[p], nullptr, 0, S(s)));
  }
  return GMG_OK;
}

gmg_status gmg_coarse_construct_remaining_links(gmg_coarse* h, gmg_stream s) {
  GMG_CHECK(h != nullptr, GMG_ERR_ARGUMENT, "null handle");
  GMG_CHECK(h->links_set, GMG_ERR_STATE, "gmg_coarse_construct_remaining_links: links not set");
  GMG_TRY(coarse_construct_remaining(h, S(s)));
  GMG_TRY(coarse_links_to_site_major(h, S(s)));
  h->self_inv_ok = h->self_inv_f_ok = false;
  if (h->links_f_ok) GMG_TRY(coarse_prepare_f32(h, S(s)));
  if (h->links_h.kind >= 0) GMG_TRY(coarse_prepare_tc(h, h->links_h.kind, S(s)));
  return GMG_OK;
}

gmg_status gmg_coarse_device_error(gmg_coarse* h, int* code) {
  GMG_CHECK(h && code, GMG_ERR_ARGUMENT, "gmg_coarse_device_error: null argument");
  GMG_CUDA(cudaDeviceSynchronize());
  GMG_CUDA(cudaMemcpy(code, h->dev_err.p, sizeof(int), cudaMemcpyDeviceToHost));
  GMG_CUDA(cudaMemset(h->dev_err.p, 0, sizeof(int)));
  if (*code) return fail(GMG_ERR_TIMEOUT, "a tensor-core kernel of this handle gave up waiting (code " +
                                             std::to_string(*code) + ")");
  return GMG_OK;
}

gmg_status gmg_coarse_neighbors(gmg_coarse* h, int32_t* nbr) {
  GMG_CHECK(h && nbr, GMG_ERR_ARGUMENT, "gmg_coarse_neighbors: null argument");
  GMG_CUDA(cudaMemcpy(nbr, h->nbr.p, sizeof(int32_t) * 9 * h->dims.vol(), cudaMemcpyDeviceToHost));
  return GMG_OK;
}

// --------------------------------------------------------------------- agg --
gmg_status gmg_agg_create(const int fine_dims[4], const int coarse_dims[4], int site_dof, int nbasis,
                          gmg_agg** h) {
  GMG_CHECK(h != nullptr, GMG_ERR_ARGUMENT, "gmg_agg_create: null handle pointer");
  *h = nullptr;
  GMG_TRY(check_dims(fine_dims, "gmg_agg_create"));
  GMG_TRY(check_dims(coarse_dims, "gmg_agg_create"));
  GMG_CHECK(site_dof >= 1 && site_dof <= 256, GMG_ERR_ARGUMENT, "gmg_agg_create: site_dof out of range");
  GMG_CHECK(nbasis >= 1 && nbasis <= 64, GMG_ERR_ARGUMENT, "gmg_agg_create: nbasis must be in [1, 64]");
  gmg_agg* a = new (std::nothrow) gmg_agg();
  GMG_CHECK(a != nullptr, GMG_ERR_NOMEM, "gmg_agg_create: host allocation failed");
  memcpy(a->fdims.d, fine_dims, sizeof(a->fdims.d));
  memcpy(a->cdims.d, coarse_dims, sizeof(a->cdims.d));
  a->bv = 1;
  for (int d = 0; d < 4; ++d) {
    if (fine_dims[d] % coarse_dims[d] != 0) {
      delete a;
      return fail(GMG_ERR_SHAPE, "gmg_agg_create: coarse lattice does not divide the fine lattice");
    }
    a->b[d] = fine_dims[d] / coarse_dims[d];
    a->bv *= a->b[d];
  }
  a->dof = site_dof;
  a->N = nbasis;
  gmg_status st = agg_build_tables(a, 0);
  if (st == GMG_OK) st = a->basis_blk.alloc(sizeof(double2) * a->cdims.vol() * nbasis * (size_t)a->bv * site_dof);
  if (st != GMG_OK) {
    delete a;
    return st;
  }
  *h = a;
  return GMG_OK;
}

gmg_status gmg_agg_destroy(gmg_agg* h) {
  if (h) {
    cudaDeviceSynchronize();
    delete h;
  }
  return GMG_OK;
}

gmg_status gmg_agg_set_coarsen_batch(gmg_agg* h, int max_batch) {
  GMG_CHECK(h != nullptr, GMG_ERR_ARGUMENT, "gmg_agg_set_coarsen_batch: null handle");
  GMG_CHECK(max_batch >= 0, GMG_ERR_ARGUMENT, "gmg_agg_set_coarsen_batch: negative batch");
  if (max_batch != h->cw_max_batch) {
    GMG_CUDA(cudaDeviceSynchronize());  // the kept workspace may still be in use
    h->cw_max_batch = max_batch;
    h->cw_nb = 0;  // the workspace is rebuilt for the new batch on the next construction
  }
  return GMG_OK;
}

gmg_status gmg_agg_set_basis(gmg_agg* h, const double* basis, int on_device, gmg_stream s) {
  GMG_CHECK(h && basis, GMG_ERR_ARGUMENT, "gmg_agg_set_basis: null argument");
  const size_t bytes = sizeof(double2) * (size_t)h->N * h->fdims.vol() * h->dof;
  const double* src = basis;
  DevBuf tmp;
  if (!on_device) {
    GMG_TRY(tmp.alloc(bytes));
    GMG_TRY(copy_in(tmp.p, basis, bytes, 0, S(s)));
    src = tmp.as<double>();
  }
  GMG_TRY(agg_basis_to_blocked(h, src, S(s)));
  if (!on_device) GMG_CUDA(cudaStreamSynchronize(S(s)));
  h->basis_set = true;
  return GMG_OK;
}

gmg_status gmg_agg_get_basis(gmg_agg* h, double* basis, int on_device, gmg_stream s) {
  GMG_CHECK(h && basis, GMG_ERR_ARGUMENT, "gmg_agg_get_basis: null argument");
  GMG_CHECK(h->basis_set, GMG_ERR_STATE, "gmg_agg_get_basis: basis not set");
  const size_t bytes = sizeof(double2) * (size_t)h->N * h->fdims.vol() * h->dof;
  if (on_device) return agg_basis_from_blocked(h, basis, S(s));
  DevBuf tmp;
  GMG_TRY(tmp.alloc(bytes));
  GMG_TRY(agg_basis_from_blocked(h, tmp.as<double>(), S(s)));
  return copy_out(basis, tmp.p, bytes, 0, S(s));
}

gmg_status gmg_agg_orthonormalise(gmg_agg* h, int passes, gmg_stream s) {
  GMG_CHECK(h != nullptr, GMG_ERR_ARGUMENT, "gmg_agg_orthonormalise: null handle");
  GMG_CHECK(h->basis_set, GMG_ERR_STATE, "gmg_agg_orthonormalise: basis not set");
  GMG_CHECK(passes >= 1 && passes <= 8, GMG_ERR_ARGUMENT, "gmg_agg_orthonormalise: passes out of range");
  return agg_orthonormalise(h, passes, S(s));
}

gmg_status gmg_agg_check_orthogonal(gmg_agg* h, double* max_err, gmg_stream s) {
  GMG_CHECK(h && max_err, GMG_ERR_ARGUMENT, "gmg_agg_check_orthogonal: null argument");
  GMG_CHECK(h->basis_set, GMG_ERR_STATE, "gmg_agg_check_orthogonal: basis not set");
  return agg_check_orthogonal(h, max_err, S(s));
}

gmg_status gmg_agg_project(gmg_agg* h, gmg_prec compute, gmg_prec vec_prec, int nrhs, const void* fine,
                           void* coarse, gmg_stream s) {
  GMG_CHECK(h && fine && coarse, GMG_ERR_ARGUMENT, "gmg_agg_project: null argument");
  GMG_CHECK(h->basis_set, GMG_ERR_STATE, "gmg_agg_project: basis not set");
  GMG_CHECK(nrhs >= 1 && nrhs <= 64, GMG_ERR_ARGUMENT, "gmg_agg_project: nrhs must be in [1, 64]");
  GMG_CHECK(vec_prec_ok(vec_prec), GMG_ERR_ARGUMENT, "gmg_agg_project: vectors must be F64 or F32");
  return agg_project(h, compute, vec_prec, nrhs, fine, coarse, nullptr, S(s));
}

gmg_status gmg_agg_promote(gmg_agg* h, gmg_prec compute, gmg_prec vec_prec, int nrhs, const void* coarse,
                           void* fine, gmg_stream s) {
  GMG_CHECK(h && fine && coarse, GMG_ERR_ARGUMENT, "gmg_agg_promote: null argument");
  GMG_CHECK(h->basis_set, GMG_ERR_STATE, "gmg_agg_promote: basis not set");
  GMG_CHECK(nrhs >= 1 && nrhs <= 64, GMG_ERR_ARGUMENT, "gmg_agg_promote: nrhs must be in [1, 64]");
  GMG_CHECK(vec_prec_ok(vec_prec), GMG_ERR_ARGUMENT, "gmg_agg_promote: vectors must be F64 or F32");
  return agg_promote(h, compute, vec_prec, nrhs, coarse, fine, S(s));
}

// ------------------------------------------------------------------ wilson --
gmg_status gmg_wilson_create(const int dims[4], double mass, double csw, int antiperiodic_t, gmg_wilson** h) {
  GMG_CHECK(h != nullptr, GMG_ERR_ARGUMENT, "gmg_wilson_create: null handle pointer");
  *h = nullptr;
  GMG_TRY(check_dims(dims, "gmg_wilson_create"));
  gmg_wilson* w = new (std::nothrow) gmg_wilson();
  GMG_CHECK(w != nullptr, GMG_ERR_NOMEM, "gmg_wilson_create: host allocation failed");
  memcpy(w->dims.d, dims, sizeof(w->dims.d));
  w->mass = mass;
  w->csw = csw;
  w->apbc = antiperiodic_t ? 1 : 0;
  gmg_status st = build_neighbors(w->dims, w->nbr, 0);
  if (st == GMG_OK) st = w->gauge.alloc(sizeof(double2) * 36 * w->dims.vol());
  if (st != GMG_OK) {
    delete w;
    return st;
  }
  *h = w;
  return GMG_OK;
}

gmg_status gmg_wilson_destroy(gmg_wilson* h) {
  if (h) {
    cudaDeviceSynchronize();
    delete h;
  }
  return GMG_OK;
}

gmg_status gmg_wilson_set_gauge(gmg_wilson* h, const double* U, int on_device, gmg_stream s) {
  GMG_CHECK(h && U, GMG_ERR_ARGUMENT, "gmg_wilson_set_gauge: null argument");
  GMG_TRY(copy_in(h->gauge.p, U, sizeof(double2) * 36 * h->dims.vol(), on_device, S(s)));
  GMG_TRY(wilson_build_clover(h, S(s)));
  h->gauge_set = true;
  return GMG_OK;
}

gmg_status gmg_wilson_get_clover(gmg_wilson* h, double* clover, int on_device, gmg_stream s) {
  GMG_CHECK(h && clover, GMG_ERR_ARGUMENT, "gmg_wilson_get_clover: null argument");
  GMG_CHECK(h->gauge_set, GMG_ERR_STATE, "gmg_wilson_get_clover: gauge not set");
  return copy_out(clover, h->clover.p, sizeof(double2) * 72 * h->dims.vol(), on_device, S(s));
}

gmg_status gmg_wilson_apply(gmg_wilson* h, gmg_op op, int dir, int disp, gmg_prec vec_prec, int nrhs,
                            const void* in, void* out, gmg_stream s) {
  GMG_CHECK(h && in && out, GMG_ERR_ARGUMENT, "gmg_wilson_apply: null argument");
  GMG_CHECK(in != out, GMG_ERR_ARGUMENT, "gmg_wilson_apply: in and out must not alias");
  GMG_CHECK(h->gauge_set, GMG_ERR_STATE, "gmg_wilson_apply: gauge not set");
  GMG_CHECK(nrhs >= 1 && nrhs <= 1024, GMG_ERR_ARGUMENT, "gmg_wilson_apply: nrhs out of range");
  GMG_CHECK(op >= GMG_OP_M && op <= GMG_OP_MDIR, GMG_ERR_ARGUMENT, "gmg_wilson_apply: bad op");
  if (op == GMG_OP_MDIR)
    GMG_CHECK(dir >= 0 && dir < 4 && (disp == 1 || disp == -1), GMG_ERR_ARGUMENT,
              "gmg_wilson_apply: bad direction / displacement");
  GMG_CHECK(vec_prec_ok(vec_prec), GMG_ERR_ARGUMENT, "gmg_wilson_apply: vectors must be F64 or F32");
  return wilson_apply(h, op, dir, disp, vec_prec, nrhs, in, out, S(s));
}

gmg_status gmg_wilson_apply_f32_in(gmg_wilson* h, gmg_op op, int nrhs, const float* in, double* out,
                                   gmg_stream s) {
  GMG_CHECK(h && in && out, GMG_ERR_ARGUMENT, "gmg_wilson_apply_f32_in: null argument");
  GMG_CHECK(h->gauge_set, GMG_ERR_STATE, "gmg_wilson_apply_f32_in: gauge not set");
  GMG_CHECK(nrhs >= 1 && nrhs <= 1024, GMG_ERR_ARGUMENT, "gmg_wilson_apply_f32_in: nrhs out of range");
  GMG_CHECK(op == GMG_OP_M || op == GMG_OP_MDAG, GMG_ERR_ARGUMENT, "gmg_wilson_apply_f32_in: op must be M or Mdag");
  return wilson_apply_f32_in(h, op, nrhs, in, out, S(s));
}

gmg_status gmg_wilson_set_kernel(gmg_wilson* h, gmg_wilson_kernel k) {
  GMG_CHECK(h != nullptr, GMG_ERR_ARGUMENT, "gmg_wilson_set_kernel: null handle");
  GMG_CHECK(k >= GMG_WILSON_AUTO && k <= GMG_WILSON_STAGED, GMG_ERR_ARGUMENT, "gmg_wilson_set_kernel: bad kernel");
  h->wforce = (int)k;
  return GMG_OK;
}

gmg_status gmg_wilson_tuned_kernel(gmg_wilson* h, gmg_prec vec_prec, int nrhs, int fused_mr, int single_hop,
                                   gmg_wilson_kernel* k) {
  GMG_CHECK(h && k, GMG_ERR_ARGUMENT, "gmg_wilson_tuned_kernel: null argument");
  const int cls = nrhs < 4 ? 0 : nrhs < 8 ? 1 : nrhs < 16 ? 2 : nrhs < 32 ? 3 : 4;
  const uint64_t key = (uint64_t)vec_prec | ((uint64_t)(fused_mr != 0) << 4) | ((uint64_t)(single_hop != 0) << 5) |
                       ((uint64_t)cls << 8);
  auto it = h->wtune.find(key);
  // internal register-budget sub-variants (ids >= 16) of the tile kernel report as TILE
  *k = it == h->wtune.end() ? GMG_WILSON_AUTO
                            : (gmg_wilson_kernel)(it->second >= 16 ? (int)GMG_WILSON_TILE : it->second);
  return GMG_OK;
}

gmg_status gmg_wilson_device_error(gmg_wilson* h, int* code) {
  GMG_CHECK(h && code, GMG_ERR_ARGUMENT, "gmg_wilson_device_error: null argument");
  *code = 0;
  GMG_CUDA(cudaDeviceSynchronize());
  if (!h->dev_err.p) return GMG_OK;
  GMG_CUDA(cudaMemcpy(code, h->dev_err.p, sizeof(int), cudaMemcpyDeviceToHost));
  GMG_CUDA(cudaMemset(h->dev_err.p, 0, sizeof(int)));
  if (*code) return fail(GMG_ERR_TIMEOUT, "a staged Wilson kernel gave up waiting for its copies (code " +
                                             std::to_string(*code) + ")");
  return GMG_OK;
}

gmg_status gmg_wilson_apply_mr(gmg_wilson* h, gmg_prec vec_prec, int nrhs, const void* in, void* out, double* d1,
                               double* d2, gmg_stream s) {
  GMG_CHECK(h && in && out && d1 && d2, GMG_ERR_ARGUMENT, "gmg_wilson_apply_mr: null argument");
  GMG_CHECK(in != out, GMG_ERR_ARGUMENT, "gmg_wilson_apply_mr: in and out must not alias");
  GMG_CHECK(h->gauge_set, GMG_ERR_STATE, "gmg_wilson_apply_mr: gauge not set");
  GMG_CHECK(nrhs >= 1 && nrhs <= 1024, GMG_ERR_ARGUMENT, "gmg_wilson_apply_mr: nrhs out of range");
  if (vec_prec == GMG_BF16)
    return wilson_apply_mr_bf16(h, nrhs, static_cast<const uint32_t*>(in), static_cast<uint32_t*>(out), (double2*)d1,
                                (double2*)d2, S(s));
  GMG_CHECK(vec_prec_ok(vec_prec), GMG_ERR_ARGUMENT, "gmg_wilson_apply_mr: vectors must be F64, F32 or BF16");
  return wilson_apply_mr(h, vec_prec, nrhs, in, out, (double2*)d1, (double2*)d2, S(s));
}

// ----------------------------------------------------------------- coarsen --
gmg_status gmg_coarsen_wilson(gmg_coarse* out, gmg_agg* agg, gmg_wilson* fine, gmg_stream s) {
  GMG_CHECK(out && agg && fine, GMG_ERR_ARGUMENT, "gmg_coarsen_wilson: null argument");
  return coarsen_wilson(out, agg, fine, S(s));
}

gmg_status gmg_coarsen_coarse(gmg_coarse* out, gmg_agg* agg, gmg_coarse* fine, gmg_stream s) {
  GMG_CHECK(out && agg && fine, GMG_ERR_ARGUMENT, "gmg_coarsen_coarse: null argument");
  return coarsen_coarse(out, agg, fine, S(s));
}

}  // extern "C"

// coarsen.cu -- Galerkin coarse-operator construction on the GPU (FP64).
//
// Restates CoarsenedMatrix::CoarsenOperator in its direction-saving form
// (include/CoarsenedMatrixUpstreamImprovedDirsaveLut.h:927-1097, multi-RHS
// batching of the fine applies as in ...LutMRHS.h:1004-1101):
//
//   for a batch of basis vectors phi_i (the fine operator sees them as RHS):
//     W_p = Mdir_p phi,               p = 4..7 (disp = -1)
//     A_p(c)[j][i] = sum_{x in c, x_dir mod b == 0} <v_j(x), W_p(x)>
//     W_8 = e*M(e phi) + o*M(o phi)   (block even/odd trick, :1053-1067)
//     A_8(c)[j][i] = sum_{x in c} <v_j(x), W_8(x)>
//   then A_{+mu}(x) = S o A_{-mu}(x+mu)^dag  (ConstructRemainingLinks, :1164-1196)
//
// The fine operator is either the Wilson-clover operator or, for
// coarse-of-coarse, the coarse stencil of the level above (its MdirCalc is the
// "fine" Mdir, ...Lut.h:820-860).
#include <algorithm>

#include "gmg_internal.cuh"

namespace gmg {

gmg_status agg_project_masked_f64(gmg_agg* h, int nrhs, const double* fine, double* coarse,
                                  const int8_t* mask, cudaStream_t s);
gmg_status agg_project_sel_f64(gmg_agg* h, int nrhs, const double* fine, double* coarse, const int32_t* sel,
                               int nsel, cudaStream_t s);

// field[sf][r][a] = basis_blk[c][i0 + r][sb*dof + a]
__global__ void basis_gather_kernel(const double2* __restrict__ basis_blk, const int32_t* __restrict__ blk_sites,
                                    double2* __restrict__ field, int64_t Vc, int N, int bv, int dof, int i0,
                                    int nb) {
  const int64_t K = (int64_t)bv * dof;
  const int64_t total = Vc * nb * K;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t k = e % K;
    const int r = (int)((e / K) % nb);
    const int64_t c = e / (K * nb);
    const int64_t sf = blk_sites[c * bv + k / dof];
    field[(sf * nb + r) * dof + k % dof] = basis_blk[(c * N + i0 + r) * K + k];
  }
}

// out[s][r][a] = mask[s] == want ? in[s][r][a] : 0
__global__ void mask_select_kernel(const double2* __restrict__ in, double2* __restrict__ out,
                                   const int8_t* __restrict__ mask, int64_t V, int width, int want) {
  const int64_t total = V * width;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t s = e / width;
    out[e] = (mask[s] == want) ? in[e] : make_double2(0, 0);
  }
}

// out = mask ? a : b
__global__ void mask_merge_kernel(const double2* __restrict__ a, const double2* __restrict__ b,
                                  double2* __restrict__ out, const int8_t* __restrict__ mask, int64_t V,
                                  int width) {
  const int64_t total = V * width;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total;
       e += (int64_t)gridDim.x * blockDim.x)
    out[e] = mask[e / width] ? a[e] : b[e];
}

// A_p(c)[j][i0 + r] = proj[c][r][j]
__global__ void link_scatter_kernel(const double2* __restrict__ proj, double2* __restrict__ A, int64_t Vc,
                                    int N, int i0, int nb) {
  const int64_t total = Vc * nb * N;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int j = (int)(e % N);
    const int r = (int)((e / N) % nb);
    const int64_t c = e / ((int64_t)N * nb);
    A[(c * N + j) * N + i0 + r] = proj[e];
  }
}

static int gsz(int64_t n) { return (int)std::min<int64_t>(std::max<int64_t>((n + 255) / 256, 1), 148 * 64); }

struct FineOpRef {
  gmg_wilson* w = nullptr;
  gmg_coarse* c = nullptr;
  int dof() const { return w ? 12 : c->N; }
  const Dims& dims() const { return w ? w->dims : c->dims; }
  gmg_status mdir(int p, int nb, const double* in, double* out, cudaStream_t s) const {
    if (w) return wilson_apply(w, GMG_OP_MDIR, p % 4, p < 4 ? 1 : -1, GMG_F64, nb, in, out, s);
    return coarse_apply_simt(c, p, p + 1, false, GMG_F64, GMG_F64, nb, in, out, nullptr, 0, s);
  }
  gmg_status m(int nb, const double* in, double* out, cudaStream_t s) const {
    if (w) return wilson_apply(w, GMG_OP_M, 0, 0, GMG_F64, nb, in, out, s);
    return coarse_apply_simt(c, 0, 9, false, GMG_F64, GMG_F64, nb, in, out, nullptr, 0, s);
  }
};

static void host_masks(const Dims& f, const int* b, std::vector<int8_t>& out) {
  // out[0..3]: faces x_dir mod b == 0 (points 4..7); out[4]: even blocks
  const int64_t V = f.vol();
  out.assign(5 * V, 0);
  for (int64_t s = 0; s < V; ++s) {
    int c[4];
    int64_t t = s;
    for (int d = 0; d < 4; ++d) { c[d] = (int)(t % f.d[d]); t /= f.d[d]; }
    int bcb = 0;
    for (int d = 0; d < 4; ++d) {
      out[d * V + s] = (c[d] % b[d]) == 0;
      bcb += c[d] / b[d];
    }
    out[4 * V + s] = (bcb % 2) == 0;
  }
}

static gmg_status coarsen_generic(gmg_coarse* out, gmg_agg* agg, const FineOpRef& op, cudaStream_t s) {
  const Dims& fd = op.dims();
  const int dof = op.dof();
  GMG_CHECK(agg->dof == dof, GMG_ERR_SHAPE, "coarsen: aggregation site dof differs from the fine operator");
  for (int d = 0; d < 4; ++d) {
    GMG_CHECK(agg->fdims.d[d] == fd.d[d], GMG_ERR_SHAPE, "coarsen: fine lattice differs");
    GMG_CHECK(agg->cdims.d[d] == out->dims.d[d], GMG_ERR_SHAPE, "coarsen: coarse lattice differs");
  }
  GMG_CHECK(agg->N == out->N, GMG_ERR_SHAPE, "coarsen: nbasis differs");
  GMG_CHECK(agg->basis_set, GMG_ERR_STATE, "coarsen: basis not set");
  const int N = agg->N;
  const int64_t Vf = fd.vol(), Vc = out->dims.vol();
  GMG_TRY(out->links_ref.alloc(sizeof(double2) * 9 * Vc * N * N));
  GMG_CUDA(cudaMemsetAsync(out->links_ref.p, 0, sizeof(double2) * 9 * Vc * N * N, s));

  // batch of basis vectors treated as right-hand sides: the projections reuse
  // each basis panel across the batch, so the batch is as large as four fields
  // of it allow in a third of the free device memory (at most 40 GB: the
  // whole basis of 40 vectors at 32^4)
  size_t free_b = 0, total_b = 0;
  GMG_CUDA(cudaMemGetInfo(&free_b, &total_b));
  const double cap = std::min(40.0e9, (double)free_b / 3.0) / 4.0;
  int nb = N;
  while (nb > 1 && (double)Vf * nb * dof * 16.0 > cap) nb = (nb + 1) / 2;
  if (agg->cw_max_batch > 0) nb = std::min(nb, agg->cw_max_batch);
  const size_t fbytes = sizeof(double2) * (size_t)Vf * nb * dof;
  DevBuf phi, w1, w2, w3, proj, masks;
  GMG_TRY(phi.alloc(fbytes));
  GMG_TRY(w1.alloc(fbytes));
  GMG_TRY(w2.alloc(fbytes));
  GMG_TRY(w3.alloc(fbytes));
  GMG_TRY(proj.alloc(sizeof(double2) * (size_t)Vc * nb * N));
  std::vector<int8_t> hm;
  host_masks(fd, agg->b, hm);
  GMG_TRY(masks.alloc(hm.size()));
  GMG_CUDA(cudaMemcpyAsync(masks.p, hm.data(), hm.size(), cudaMemcpyHostToDevice, s));
  const int8_t* face = masks.as<int8_t>();
  // in-block indices of each backward face (local x_mu == 0): the face
  // projections sum over those sites only, the same sites the face masks keep
  std::vector<int32_t> hsel;
  int nsel[4];
  for (int d = 0; d < 4; ++d) {
    nsel[d] = 0;
    for (int k = 0; k < agg->bv; ++k) {
      int t = k, lc[4];
      for (int q = 0; q < 4; ++q) { lc[q] = t % agg->b[q]; t /= agg->b[q]; }
      if (lc[d] == 0) {
        hsel.push_back(k);
        ++nsel[d];
      }
    }
  }
  DevBuf sel;
  GMG_TRY(sel.alloc(sizeof(int32_t) * hsel.size()));
  GMG_CUDA(cudaMemcpyAsync(sel.p, hsel.data(), sizeof(int32_t) * hsel.size(), cudaMemcpyHostToDevice, s));
  const int sel_off[4] = {0, nsel[0], nsel[0] + nsel[1], nsel[0] + nsel[1] + nsel[2]};
  const int8_t* even = face + 4 * Vf;
  double2* A = out->links_ref.as<double2>();
  const int width = nb * dof;

  for (int i0 = 0; i0 < N; i0 += nb) {
    const int cur = std::min(nb, N - i0);
    const int wdt = cur * dof;
    basis_gather_kernel<<<gsz(Vc * cur * agg->bv * dof), 256, 0, s>>>(
        agg->basis_blk.as<double2>(), agg->blk_sites.as<int32_t>(), phi.as<double2>(), Vc, N, agg->bv,
        dof, i0, cur);
    GMG_CUDA(cudaGetLastError());
    for (int p = 4; p < 8; ++p) {
      GMG_TRY(op.mdir(p, cur, phi.as<double>(), w1.as<double>(), s));
      GMG_TRY(agg_project_sel_f64(agg, cur, w1.as<double>(), proj.as<double>(), sel.as<int32_t>() + sel_off[p - 4],
                                  nsel[p - 4], s));
      link_scatter_kernel<<<gsz(Vc * cur * N), 256, 0, s>>>(proj.as<double2>(), A + (int64_t)p * Vc * N * N,
                                                             Vc, N, i0, cur);
      GMG_CUDA(cudaGetLastError());
    }
    // self term
    mask_select_kernel<<<gsz(Vf * wdt), 256, 0, s>>>(phi.as<double2>(), w1.as<double2>(), even, Vf, wdt, 1);
    GMG_TRY(op.m(cur, w1.as<double>(), w2.as<double>(), s));   // M(e phi)
    mask_select_kernel<<<gsz(Vf * wdt), 256, 0, s>>>(phi.as<double2>(), w1.as<double2>(), even, Vf, wdt, 0);
    GMG_TRY(op.m(cur, w1.as<double>(), w3.as<double>(), s));   // M(o phi)
    mask_merge_kernel<<<gsz(Vf * wdt), 256, 0, s>>>(w2.as<double2>(), w3.as<double2>(), w1.as<double2>(), even,
                                                    Vf, wdt);
    GMG_CUDA(cudaGetLastError());
    GMG_TRY(agg_project_masked_f64(agg, cur, w1.as<double>(), proj.as<double>(), nullptr, s));
    link_scatter_kernel<<<gsz(Vc * cur * N), 256, 0, s>>>(proj.as<double2>(), A + (int64_t)8 * Vc * N * N, Vc,
                                                           N, i0, cur);
    GMG_CUDA(cudaGetLastError());
  }
  (void)width;
  GMG_TRY(coarse_construct_remaining(out, s));
  GMG_TRY(coarse_links_to_site_major(out, s));
  out->links_set = true;
  out->links_f_ok = false;
  out->self_inv_ok = out->self_inv_f_ok = false;
  out->links_h.kind = -1;
  // temporaries are freed at scope exit: make sure the stream is done with them
  GMG_CUDA(cudaStreamSynchronize(s));
  return GMG_OK;
}

// Workspace of the Wilson-clover coarsening, built on the first call and kept
// in the aggregation: the batch size comes from the free memory then (two
// fields of it in a third of it, at most 40 GB), the face lists and block
// parities from the geometry.
static gmg_status coarsen_workspace(gmg_agg* agg, cudaStream_t s) {
  if (agg->cw_nb > 0) return GMG_OK;
  const Dims& fd = agg->fdims;
  const int64_t Vf = fd.vol(), Vc = agg->cdims.vol();
  const int N = agg->N, dof = agg->dof;
  size_t free_b = 0, total_b = 0;
  GMG_CUDA(cudaMemGetInfo(&free_b, &total_b));
  const double cap = std::min(40.0e9, (double)free_b / 3.0) / 2.0;
  int nb = N;
  while (nb > 1 && (double)Vf * nb * dof * 16.0 > cap) nb = (nb + 1) / 2;
  if (agg->cw_max_batch > 0) nb = std::min(nb, agg->cw_max_batch);
  const size_t fbytes = sizeof(double2) * (size_t)Vf * nb * dof;
  GMG_TRY(agg->cw_phi.alloc(fbytes));
  GMG_TRY(agg->cw_w.alloc(fbytes));
  GMG_TRY(agg->cw_proj.alloc(sizeof(double2) * (size_t)Vc * nb * N));
  std::vector<int32_t> face, sel;
  std::vector<uint8_t> bpar(Vf), hskip(Vf);
  for (int d = 0; d < 4; ++d) {
    agg->cw_nface[d] = 0;
    for (int64_t x = 0; x < Vf; ++x) {
      int64_t t = x;
      int c = 0;
      for (int q = 0; q <= d; ++q) {
        c = (int)(t % fd.d[q]);
        t /= fd.d[q];
      }
      if (c % agg->b[d] == 0) {
        face.push_back((int32_t)x);
        ++agg->cw_nface[d];
      }
    }
    agg->cw_nsel[d] = 0;
    for (int k = 0; k < agg->bv; ++k) {
      int t = k, lc[4];
      for (int q = 0; q < 4; ++q) {
        lc[q] = t % agg->b[q];
        t /= agg->b[q];
      }
      if (lc[d] == 0) {
        sel.push_back(k);
        ++agg->cw_nsel[d];
      }
    }
  }
  for (int64_t x = 0; x < Vf; ++x) {
    int64_t t = x;
    int par = 0;
    for (int q = 0; q < 4; ++q) {
      par += (int)(t % fd.d[q]) / agg->b[q];
      t /= fd.d[q];
    }
    bpar[x] = (uint8_t)(par & 1);
  }
  // hop p = (mu = p mod 4, +1 for p < 4, -1 otherwise), periodic neighbours
  int64_t stride[4] = {1, 1, 1, 1};
  for (int q = 1; q < 4; ++q) stride[q] = stride[q - 1] * fd.d[q - 1];
  for (int64_t x = 0; x < Vf; ++x) {
    uint8_t m = 0;
    for (int p = 0; p < 8; ++p) {
      const int mu = p & 3;
      const int xm = (int)((x / stride[mu]) % fd.d[mu]);
      const int ym = (xm + (p < 4 ? 1 : fd.d[mu] - 1)) % fd.d[mu];
      const int64_t y = x + (int64_t)(ym - xm) * stride[mu];
      if (bpar[y] != bpar[x]) m |= (uint8_t)(1u << p);
    }
    hskip[x] = m;
  }
  GMG_TRY(agg->cw_face.alloc(sizeof(int32_t) * face.size()));
  GMG_TRY(agg->cw_sel.alloc(sizeof(int32_t) * sel.size()));
  GMG_TRY(agg->cw_hskip.alloc(hskip.size()));
  GMG_CUDA(cudaMemcpyAsync(agg->cw_face.p, face.data(), sizeof(int32_t) * face.size(), cudaMemcpyHostToDevice, s));
  GMG_CUDA(cudaMemcpyAsync(agg->cw_sel.p, sel.data(), sizeof(int32_t) * sel.size(), cudaMemcpyHostToDevice, s));
  GMG_CUDA(cudaMemcpyAsync(agg->cw_hskip.p, hskip.data(), hskip.size(), cudaMemcpyHostToDevice, s));
  GMG_CUDA(cudaStreamSynchronize(s));  // the host vectors go out of scope
  agg->cw_nb = nb;
  return GMG_OK;
}

// CoarsenOperator over the Wilson-clover operator.  Per batch of basis
// vectors: the backward hop Mdir_p evaluated on the face sites only (the only
// sites its face projection reads), and the self term e D e + o D o as one
// pass of the operator with the hops between blocks of opposite parity left
// out.  Both give, at every site the projections read, the same sums in the
// same order as the masked full-lattice form of coarsen_generic.
static gmg_status coarsen_wilson_faces(gmg_coarse* out, gmg_agg* agg, gmg_wilson* w, cudaStream_t s) {
  const int dof = 12;
  GMG_CHECK(agg->dof == dof, GMG_ERR_SHAPE, "coarsen: aggregation site dof differs from the fine operator");
  for (int d = 0; d < 4; ++d) {
    GMG_CHECK(agg->fdims.d[d] == w->dims.d[d], GMG_ERR_SHAPE, "coarsen: fine lattice differs");
    GMG_CHECK(agg->cdims.d[d] == out->dims.d[d], GMG_ERR_SHAPE, "coarsen: coarse lattice differs");
  }
  GMG_CHECK(agg->N == out->N, GMG_ERR_SHAPE, "coarsen: nbasis differs");
  GMG_CHECK(agg->basis_set, GMG_ERR_STATE, "coarsen: basis not set");
  const int N = agg->N;
  const int64_t Vc = out->dims.vol();
  GMG_TRY(out->links_ref.alloc(sizeof(double2) * 9 * Vc * N * N));
  GMG_CUDA(cudaMemsetAsync(out->links_ref.p, 0, sizeof(double2) * 9 * Vc * N * N, s));
  GMG_TRY(coarsen_workspace(agg, s));
  const int nb = agg->cw_nb;
  double* phi = agg->cw_phi.as<double>();
  double* wf = agg->cw_w.as<double>();
  double* proj = agg->cw_proj.as<double>();
  const int32_t* face = agg->cw_face.as<int32_t>();
  const int32_t* sel = agg->cw_sel.as<int32_t>();
  double2* A = out->links_ref.as<double2>();
  for (int i0 = 0; i0 < N; i0 += nb) {
    const int cur = std::min(nb, N - i0);
    basis_gather_kernel<<<gsz(Vc * cur * agg->bv * dof), 256, 0, s>>>(
        agg->basis_blk.as<double2>(), agg->blk_sites.as<int32_t>(), reinterpret_cast<double2*>(phi), Vc, N,
        agg->bv, dof, i0, cur);
    GMG_CUDA(cudaGetLastError());
    int fo = 0, so = 0;
    for (int d = 0; d < 4; ++d) {
      GMG_TRY(wilson_apply_face(w, 4 + d, cur, phi, wf, face + fo, agg->cw_nface[d], s));
      GMG_TRY(agg_project_sel_f64(agg, cur, wf, proj, sel + so, agg->cw_nsel[d], s));
      link_scatter_kernel<<<gsz(Vc * cur * N), 256, 0, s>>>(reinterpret_cast<const double2*>(proj),
                                                             A + (int64_t)(4 + d) * Vc * N * N, Vc, N, i0, cur);
      GMG_CUDA(cudaGetLastError());
      fo += agg->cw_nface[d];
      so += agg->cw_nsel[d];
    }
    GMG_TRY(wilson_apply_sel(w, GMG_OP_M, 0, 0, cur, phi, wf, nullptr, 0, agg->cw_hskip.as<uint8_t>(), s));
    GMG_TRY(agg_project_masked_f64(agg, cur, wf, proj, nullptr, s));
    link_scatter_kernel<<<gsz(Vc * cur * N), 256, 0, s>>>(reinterpret_cast<const double2*>(proj),
                                                           A + (int64_t)8 * Vc * N * N, Vc, N, i0, cur);
    GMG_CUDA(cudaGetLastError());
  }
  GMG_TRY(coarse_construct_remaining(out, s));
  GMG_TRY(coarse_links_to_site_major(out, s));
  out->links_set = true;
  out->links_f_ok = false;
  out->self_inv_ok = out->self_inv_f_ok = false;
  out->links_h.kind = -1;
  return GMG_OK;
}

gmg_status coarsen_wilson(gmg_coarse* out, gmg_agg* agg, gmg_wilson* fine, cudaStream_t s) {
  GMG_CHECK(fine->gauge_set, GMG_ERR_STATE, "coarsen: gauge field not set");
  return coarsen_wilson_faces(out, agg, fine, s);
}

gmg_status coarsen_coarse(gmg_coarse* out, gmg_agg* agg, gmg_coarse* fine, cudaStream_t s) {
  GMG_CHECK(fine->links_set, GMG_ERR_STATE, "coarsen: fine links not set");
  FineOpRef op;
  op.c = fine;
  return coarsen_generic(out, agg, op, s);
}

}  // namespace gmg

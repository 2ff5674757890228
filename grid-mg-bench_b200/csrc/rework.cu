// rework.cu -- the two-spin (Rework) forms of the aggregation subspace and of
// the coarse link fields, for the Rework class surface (include/gmg_rework.hpp).
//
// The Rework classes (include/CoarseningPolicyRework.h:56-109,
// AggregationRework.h:75-146, CoarsenedMatrixRework.h:60-101) keep Nc_c basis
// vectors and give the coarse field Ns_c "spins": coarse component (s, c) is
// the projection onto the part of basis vector c on the s-th of Ns_c equal
// slices of the fine site dof (for the Wilson spinor with Ns_c = 2 the two
// chiralities, spins {0,1} and {2,3}; for a coarse fine level the G5C halves).
// That is the chirally doubled basis of the Upstream classes with flat index
// n = s * Nc_c + c (include/Layout_converters.h:49-56, 107-110), which is how
// this library stores it: the subspace entries below split Nc_c vectors into
// the Ns_c * Nc_c doubled basis and sum them back, and the link entries map the
// flat [N][N] link matrices to the [Ns_c][Ns_c][Nc_c][Nc_c] blocks of the
// Rework link field.  Coarse vectors need no map: [s][c] and the flat index
// n = s * Nc_c + c are the same memory order.
#include <algorithm>

#include "gmg_internal.cuh"

namespace gmg {

__global__ void spin_split_kernel(const double2* __restrict__ vecs, double2* __restrict__ basis, int nvec, int ns,
                                  int64_t Vf, int dof) {
  const int slice = dof / ns;
  const int64_t total = (int64_t)nvec * Vf * dof;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int a = (int)(e % dof);
    const int64_t cs = e / dof;  // c * Vf + site
    const int c = (int)(cs / Vf);
    const int64_t site = cs % Vf;
    const double2 v = vecs[e];
    for (int s = 0; s < ns; ++s)
      basis[(((int64_t)s * nvec + c) * Vf + site) * dof + a] = (a / slice == s) ? v : make_double2(0.0, 0.0);
  }
}

__global__ void spin_merge_kernel(const double2* __restrict__ basis, double2* __restrict__ vecs, int nvec, int ns,
                                  int64_t Vf, int dof) {
  const int64_t total = (int64_t)nvec * Vf * dof;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int a = (int)(e % dof);
    const int64_t cs = e / dof;
    const int c = (int)(cs / Vf);
    const int64_t site = cs % Vf;
    double2 acc = make_double2(0.0, 0.0);
    for (int s = 0; s < ns; ++s) {
      const double2 v = basis[(((int64_t)s * nvec + c) * Vf + site) * dof + a];
      acc.x += v.x;
      acc.y += v.y;
    }
    vecs[e] = acc;
  }
}

static int grid_for(int64_t n) { return (int)std::min<int64_t>(std::max<int64_t>((n + 255) / 256, 1), 148 * 64); }

static gmg_status check_spins(const gmg_agg* h, int ns, const char* what) {
  GMG_CHECK(h != nullptr, GMG_ERR_ARGUMENT, std::string(what) + ": null handle");
  GMG_CHECK(ns >= 1 && h->N % ns == 0 && h->dof % ns == 0, GMG_ERR_SHAPE,
            std::string(what) + ": nbasis and the site dof must be multiples of the coarse spin count");
  return GMG_OK;
}

}  // namespace gmg

using namespace gmg;

extern "C" gmg_status gmg_agg_set_subspace_spins(gmg_agg* h, int ncoarse_spins, const double* vecs, int on_device,
                                                 gmg_stream stream) {
  GMG_TRY(check_spins(h, ncoarse_spins, "gmg_agg_set_subspace_spins"));
  GMG_CHECK(vecs != nullptr, GMG_ERR_ARGUMENT, "gmg_agg_set_subspace_spins: null vectors");
  cudaStream_t s = S(stream);
  const int nvec = h->N / ncoarse_spins;
  const int64_t Vf = h->fdims.vol();
  const size_t vbytes = sizeof(double2) * (size_t)nvec * Vf * h->dof;
  DevBuf in, basis;
  const double2* src = reinterpret_cast<const double2*>(vecs);
  if (!on_device) {
    GMG_TRY(in.alloc(vbytes));
    GMG_CUDA(cudaMemcpyAsync(in.p, vecs, vbytes, cudaMemcpyHostToDevice, s));
    src = in.as<double2>();
  }
  GMG_TRY(basis.alloc(vbytes * ncoarse_spins));
  spin_split_kernel<<<grid_for((int64_t)nvec * Vf * h->dof), 256, 0, s>>>(src, basis.as<double2>(), nvec,
                                                                          ncoarse_spins, Vf, h->dof);
  GMG_CUDA(cudaGetLastError());
  GMG_TRY(agg_basis_to_blocked(h, basis.as<double>(), s));
  GMG_CUDA(cudaStreamSynchronize(s));  // the temporaries are freed on return
  h->basis_set = true;
  return GMG_OK;
}

extern "C" gmg_status gmg_agg_get_subspace_spins(gmg_agg* h, int ncoarse_spins, double* vecs, int on_device,
                                                 gmg_stream stream) {
  GMG_TRY(check_spins(h, ncoarse_spins, "gmg_agg_get_subspace_spins"));
  GMG_CHECK(vecs != nullptr, GMG_ERR_ARGUMENT, "gmg_agg_get_subspace_spins: null vectors");
  GMG_CHECK(h->basis_set, GMG_ERR_STATE, "gmg_agg_get_subspace_spins: basis not set");
  cudaStream_t s = S(stream);
  const int nvec = h->N / ncoarse_spins;
  const int64_t Vf = h->fdims.vol();
  const size_t vbytes = sizeof(double2) * (size_t)nvec * Vf * h->dof;
  DevBuf basis, out;
  GMG_TRY(basis.alloc(vbytes * ncoarse_spins));
  GMG_TRY(agg_basis_from_blocked(h, basis.as<double>(), s));
  double2* dst = reinterpret_cast<double2*>(vecs);
  if (!on_device) {
    GMG_TRY(out.alloc(vbytes));
    dst = out.as<double2>();
  }
  spin_merge_kernel<<<grid_for((int64_t)nvec * Vf * h->dof), 256, 0, s>>>(basis.as<double2>(), dst, nvec,
                                                                          ncoarse_spins, Vf, h->dof);
  GMG_CUDA(cudaGetLastError());
  if (!on_device) GMG_CUDA(cudaMemcpyAsync(vecs, out.p, vbytes, cudaMemcpyDeviceToHost, s));
  GMG_CUDA(cudaStreamSynchronize(s));
  return GMG_OK;
}

extern "C" gmg_status gmg_coarse_get_links_spins(gmg_coarse* h, int ncoarse_spins, int point, double* links,
                                                 int on_device, gmg_stream stream) {
  GMG_CHECK(h && links, GMG_ERR_ARGUMENT, "gmg_coarse_get_links_spins: null argument");
  GMG_CHECK(h->links_set, GMG_ERR_STATE, "gmg_coarse_get_links_spins: links not set");
  GMG_CHECK(point >= 0 && point < 9, GMG_ERR_ARGUMENT, "gmg_coarse_get_links_spins: point out of range");
  GMG_CHECK(ncoarse_spins >= 1 && h->N % ncoarse_spins == 0, GMG_ERR_SHAPE,
            "gmg_coarse_get_links_spins: nbasis must be a multiple of the coarse spin count");
  cudaStream_t s = S(stream);
  const int64_t V = h->dims.vol(), NN = (int64_t)h->N * h->N;
  const size_t bytes = sizeof(double2) * (size_t)V * NN;
  DevBuf tmp;
  double2* dst = reinterpret_cast<double2*>(links);
  if (!on_device) {
    GMG_TRY(tmp.alloc(bytes));
    dst = tmp.as<double2>();
  }
  GMG_TRY(gmg_layout_links(V, h->N, ncoarse_spins, h->links_ref.as<double>() + 2 * point * V * NN,
                           reinterpret_cast<double*>(dst), 0, stream));
  if (!on_device) {
    GMG_CUDA(cudaMemcpyAsync(links, tmp.p, bytes, cudaMemcpyDeviceToHost, s));
    GMG_CUDA(cudaStreamSynchronize(s));
  }
  return GMG_OK;
}

extern "C" gmg_status gmg_coarse_set_links_spins(gmg_coarse* h, int ncoarse_spins, const double* links,
                                                 int on_device, gmg_stream stream) {
  GMG_CHECK(h && links, GMG_ERR_ARGUMENT, "gmg_coarse_set_links_spins: null argument");
  GMG_CHECK(ncoarse_spins >= 1 && h->N % ncoarse_spins == 0, GMG_ERR_SHAPE,
            "gmg_coarse_set_links_spins: nbasis must be a multiple of the coarse spin count");
  cudaStream_t s = S(stream);
  const int64_t V = h->dims.vol(), NN = (int64_t)h->N * h->N;
  const size_t bytes = sizeof(double2) * (size_t)9 * V * NN;
  DevBuf src, flat;
  const double2* in = reinterpret_cast<const double2*>(links);
  if (!on_device) {
    GMG_TRY(src.alloc(bytes));
    GMG_CUDA(cudaMemcpyAsync(src.p, links, bytes, cudaMemcpyHostToDevice, s));
    in = src.as<double2>();
  }
  GMG_TRY(flat.alloc(bytes));
  for (int p = 0; p < 9; ++p)
    GMG_TRY(gmg_layout_links(V, h->N, ncoarse_spins, reinterpret_cast<const double*>(in + p * V * NN),
                             flat.as<double>() + 2 * p * V * NN, 1, stream));
  GMG_TRY(gmg_coarse_set_links(h, flat.as<double>(), 1, stream));
  GMG_CUDA(cudaStreamSynchronize(s));
  return GMG_OK;
}

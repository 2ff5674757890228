// common.cu -- error state, device buffers, lattice tables.
#include <cstdio>
#include <cstring>
#include <string>

#include "gmg_internal.cuh"

namespace gmg {

static thread_local std::string g_last_error;

void set_error(const std::string& msg) { g_last_error = msg; }

const char* last_error_cstr() { return g_last_error.c_str(); }

gmg_status fail(gmg_status st, const std::string& msg) {
  set_error(msg);
  return st;
}

gmg_status cuda_fail(cudaError_t e, const char* what) {
  std::string m = std::string("CUDA error ") + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) +
                  ") in " + what;
  set_error(m);
  return e == cudaErrorMemoryAllocation ? GMG_ERR_NOMEM : GMG_ERR_CUDA;
}

gmg_status check_dims(const int* dims, const char* what) {
  GMG_CHECK(dims != nullptr, GMG_ERR_ARGUMENT, std::string(what) + ": dims is null");
  int64_t v = 1;
  for (int d = 0; d < 4; ++d) {
    GMG_CHECK(dims[d] > 0 && dims[d] <= 4096, GMG_ERR_SHAPE,
              std::string(what) + ": lattice extent out of range");
    v *= dims[d];
  }
  GMG_CHECK(v < (int64_t(1) << 31), GMG_ERR_SHAPE, std::string(what) + ": volume too large");
  return GMG_OK;
}

gmg_status DevBuf::alloc(size_t n) {
  if (p && bytes >= n) return GMG_OK;
  free();
  if (n == 0) return GMG_OK;
  cudaError_t e = cudaMalloc(&p, n);
  if (e != cudaSuccess) {
    p = nullptr;
    return cuda_fail(e, "cudaMalloc");
  }
  bytes = n;
  return GMG_OK;
}

void DevBuf::free() {
  if (p) cudaFree(p);
  p = nullptr;
  bytes = 0;
}

// nbr[p][s]: p<4 -> x + e_p, 4<=p<8 -> x - e_{p-4}, 8 -> x  (periodic wrap)
void host_neighbors(const Dims& d, int32_t* nbr) {
  const int64_t V = d.vol();
  for (int64_t s = 0; s < V; ++s) {
    int c[4];
    int64_t t = s;
    for (int k = 0; k < 4; ++k) { c[k] = (int)(t % d.d[k]); t /= d.d[k]; }
    for (int p = 0; p < 9; ++p) {
      int cc[4] = {c[0], c[1], c[2], c[3]};
      if (p < 8) {
        const int dir = p % 4, disp = p < 4 ? 1 : -1;
        cc[dir] = (cc[dir] + disp + d.d[dir]) % d.d[dir];
      }
      int64_t idx = 0;
      for (int k = 3; k >= 0; --k) idx = idx * d.d[k] + cc[k];
      nbr[p * V + s] = (int32_t)idx;
    }
  }
}

gmg_status build_neighbors(const Dims& d, DevBuf& nbr, cudaStream_t s) {
  const int64_t V = d.vol();
  std::vector<int32_t> h(9 * V);
  host_neighbors(d, h.data());
  GMG_TRY(nbr.alloc(h.size() * sizeof(int32_t)));
  GMG_CUDA(cudaMemcpyAsync(nbr.p, h.data(), h.size() * sizeof(int32_t), cudaMemcpyHostToDevice, s));
  GMG_CUDA(cudaStreamSynchronize(s));  // h goes out of scope
  return GMG_OK;
}

}  // namespace gmg

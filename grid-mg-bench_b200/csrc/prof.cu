// prof.cu -- optional live timing of the hot kernels with CUDA events.
//
// When enabled (gmg_profile_enable), each instrumented launch records a pair
// of CUDA events on the stream it is launched on; gmg_profile_read
// synchronises those events and returns the summed kernel time and launch
// count for one kernel name.  Disabled by default: then a launch costs one
// branch.
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "gmg_internal.cuh"

namespace gmg {

namespace {
struct Rec {
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev;
};
std::mutex g_mu;
bool g_on = false;
std::map<std::string, Rec> g_recs;
std::vector<cudaEvent_t> g_pool;  // events returned by gmg_profile_read, reused

cudaEvent_t take_event() {
  {
    std::lock_guard<std::mutex> g(g_mu);
    if (!g_pool.empty()) {
      cudaEvent_t e = g_pool.back();
      g_pool.pop_back();
      return e;
    }
  }
  cudaEvent_t e = nullptr;
  cudaEventCreate(&e);
  return e;
}
}  // namespace

bool prof_enabled() { return g_on; }

KernelTimer::KernelTimer(const char* name, cudaStream_t s) : name_(name), s_(s) {
  if (!g_on) return;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(s_, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) return;  // not in graphs
  a_ = take_event();
  b_ = take_event();
  cudaEventRecord(a_, s_);
  active_ = true;
}

KernelTimer::~KernelTimer() {
  if (!active_) return;
  cudaEventRecord(b_, s_);
  std::lock_guard<std::mutex> g(g_mu);
  g_recs[name_].ev.emplace_back(a_, b_);
}

}  // namespace gmg

extern "C" gmg_status gmg_profile_enable(int on) {
  std::lock_guard<std::mutex> g(gmg::g_mu);
  gmg::g_on = on != 0;
  return GMG_OK;
}

extern "C" gmg_status gmg_profile_read(const char* kernel, double* total_ms, int64_t* launches) {
  GMG_CHECK(kernel && total_ms && launches, GMG_ERR_ARGUMENT, "gmg_profile_read: null argument");
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev;
  {
    std::lock_guard<std::mutex> g(gmg::g_mu);
    auto it = gmg::g_recs.find(kernel);
    if (it != gmg::g_recs.end()) ev.swap(it->second.ev);
  }
  double t = 0;
  for (auto& e : ev) {
    float ms = 0;
    GMG_CUDA(cudaEventSynchronize(e.second));
    GMG_CUDA(cudaEventElapsedTime(&ms, e.first, e.second));
    t += ms;
  }
  {
    std::lock_guard<std::mutex> g(gmg::g_mu);
    for (auto& e : ev) {
      gmg::g_pool.push_back(e.first);
      gmg::g_pool.push_back(e.second);
    }
  }
  *total_ms = t;
  *launches = (int64_t)ev.size();
  return GMG_OK;
}

// Kernel timing for measurement runs: CUDA events recorded around the main
// kernels of each stage, on the stream each kernel is launched on.
//
// Off by default. lh_kernel_timing(1) clears the record and starts it;
// every timed launch then records one event before and one after itself.
// lh_kernel_timing_read waits for the recorded events and returns, per
// kernel, the launch count and the summed duration. Events recorded inside a
// stream capture would become graph nodes, so timing is skipped while the
// launching stream is capturing.
#include <mutex>
#include <vector>

#include "lh_timing.cuh"

namespace {

struct Pending {
  int kernel;
  cudaEvent_t start, stop;
};

__device__ unsigned long long g_units[LH_KT_COUNT];

std::mutex g_timing_lock;
bool g_timing_on = false;
std::vector<Pending> g_pending;
std::vector<cudaEvent_t> g_free;

cudaEvent_t take_event() {
  if (!g_free.empty()) {
    cudaEvent_t e = g_free.back();
    g_free.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
  return e;
}

}  // namespace

namespace lh {

unsigned long long* kernel_units() {
  static unsigned long long* address = nullptr;
  if (!address) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_units) != cudaSuccess) return nullptr;
    address = static_cast<unsigned long long*>(p);
  }
  return address;
}

TimedLaunch::TimedLaunch(int kernel, cudaStream_t stream) : kernel_(kernel), stream_(stream) {
  std::lock_guard<std::mutex> guard(g_timing_lock);
  if (!g_timing_on) return;
  cudaStreamCaptureStatus capture = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(stream, &capture) != cudaSuccess ||
      capture != cudaStreamCaptureStatusNone)
    return;
  start_ = take_event();
  stop_ = take_event();
  if (!start_ || !stop_) return;
  cudaEventRecord(start_, stream);
  armed_ = true;
}

TimedLaunch::~TimedLaunch() {
  if (!armed_) return;
  cudaEventRecord(stop_, stream_);
  std::lock_guard<std::mutex> guard(g_timing_lock);
  g_pending.push_back(Pending{kernel_, start_, stop_});
}

}  // namespace lh

extern "C" int lh_kernel_timing(int enable) {
  std::lock_guard<std::mutex> guard(g_timing_lock);
  for (Pending& p : g_pending) {
    g_free.push_back(p.start);
    g_free.push_back(p.stop);
  }
  g_pending.clear();
  g_timing_on = enable != 0;
  if (enable) {  // the unit counters start from zero with the record
    unsigned long long* units = lh::kernel_units();
    if (!units || cudaDeviceSynchronize() != cudaSuccess ||
        cudaMemset(units, 0, sizeof(unsigned long long) * LH_KT_COUNT) != cudaSuccess ||
        cudaDeviceSynchronize() != cudaSuccess)
      return LH_ECUDA;
  }
  return LH_OK;
}

extern "C" int lh_kernel_units_read(int32_t n_kernels, int64_t* units) {
  if (n_kernels < 0 || (n_kernels && !units)) return LH_EINVAL;
  unsigned long long host[LH_KT_COUNT];
  unsigned long long* device = lh::kernel_units();
  if (!device || cudaDeviceSynchronize() != cudaSuccess ||
      cudaMemcpy(host, device, sizeof(host), cudaMemcpyDeviceToHost) != cudaSuccess)
    return LH_ECUDA;
  for (int k = 0; k < n_kernels; ++k) units[k] = k < LH_KT_COUNT ? (int64_t)host[k] : 0;
  return LH_OK;
}

extern "C" int lh_kernel_timing_read(int32_t n_kernels, int64_t* launches, double* total_ms) {
  if (n_kernels < 0 || (n_kernels && (!launches || !total_ms))) return LH_EINVAL;
  for (int k = 0; k < n_kernels; ++k) {
    launches[k] = 0;
    total_ms[k] = 0.0;
  }
  std::vector<Pending> done;
  {
    std::lock_guard<std::mutex> guard(g_timing_lock);
    done.swap(g_pending);
  }
  int rc = LH_OK;
  for (Pending& p : done) {
    float ms = 0.f;
    if (cudaEventSynchronize(p.stop) != cudaSuccess ||
        cudaEventElapsedTime(&ms, p.start, p.stop) != cudaSuccess) {
      rc = LH_ECUDA;
      continue;
    }
    if (p.kernel >= 0 && p.kernel < n_kernels) {
      launches[p.kernel] += 1;
      total_ms[p.kernel] += ms;
    }
  }
  std::lock_guard<std::mutex> guard(g_timing_lock);
  for (Pending& p : done) {
    g_free.push_back(p.start);
    g_free.push_back(p.stop);
  }
  return rc;
}

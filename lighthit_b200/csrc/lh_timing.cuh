// Kernel timing for measurement runs (see lh_timing.cu): a scope object that
// records a CUDA event pair around the launches made while it lives.
#pragma once

#include <cuda_runtime.h>

#include "../../include/lighthit_b200.h"

namespace lh {

class TimedLaunch {
 public:
  TimedLaunch(int kernel, cudaStream_t stream);
  ~TimedLaunch();
  TimedLaunch(const TimedLaunch&) = delete;
  TimedLaunch& operator=(const TimedLaunch&) = delete;

 private:
  int kernel_;
  cudaStream_t stream_;
  cudaEvent_t start_ = nullptr, stop_ = nullptr;
  bool armed_ = false;
};

// Device counters of algorithmic work units, one per timed kernel id
// (LH_KT_*): a kernel adds its units to kernel_units()[id].
unsigned long long* kernel_units();

}  // namespace lh

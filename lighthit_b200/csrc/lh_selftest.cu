// Failure detection without a fault (no counterpart in the reference).
//
// Every wait of the tensor-core kernels on an mbarrier (bulk copies, MMA
// completion) is bounded in time (mbar_wait, lh_common.cuh): when it gives up
// the kernel sets LH_STATUS_TIMEOUT in its status word, finishes its own
// copies, frees its tensor memory and returns, so the context stays usable and
// the host raises. lh_wait_selftest runs one such wait on an mbarrier that
// nothing completes, so that this path can be checked on a GPU without
// faulting or hanging it.
#include "lh_common.cuh"

namespace lh {

__global__ void wait_selftest_kernel(int32_t* status, long long limit_ns) {
  __shared__ uint64_t bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    fence_barrier_init();
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned long long start = global_ns();
    const bool ok = mbar_wait(&bar, 0, limit_ns);  // no thread arrives: runs out
    const unsigned long long waited = global_ns() - start;
    if (!ok) atomicOr(reinterpret_cast<unsigned*>(status), LH_STATUS_TIMEOUT);
    *reinterpret_cast<unsigned long long*>(status + 2) = waited;
  }
}

}  // namespace lh

extern "C" int lh_wait_selftest(int32_t* status, int64_t limit_ns, void* stream) {
  if (!status || (reinterpret_cast<uintptr_t>(status) & 7) || limit_ns <= 0 ||
      limit_ns > lh::kWaitLimitNs)
    return LH_EINVAL;
  lh::wait_selftest_kernel<<<1, 32, 0, static_cast<cudaStream_t>(stream)>>>(status,
                                                                           (long long)limit_ns);
  return cudaGetLastError() == cudaSuccess ? LH_OK : LH_ECUDA;
}

// Flash transport for callers that cannot allocate device memory.
//
// lh_flash_transport needs a caller-supplied workspace for the readout rows of
// the plain FP32 path. Some callers have no way to provide one: a trigger or
// data-acquisition process whose device memory is reserved up front by its own
// framework allocator, or a latency-critical loop in which cudaMalloc/cudaFree
// would synchronise the device. lh_flash_transport_noalloc runs the same plain
// FP32 kernels with their scratch in a file-scope __device__ array instead, so
// the call allocates nothing; the caller still passes inputs and outputs.
//
// The array's host-side name is only a stand-in for the symbol, not a device
// address. Its device address is looked up with cudaGetSymbolAddress once per
// device, with that device current, on the first call made on that device; that
// first call should therefore come before any stream capture. The address is
// cached for the life of the process; cudaDeviceReset ends the context it
// belongs to, so a process that resets a device must not call this entry point
// on that device afterwards. Every call on a device shares the one array and it
// keeps the last call's contents: calls whose work overlaps on the GPU (other
// streams, other host threads) race on it and must be serialised by the caller.
#include <cstdio>
#include <mutex>

#include "lh_common.cuh"
#include "lh_readout.cuh"

namespace lh {
__global__ void flash_plain_kernel(lh_flash_problem p, lh_flash_batch b, int kpad, int n_bins,
                                   float* a_rows);
}  // namespace lh

// 4 MiB: the readout rows of 2 * n_flash * n_om rows of k_pad floats, e.g. 75
// flashes on a 48-OM array at k_pad = 144. Held by every GPU that loads the
// library until the process exits.
constexpr size_t kScratchBytes = size_t(4) << 20;
static __device__ __align__(256) unsigned char g_flash_scratch[kScratchBytes];

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_lock;
void* g_scratch_ptr[kMaxDevices] = {};

// Device address of the scratch array on the current device (looked up once).
int scratch_address(void** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return LH_ECUDA;
  if (dev < 0 || dev >= kMaxDevices) return LH_EUNSUPPORTED;
  std::lock_guard<std::mutex> guard(g_lock);
  if (!g_scratch_ptr[dev]) {
    void* ptr = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&ptr, g_flash_scratch);
    if (e != cudaSuccess || !ptr) {
      fprintf(stderr, "lighthit_b200: cudaGetSymbolAddress(scratch) failed: %s\n",
              cudaGetErrorString(e));
      return LH_ECUDA;
    }
    g_scratch_ptr[dev] = ptr;
  }
  *out = g_scratch_ptr[dev];
  return LH_OK;
}

}  // namespace

extern "C" int lh_flash_transport_noalloc(const lh_flash_problem* p, const lh_readout_operator* op,
                                          const lh_flash_batch* b, void* stream) {
  using namespace lh;
  if (!p || !b || !op || p->n_om <= 0 || b->n_flash < 0 || p->acc_top < 0 || p->acc_top > 8 ||
      p->n_omega < 2 || op->k_pad <= 0 || op->k_pad % 16 != 0 || 2 * p->n_omega > op->k_pad ||
      p->n_radii < 4 || p->n_edges < 2 || op->n_bins != p->n_edges - 1 || !op->b_fp32 ||
      !b->status)
    return LH_EINVAL;
  if (b->n_flash == 0) return LH_OK;
  const int64_t n_pairs = (int64_t)b->n_flash * p->n_om;
  const size_t need = (size_t)2 * n_pairs * op->k_pad * sizeof(float);
  if (need > kScratchBytes) {
    fprintf(stderr,
            "lighthit_b200: lh_flash_transport_noalloc needs %zu bytes of scratch for %d flashes "
            "x %d OMs; its static scratch holds %zu bytes\n",
            need, b->n_flash, p->n_om, kScratchBytes);
    return LH_ESCRATCH;
  }
  void* scratch = nullptr;
  int rc = scratch_address(&scratch);
  if (rc != LH_OK) return rc;
  // Nothing in the scratch has to start at zero: flash_plain_kernel writes all
  // 2 * n_flash * n_om rows the readout reads (zero rows for flashes past a
  // device count, every padding column zeroed), so no earlier call's rows
  // reach the output.
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  float* rows = static_cast<float*>(scratch);
  const int64_t tiles = (n_pairs + 63) / 64;
  flash_plain_kernel<<<(unsigned)tiles, 256, 0, s>>>(*p, *b, op->k_pad, op->n_bins, rows);
  if (cudaGetLastError() != cudaSuccess) return LH_ECUDA;
  RowMap map{2, 3ll * op->n_bins, op->n_bins};
  dim3 grid((unsigned)((2 * n_pairs + 7) / 8), (op->n_bins + 31) / 32);
  readout_fp32_kernel<<<grid, dim3(32, 8), 8 * op->k_pad * sizeof(float), s>>>(
      rows, 2 * n_pairs, op->k_pad, op->b_fp32, op->n_bins, map, b->components + op->n_bins);
  return cudaGetLastError() == cudaSuccess ? LH_OK : LH_ECUDA;
}

// Readout kernels shared by the flash and shower paths.
#pragma once
#include <cstdint>
#include <cuda_bf16.h>

namespace lh {

// Output row placement: row r goes to (r / g) * group_stride + (r % g) * row_stride.
struct RowMap {
  int g;
  int64_t group_stride;
  int64_t row_stride;
  __host__ __device__ int64_t offset(int64_t row) const {
    return (row / g) * group_stride + (row % g) * row_stride;
  }
};

__global__ void readout_pack_fp32_kernel(const float2* spec, int n_omega, int64_t rows, int kpad,
                                         float* a);
__global__ void readout_pack_bf16_kernel(const float2* spec, int n_omega, int64_t rows, int kpad,
                                         __nv_bfloat16* a_hi, __nv_bfloat16* a_lo);
__global__ void readout_fp32_kernel(const float* a, int64_t rows, int kpad, const float* b,
                                    int n_bins, RowMap map, float* out);
__global__ void readout_tc_kernel(const __nv_bfloat16* a_hi, const __nv_bfloat16* a_lo,
                                  int64_t rows, int kpad, const __nv_bfloat16* b_hi,
                                  const __nv_bfloat16* b_lo, int n_bins, int n_tile, int n_tiles,
                                  int passes, RowMap map, float* out, int32_t* status);
size_t readout_tc_smem_bytes(int kpad, int n_tile);

}  // namespace lh

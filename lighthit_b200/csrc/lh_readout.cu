// Spectrum -> time-bin readout (reference readout.py:18-72).
//
// The reference demodulates each OM's spectrum by its clock, refines 65 -> 321
// frequencies with a not-a-knot cubic spline and integrates every bin exactly
// (inverse_bins). All of that is linear in the spectrum, so the host folds it
// into one real operator B[bin][k] over the packed relative spectrum
// (Re w_0..w_{n-1}, Im w_0..w_{n-1}); the device runs one GEMM:
//
//   bins[row][bin] = sum_k A[row][k] * B[bin][k]
//
// * readout_fp32_kernel: CUDA-core fp32, the plain GPU path.
// * readout_tc_kernel: tcgen05.mma, 128-row tiles, BF16 operands with an
//   optional hi+lo split (A_hi*B_hi + A_hi*B_lo + A_lo*B_hi, fp32 accumulate in
//   TMEM) that keeps ~16 significant bits. Tiles stream in by cp.async.bulk.
#include "lh_common.cuh"
#include "lh_readout.cuh"

namespace lh {

// ---------------------------------------------------------------- packing
__global__ void readout_pack_fp32_kernel(const float2* __restrict__ spec, int n_omega,
                                         int64_t rows, int kpad, float* __restrict__ a) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  int64_t total = rows * kpad;
  if (i >= total) return;
  int64_t row = i / kpad;
  int k = (int)(i % kpad);
  float v = 0.f;
  if (k < n_omega) v = spec[row * n_omega + k].x;
  else if (k < 2 * n_omega) v = spec[row * n_omega + (k - n_omega)].y;
  a[i] = v;
}

__global__ void readout_pack_bf16_kernel(const float2* __restrict__ spec, int n_omega,
                                         int64_t rows, int kpad,
                                         __nv_bfloat16* __restrict__ a_hi,
                                         __nv_bfloat16* __restrict__ a_lo) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  int64_t tiles = (rows + 127) / 128;
  int64_t total = tiles * 128 * kpad;
  if (i >= total) return;
  int64_t row = i / kpad;
  int k = (int)(i % kpad);
  float v = 0.f;
  if (row < rows) {
    if (k < n_omega) v = spec[row * n_omega + k].x;
    else if (k < 2 * n_omega) v = spec[row * n_omega + (k - n_omega)].y;
  }
  int64_t off = (row / 128) * (int64_t)128 * kpad + tile_offset((int)(row % 128), k);
  __nv_bfloat16 hi, lo;
  split_bf16(v, hi, lo);
  a_hi[off] = hi;
  if (a_lo) a_lo[off] = lo;
}

// ---------------------------------------------------------------- plain fp32
// One thread per (row, bin); 32 bins x 8 rows per block, A rows staged in smem.
__global__ void readout_fp32_kernel(const float* __restrict__ a, int64_t rows, int kpad,
                                    const float* __restrict__ b, int n_bins, RowMap map,
                                    float* __restrict__ out) {
  extern __shared__ float sa[];  // [8][kpad]
  int64_t row0 = blockIdx.x * 8ll;
  for (int i = threadIdx.y * 32 + threadIdx.x; i < 8 * kpad; i += 256) {
    int64_t r = row0 + i / kpad;
    sa[i] = r < rows ? a[r * kpad + (i % kpad)] : 0.f;
  }
  __syncthreads();
  int bin = blockIdx.y * 32 + threadIdx.x;
  int64_t row = row0 + threadIdx.y;
  if (bin >= n_bins || row >= rows) return;
  const float* br = b + (int64_t)bin * kpad;
  const float* ar = sa + threadIdx.y * kpad;
  float acc = 0.f;
  for (int k = 0; k < kpad; ++k) acc = fmaf(ar[k], __ldg(br + k), acc);
  out[map.offset(row) + bin] = acc;
}

// ---------------------------------------------------------------- tcgen05
// 128 threads (4 warps). Persistent over 128-row tiles; each tile is loaded
// with one bulk copy per operand part, multiplied against every N tile of B,
// and drained from TMEM by the four warps (warp w owns TMEM lanes 32w..32w+31).
__global__ void __launch_bounds__(128, 1)
readout_tc_kernel(const __nv_bfloat16* __restrict__ a_hi, const __nv_bfloat16* __restrict__ a_lo,
                  int64_t rows, int kpad, const __nv_bfloat16* __restrict__ b_hi,
                  const __nv_bfloat16* __restrict__ b_lo, int n_bins, int n_tile, int n_tiles,
                  int passes, RowMap map, float* __restrict__ out, int32_t* status) {
  extern __shared__ __align__(1024) uint8_t smem[];
  const uint32_t a_bytes = 128u * kpad * 2u;
  const uint32_t b_bytes = (uint32_t)n_tile * kpad * 2u;
  __nv_bfloat16* s_ahi = reinterpret_cast<__nv_bfloat16*>(smem);
  __nv_bfloat16* s_alo = reinterpret_cast<__nv_bfloat16*>(smem + a_bytes);
  __nv_bfloat16* s_bhi = reinterpret_cast<__nv_bfloat16*>(smem + 2 * a_bytes);
  __nv_bfloat16* s_blo = reinterpret_cast<__nv_bfloat16*>(smem + 2 * a_bytes + b_bytes);
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + 2 * a_bytes + 2 * b_bytes);
  uint32_t* s_tmem = reinterpret_cast<uint32_t*>(bars + 2);
  int* s_fail = reinterpret_cast<int*>(s_tmem + 1);
  uint64_t* bar_load = bars;
  uint64_t* bar_mma = bars + 1;

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const bool need_lo_a = passes >= 3;
  const bool need_lo_b = passes >= 2;
  if (tid == 0) {
    mbar_init(bar_load, 1);
    mbar_init(bar_mma, 1);
    *s_fail = 0;
    fence_barrier_init();
  }
  if (warp == 0) {
    tmem_alloc(s_tmem, 256);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *s_tmem;
  const uint32_t idesc = instr_desc_bf16_f32(128, n_tile);
  uint32_t ph_load = 0, ph_mma = 0;
  const int64_t row_tiles = (rows + 127) / 128;
  bool failed = false, mma_pending = false;

  for (int64_t tile = blockIdx.x; tile < row_tiles && !failed; tile += gridDim.x) {
    for (int nt = 0; nt < n_tiles && !failed; ++nt) {
      if (tid == 0) {
        uint32_t bytes = 0;
        bool load_a = (nt == 0);
        bool load_b = (n_tiles > 1) || (tile == blockIdx.x);
        if (load_a) bytes += a_bytes * (need_lo_a ? 2u : 1u);
        if (load_b) bytes += b_bytes * (need_lo_b ? 2u : 1u);
        mbar_expect_tx(bar_load, bytes);
        if (load_a) {
          bulk_g2s(s_ahi, a_hi + tile * 128ll * kpad, a_bytes, bar_load);
          if (need_lo_a) bulk_g2s(s_alo, a_lo + tile * 128ll * kpad, a_bytes, bar_load);
        }
        if (load_b) {
          bulk_g2s(s_bhi, b_hi + (int64_t)nt * n_tile * kpad, b_bytes, bar_load);
          if (need_lo_b) bulk_g2s(s_blo, b_lo + (int64_t)nt * n_tile * kpad, b_bytes, bar_load);
        }
      }
      bool ok = mbar_wait(bar_load, ph_load);
      ph_load ^= 1u;
      if (__syncthreads_or(!ok)) { failed = true; break; }
      tc_fence_after();
      if (tid == 0) {
        const int ksteps = kpad / 16;
        const uint32_t lbo_a = 128u * 16u, lbo_b = (uint32_t)n_tile * 16u;
        int first = 1;
        for (int pass = 0; pass < passes; ++pass) {
          const __nv_bfloat16* pa = (pass == 2) ? s_alo : s_ahi;
          const __nv_bfloat16* pb = (pass == 1) ? s_blo : s_bhi;
          for (int kk = 0; kk < ksteps; ++kk) {
            uint64_t da = smem_desc_kmajor(reinterpret_cast<const uint8_t*>(pa) + kk * 2 * lbo_a,
                                           lbo_a, 128);
            uint64_t db = smem_desc_kmajor(reinterpret_cast<const uint8_t*>(pb) + kk * 2 * lbo_b,
                                           lbo_b, 128);
            tc_mma_bf16(tmem, da, db, idesc, first ? 0u : 1u);
            first = 0;
          }
        }
        tc_commit(bar_mma);
      }
      ok = mbar_wait(bar_mma, ph_mma);
      ph_mma ^= 1u;
      if (__syncthreads_or(!ok)) { failed = true; mma_pending = true; break; }
      tc_fence_after();
      // epilogue: warp w drains TMEM lanes 32w..32w+31
      const int64_t row = tile * 128 + warp * 32 + lane;
      const uint32_t lane_addr = tmem + ((uint32_t)(warp * 32) << 16);
      for (int c0 = 0; c0 < n_tile; c0 += 16) {
        float v[16];
        tmem_ld16(lane_addr + (uint32_t)c0, v);
        if (row < rows) {
          float* dst = out + map.offset(row) + (int64_t)nt * n_tile + c0;
          int bin0 = nt * n_tile + c0;
#pragma unroll
          for (int i = 0; i < 16; ++i)
            if (bin0 + i < n_bins) dst[i] = v[i];
        }
      }
      tc_fence_before();
      __syncthreads();
    }
  }
  if (failed && tid == 0) atomicOr(reinterpret_cast<unsigned*>(status), LH_STATUS_TIMEOUT);
  // Drain anything still in flight before releasing TMEM (bounded waits).
  if (mma_pending) mbar_wait(bar_mma, ph_mma ^ 1u);
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, 256);
}

size_t readout_tc_smem_bytes(int kpad, int n_tile) {
  return 2ull * 128 * kpad * 2 + 2ull * n_tile * kpad * 2 + 64;
}

}  // namespace lh

// C ABI entry points (include/lighthit_b200.h): argument checks, launch
// shapes and shared-memory opt-in. No allocation happens here; callers pass
// device buffers and a workspace.
#include <cstdio>

#include "lh_common.cuh"
#include "lh_timing.cuh"
#include "lh_readout.cuh"

namespace lh {
__global__ void flash_plain_kernel(lh_flash_problem p, lh_flash_batch b, int kpad, int n_bins,
                                   float* a_rows);
__global__ void flash_tc_kernel(lh_flash_problem p, lh_flash_batch b, const __nv_bfloat16* g_bhi,
                                const __nv_bfloat16* g_blo, int kpad, int n_bins, int n_tile,
                                int passes);
size_t flash_tc_smem_bytes(int kpad, int n_tile);
__global__ void flash_combine_kernel(lh_flash_problem p, lh_flash_nodes nd, lh_flash_batch b);
}  // namespace lh

using namespace lh;

namespace {

int sm_count() {
  static int count = 0;
  if (!count) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&count, cudaDevAttrMultiProcessorCount, dev);
    if (count <= 0) count = 148;
  }
  return count;
}

int check_launch() {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    fprintf(stderr, "lighthit_b200: launch failed: %s\n", cudaGetErrorString(e));
    return LH_ECUDA;
  }
  return LH_OK;
}

int passes_of(int mode) { return mode == LH_MODE_SPLIT_BF16 ? 3 : 1; }

bool op_valid(const lh_readout_operator* op) {
  return op && op->n_bins > 0 && op->k_pad > 0 && op->k_pad % 16 == 0 && op->n_tile > 0 &&
         op->n_tile % 16 == 0 && op->n_tile <= 256 && op->n_tiles >= 1 &&
         (int64_t)op->n_tile * op->n_tiles >= op->n_bins;
}

}  // namespace

extern "C" {

const char* lh_version(void) { return "lighthit_b200 0.1 (sm_100a)"; }

size_t lh_readout_packed_bytes(const lh_readout_operator* op, int mode, int64_t rows) {
  if (!op_valid(op) || rows < 0) return 0;
  if (mode == LH_MODE_PLAIN_FP32) return (size_t)rows * op->k_pad * sizeof(float);
  const int64_t tiles = (rows + 127) / 128;
  const size_t one = (size_t)tiles * 128 * op->k_pad * 2;
  return mode == LH_MODE_SPLIT_BF16 ? 2 * one : one;
}

int lh_readout_pack(const lh_readout_operator* op, int mode, const float* spectra_c64,
                    int32_t n_omega, int64_t rows, void* a_packed, void* stream) {
  if (!op_valid(op) || !spectra_c64 || !a_packed || rows < 0 || 2 * n_omega > op->k_pad)
    return LH_EINVAL;
  if (rows == 0) return LH_OK;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const float2* spec = reinterpret_cast<const float2*>(spectra_c64);
  if (mode == LH_MODE_PLAIN_FP32) {
    int64_t total = rows * op->k_pad;
    readout_pack_fp32_kernel<<<(unsigned)((total + 255) / 256), 256, 0, s>>>(
        spec, n_omega, rows, op->k_pad, static_cast<float*>(a_packed));
  } else {
    const int64_t tiles = (rows + 127) / 128;
    int64_t total = tiles * 128 * op->k_pad;
    __nv_bfloat16* hi = static_cast<__nv_bfloat16*>(a_packed);
    __nv_bfloat16* lo = mode == LH_MODE_SPLIT_BF16 ? hi + tiles * 128 * op->k_pad : nullptr;
    readout_pack_bf16_kernel<<<(unsigned)((total + 255) / 256), 256, 0, s>>>(
        spec, n_omega, rows, op->k_pad, hi, lo);
  }
  return check_launch();
}

int lh_readout_rows(const lh_readout_operator* op, int mode, const void* a_packed, int64_t rows,
                    float* out, int64_t out_row_stride, int32_t* status, void* stream) {
  if (!op_valid(op) || !a_packed || !out || rows < 0 || out_row_stride < op->n_bins)
    return LH_EINVAL;
  if (rows == 0) return LH_OK;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  RowMap map{1, out_row_stride, out_row_stride};
  if (mode == LH_MODE_PLAIN_FP32) {
    dim3 grid((unsigned)((rows + 7) / 8), (op->n_bins + 31) / 32);
    size_t smem = 8 * op->k_pad * sizeof(float);
    readout_fp32_kernel<<<grid, dim3(32, 8), smem, s>>>(static_cast<const float*>(a_packed), rows,
                                                        op->k_pad, op->b_fp32, op->n_bins, map,
                                                        out);
    return check_launch();
  }
  if (!status) return LH_EINVAL;
  const int64_t tiles = (rows + 127) / 128;
  const __nv_bfloat16* hi = static_cast<const __nv_bfloat16*>(a_packed);
  const __nv_bfloat16* lo = mode == LH_MODE_SPLIT_BF16 ? hi + tiles * 128 * op->k_pad : nullptr;
  size_t smem = readout_tc_smem_bytes(op->k_pad, op->n_tile);
  if (smem > 227 * 1024) return LH_EUNSUPPORTED;
  cudaFuncSetAttribute(readout_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  int grid = (int)(tiles < sm_count() ? tiles : sm_count());
  {
    lh::TimedLaunch timed_launch(LH_KT_READOUT, s);
    readout_tc_kernel<<<grid, 128, smem, s>>>(
        hi, lo, rows, op->k_pad, reinterpret_cast<const __nv_bfloat16*>(op->b_hi),
        reinterpret_cast<const __nv_bfloat16*>(op->b_lo), op->n_bins, op->n_tile, op->n_tiles,
        passes_of(mode), map, out, status);
  }
  return check_launch();
}

size_t lh_flash_workspace_bytes(const lh_flash_problem* p, const lh_readout_operator* op,
                                int mode, int32_t n_flash) {
  if (!p || !op_valid(op) || n_flash < 0) return 0;
  if (mode != LH_MODE_PLAIN_FP32) return 0;  // the fused kernel keeps its rows on chip
  return (size_t)2 * n_flash * p->n_om * op->k_pad * sizeof(float);
}

int lh_flash_transport(const lh_flash_problem* p, const lh_readout_operator* op, int mode,
                       const lh_flash_batch* b, void* workspace, size_t workspace_bytes,
                       void* stream) {
  if (!p || !b || !op_valid(op) || p->n_om <= 0 || b->n_flash < 0 || p->acc_top < 0 ||
      p->acc_top > 8 || p->n_omega < 2 || 2 * p->n_omega > op->k_pad || p->n_radii < 4 ||
      p->n_edges < 2 || op->n_bins != p->n_edges - 1 || !b->status)
    return LH_EINVAL;
  if (b->n_flash == 0) return LH_OK;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int64_t n_pairs = (int64_t)b->n_flash * p->n_om;
  const int64_t tiles = (n_pairs + 63) / 64;
  if (mode == LH_MODE_PLAIN_FP32) {
    size_t need = lh_flash_workspace_bytes(p, op, mode, b->n_flash);
    if (!workspace || workspace_bytes < need) return LH_ENOMEM;
    float* rows = static_cast<float*>(workspace);
    flash_plain_kernel<<<(unsigned)tiles, 256, 0, s>>>(*p, *b, op->k_pad, op->n_bins, rows);
    int rc = check_launch();
    if (rc) return rc;
    RowMap map{2, 3ll * op->n_bins, op->n_bins};
    dim3 grid((unsigned)((2 * n_pairs + 7) / 8), (op->n_bins + 31) / 32);
    readout_fp32_kernel<<<grid, dim3(32, 8), 8 * op->k_pad * sizeof(float), s>>>(
        rows, 2 * n_pairs, op->k_pad, op->b_fp32, op->n_bins, map, b->components + op->n_bins);
    return check_launch();
  }
  if (op->n_tiles != 1) return LH_EUNSUPPORTED;  // fused path: all bins in one tile
  size_t smem = flash_tc_smem_bytes(op->k_pad, op->n_tile);
  if (smem > 227 * 1024) return LH_EUNSUPPORTED;
  cudaFuncSetAttribute(flash_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  int grid = (int)(tiles < sm_count() ? tiles : sm_count());
  const int threads = b->block_threads == 0 ? 512 : b->block_threads;
  if (threads != 256 && threads != 512) return LH_EINVAL;
  {
    lh::TimedLaunch timed_launch(LH_KT_FLASH, s);
    flash_tc_kernel<<<grid, threads, smem, s>>>(*p, *b, reinterpret_cast<const __nv_bfloat16*>(op->b_hi),
                                            reinterpret_cast<const __nv_bfloat16*>(op->b_lo),
                                            op->k_pad, op->n_bins, op->n_tile, passes_of(mode));
  }
  return check_launch();
}

int lh_flash_combine(const lh_flash_problem* p, const lh_flash_nodes* nodes,
                     const lh_flash_batch* b, void* stream) {
  if (!p || !nodes || !b || p->n_om <= 0 || b->n_flash < 0 || p->acc_top < 0 || p->acc_top > 8 ||
      p->n_omega < 1 || p->n_edges < 2 || nodes->n_nodes < 1 ||
      nodes->n_nodes > LH_FLASH_MAX_NODES || !b->status || !b->spectrum || !b->components ||
      !b->charge || !b->active || !b->pos)
    return LH_EINVAL;
  for (int n = 0; n < nodes->n_nodes; ++n)
    if (!nodes->spectrum[n] || !nodes->components[n] || !nodes->charge[n] || !nodes->photons[n])
      return LH_EINVAL;
  if (b->n_flash == 0) return LH_OK;
  const int64_t work = (int64_t)b->n_flash * p->n_om * p->n_omega * 6;
  const int64_t want = (work + 255) / 256;
  const int grid = (int)(want < 16 * sm_count() ? want : 16 * sm_count());
  flash_combine_kernel<<<grid, 256, 0, static_cast<cudaStream_t>(stream)>>>(*p, *nodes, *b);
  return check_launch();
}

}  // extern "C"

namespace lh {
size_t ge2_workspace(const lh_ge2_table& T, const lh_ge2_problem& P);
int ge2_launch(const lh_ge2_table& T, const lh_ge2_problem& P, void* ws, cudaStream_t s);
size_t ge2_slot_size();
size_t ge2_batch_workspace(const lh_ge2_table& T, const lh_ge2_problem* P, int32_t n);
int ge2_batch_launch(const lh_ge2_table& T, const lh_ge2_problem* P, int32_t n, void* ws,
                     void* host_slots, cudaStream_t s);
}  // namespace lh

namespace {
bool ge2_valid(const lh_ge2_table* t, const lh_ge2_problem* p) {
  if (!t || !p) return false;
  if (t->n_bands < 1 || t->n_intervals < 1 || t->degree < 0 || t->degree > 16 ||
      t->acc_degree < 0 || t->acc_degree > 4 || t->max_m < 0 || t->max_m > 4 ||
      t->max_m > t->degree || t->n_pairs < 1 || t->n_pairs > 8 || t->nch < 1 ||
      t->n_omega < 1 || t->jmax < t->max_m || t->jmax < t->acc_degree)
    return false;
  if (!t->coef || !t->log_r || !t->absorption || !t->speed || !t->omega || !t->pair_lambda ||
      !t->pair_mu || !t->alpha || !t->starts || !t->start_norm)
    return false;
  if (p->n_points < 0 || p->n_om < 0 || p->n_omega < 1 || p->n_omega > t->n_omega ||
      p->n_omega_channels < p->n_omega || !p->result)
    return false;
  if (p->n_points && (!p->points || !p->channels)) return false;
  if (p->n_om && (!p->receivers || !p->looks || !p->out_scale)) return false;
  if ((size_t)t->nch * t->n_pairs * 32 * sizeof(float) + 32 * 128 * 8 > 200 * 1024) return false;
  return true;
}
}  // namespace

extern "C" size_t lh_ge2_workspace_bytes(const lh_ge2_table* t, const lh_ge2_problem* p) {
  if (!ge2_valid(t, p)) return 0;
  return lh::ge2_workspace(*t, *p);
}

extern "C" int lh_ge2_apply(const lh_ge2_table* t, const lh_ge2_problem* p, void* workspace,
                            size_t workspace_bytes, void* stream) {
  if (!ge2_valid(t, p)) return LH_EINVAL;
  if (p->n_om == 0) return LH_OK;
  if (!workspace || workspace_bytes < lh::ge2_workspace(*t, *p)) return LH_ENOMEM;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (p->n_points == 0) {
    cudaMemsetAsync(p->result, 0, (size_t)p->n_om * p->n_omega * 2 * sizeof(double), s);
    return cudaGetLastError() == cudaSuccess ? LH_OK : LH_ECUDA;
  }
  return lh::ge2_launch(*t, *p, workspace, s);
}

extern "C" size_t lh_ge2_batch_workspace_bytes(const lh_ge2_table* t, const lh_ge2_problem* p,
                                               int32_t n) {
  if (!t || !p || n < 1 || n > 65535) return 0;
  for (int i = 0; i < n; ++i)
    if (!ge2_valid(t, p + i)) return 0;
  return lh::ge2_batch_workspace(*t, p, n);
}

extern "C" size_t lh_ge2_batch_slot_bytes(int32_t n) {
  return n < 1 ? 0 : (size_t)n * lh::ge2_slot_size();
}

extern "C" int lh_ge2_apply_batch(const lh_ge2_table* t, const lh_ge2_problem* p, int32_t n,
                                  void* workspace, size_t workspace_bytes, void* host_slots,
                                  void* stream) {
  if (!t || !p || n < 1 || n > 65535 || !host_slots) return LH_EINVAL;
  for (int i = 0; i < n; ++i)
    if (!ge2_valid(t, p + i)) return LH_EINVAL;
  if (!workspace || workspace_bytes < lh::ge2_batch_workspace(*t, p, n)) return LH_ENOMEM;
  return lh::ge2_batch_launch(*t, p, n, workspace, host_slots, static_cast<cudaStream_t>(stream));
}

namespace lh {
bool ge2_tc_supported(const lh_ge2_table& T, int& halves, int& n_pad_max);
size_t ge2_tc_pack_bytes(const lh_ge2_table& T);
int ge2_tc_pack(const lh_ge2_table& T, void* packed, cudaStream_t s);
size_t ge2_tc_workspace(const lh_ge2_table& T, const lh_ge2_problem* P, int32_t n);
int ge2_tc_batch_launch(const lh_ge2_table& T, const lh_ge2_problem* P, int32_t n, int passes,
                        const void* packed, void* ws, void* host_slots, int32_t* status,
                        cudaStream_t s);
}  // namespace lh

extern "C" size_t lh_ge2_tc_pack_bytes(const lh_ge2_table* t) {
  if (!t || t->n_bands < 1 || t->n_intervals < 1 || t->degree < 0 || t->degree > 16 ||
      t->n_pairs < 1 || t->n_pairs > 8 || t->n_omega < 1 || !t->coef)
    return 0;
  return lh::ge2_tc_pack_bytes(*t);
}

extern "C" int lh_ge2_tc_pack(const lh_ge2_table* t, void* packed, size_t packed_bytes,
                              void* stream) {
  const size_t need = lh_ge2_tc_pack_bytes(t);
  if (need == 0) return LH_EUNSUPPORTED;
  if (!packed || packed_bytes < need) return LH_ENOMEM;
  if (reinterpret_cast<uintptr_t>(packed) % 16) return LH_EINVAL;  // bulk copies start there
  return lh::ge2_tc_pack(*t, packed, static_cast<cudaStream_t>(stream));
}

extern "C" size_t lh_ge2_tc_workspace_bytes(const lh_ge2_table* t, const lh_ge2_problem* p,
                                            int32_t n) {
  if (!t || !p || n < 1 || n > 65535 || lh_ge2_tc_pack_bytes(t) == 0) return 0;
  for (int i = 0; i < n; ++i)
    if (!ge2_valid(t, p + i) || p[i].n_omega != t->n_omega) return 0;
  return lh::ge2_tc_workspace(*t, p, n);
}

extern "C" int lh_ge2_apply_batch_tc(const lh_ge2_table* t, const lh_ge2_problem* p, int32_t n,
                                     int32_t mode, const void* packed, void* workspace,
                                     size_t workspace_bytes, void* host_slots, int32_t* status,
                                     void* stream) {
  if (!t || !p || n < 1 || n > 65535 || !host_slots || !packed || !status) return LH_EINVAL;
  if (mode != LH_MODE_SPLIT_BF16 && mode != LH_MODE_BF16) return LH_EINVAL;
  if (lh_ge2_tc_pack_bytes(t) == 0) return LH_EUNSUPPORTED;
  if (reinterpret_cast<uintptr_t>(packed) % 16) return LH_EINVAL;
  for (int i = 0; i < n; ++i)
    if (!ge2_valid(t, p + i) || p[i].n_omega != t->n_omega) return LH_EINVAL;
  if (!workspace || workspace_bytes < lh::ge2_tc_workspace(*t, p, n)) return LH_ENOMEM;
  return lh::ge2_tc_batch_launch(*t, p, n, mode == LH_MODE_SPLIT_BF16 ? 6 : 1, packed, workspace,
                                 host_slots, status, static_cast<cudaStream_t>(stream));
}

// Shared device helpers for the LightHit B200 kernels (sm_100a only).
//
// Inline-PTX wrappers for the Blackwell pieces the kernels use: mbarriers,
// bulk asynchronous copies (cp.async.bulk, no multicast), the 5th-generation
// tensor core (tcgen05.mma with TMEM accumulators) and TMEM loads. Every wait
// on an mbarrier is bounded: after LH_SPIN_LIMIT polls the wait gives up and
// reports a timeout, so a broken pipeline returns an error status instead of
// hanging the GPU.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>
#include <cuda_bf16.h>

#include "../../include/lighthit_b200.h"

#define LH_DEVICE __device__ __forceinline__

namespace lh {

constexpr double kPi = 3.14159265358979323846;
constexpr double kCVacuumMPerNs = 0.299792458;
constexpr long long kWaitLimitNs = 1000000000ll;  // a bounded device wait gives up after 1 s

// ---------------------------------------------------------------- float64 geometry
// The reference computes its geometry in NumPy float64 without fused
// multiply-adds; these helpers keep that rounding so distances, clocks and the
// bin index derived from them are bit-identical.
LH_DEVICE double dot3_rn(double ax, double ay, double az, double bx, double by, double bz) {
  return __dadd_rn(__dadd_rn(__dmul_rn(ax, bx), __dmul_rn(ay, by)), __dmul_rn(az, bz));
}

// searchsorted(edges, x, side="right") - 1 over n ascending values.
LH_DEVICE int bin_right(const double* edges, int n, double x) {
  int lo = 0, hi = n;  // first index with edges[i] > x
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if (edges[mid] > x) hi = mid; else lo = mid + 1;
  }
  return lo - 1;
}

// ---------------------------------------------------------------- mbarrier / bulk copy
LH_DEVICE uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

LH_DEVICE void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count));
}

LH_DEVICE void fence_barrier_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

LH_DEVICE void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

LH_DEVICE void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
               "r"(bytes)
               : "memory");
}

LH_DEVICE void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

// Nanoseconds of the GPU's global timer.
LH_DEVICE unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Returns true when the phase with the given parity completed, false once
// `limit_ns` of global time have passed (checked every 256 polls).
LH_DEVICE bool mbar_wait(uint64_t* bar, uint32_t parity, long long limit_ns = kWaitLimitNs) {
  const uint32_t addr = smem_addr(bar);
  const unsigned long long start = global_ns();
  for (unsigned spin = 0; spin < 0x7fffffffu; ++spin) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(addr), "r"(parity)
        : "memory");
    if (done) return true;
    if ((spin & 255u) == 255u && global_ns() - start > (unsigned long long)limit_ns) return false;
  }
  return false;
}

// Untiled bulk copy global -> shared, completion counted on an mbarrier.
// Both addresses 16-byte aligned, size a multiple of 16.
LH_DEVICE void bulk_g2s(void* smem_dst, const void* gmem_src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_addr(smem_dst)),
      "l"(gmem_src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}

// ---------------------------------------------------------------- tcgen05
// Shared-memory matrix descriptor, K-major, no swizzle: 8-row x 16-byte core
// matrices; ``lbo`` = byte distance between core matrices along K, ``sbo`` =
// byte distance between 8-row groups along M/N.
LH_DEVICE uint64_t smem_desc_kmajor(const void* base, uint32_t lbo, uint32_t sbo) {
  uint64_t addr = smem_addr(base);
  uint64_t d = 0;
  d |= (addr & 0x3FFFFull) >> 4;                 // start address  [0,14)
  d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;    // leading offset [16,30)
  d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;    // stride offset  [32,46)
  d |= 1ull << 46;                               // descriptor version (sm_100)
  // base offset 0, lbo mode 0, layout type 0 (no swizzle)
  return d;
}

// Instruction descriptor: BF16 x BF16 -> FP32, both operands K-major.
__host__ __device__ constexpr uint32_t instr_desc_bf16_f32(int m, int n) {
  return (1u << 4)                      // D format f32
         | (1u << 7)                    // A format bf16
         | (1u << 10)                   // B format bf16
         | ((uint32_t)(n >> 3) << 17)   // N / 8
         | ((uint32_t)(m >> 4) << 24);  // M / 16
}

LH_DEVICE void tc_mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                           uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}

LH_DEVICE void tc_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   smem_addr(bar))
               : "memory");
}

LH_DEVICE void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
LH_DEVICE void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Allocation is warp-wide; the TMEM base address is written to shared memory.
LH_DEVICE void tmem_alloc(uint32_t* dst_smem, uint32_t columns) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                   smem_addr(dst_smem)),
               "r"(columns)
               : "memory");
}
LH_DEVICE void tmem_relinquish() {
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
LH_DEVICE void tmem_dealloc(uint32_t base, uint32_t columns) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(base), "r"(columns)
               : "memory");
}

// 32 lanes x 32 bits x 16 columns: thread i of the warp receives TMEM lane
// (warp's lane quarter + i), columns [col, col+16).
LH_DEVICE void tmem_ld16(uint32_t addr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(addr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// 32 lanes x 32 bits x 8 columns (as tmem_ld16, columns [col, col+8)).
LH_DEVICE void tmem_ld8(uint32_t addr, float (&v)[8]) {
  uint32_t r[8];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7])
      : "r"(addr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 8; ++i) v[i] = __uint_as_float(r[i]);
}

// ---------------------------------------------------------------- bf16 split
// x = hi + lo with both parts bf16: hi carries 8 significant bits, lo the next 8.
LH_DEVICE void split_bf16(float x, __nv_bfloat16& hi, __nv_bfloat16& lo) {
  hi = __float2bfloat16_rn(x);
  lo = __float2bfloat16_rn(x - __bfloat162float(hi));
}

// Offset (in elements) of (row, k) inside a 128-row K-major no-swizzle tile
// with ``kpad`` columns: [k/8][row][k%8].
LH_DEVICE int tile_offset(int row_in_tile, int k) {
  return ((k >> 3) * 128 + row_in_tile) * 8 + (k & 7);
}

}  // namespace lh

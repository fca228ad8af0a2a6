// Order 1 (single scattering) of spectral elements, grouped pencils.
//
// Reference: transport_prompt's grouped order 1 (prompt.py:1020-1258) with
//   stage A  compress (prompt.py:1317-1402): subsegment_cells,
//            compress_subsegments, finish_pencils (_prompt_numba.py:1094-1232,
//            2247-2354): every element is cut into ceil(L / a_step)
//            sub-segments, each sub-segment's Cherenkov ring is sampled at
//            `ring_nodes` azimuths, and the nodes are summed into
//            (0.5 m position cell, cube-sphere direction pixel) pencils that
//            carry 23 moments (weights, mean position/time/direction and their
//            covariances);
//   stage B  grouped_pencils_order1 (_prompt_numba.py:1750-2086): for each OM
//            the pencils are merged into (tau, log r, hemisphere, theta) groups
//            carrying acceptance moments; the groups of one (tau, r) batch
//            share a path grid in asinh((S - r) / sigma), their single-
//            scattering profile is summed on it, and the profile is deposited
//            per wavelength band as exact exp x quadratic panels into the bins
//            (_batch_grid, _batch_add_moments, _batch_deposit, _deposit_panel,
//            _finalize: _prompt_numba.py:157-632).
//
// B200 layout. Stage A: one thread per ring node writes its moments into a
// global open-addressing table keyed by (cell, pixel) with float64 atomics;
// one thread per occupied slot then forms the pencil. Stage B: one thread per
// (OM, pencil) computes the pencil's geometry against the OM and adds its
// moments into that OM's group table (atomics); one CTA per OM sorts its
// group keys in shared memory (bitonic) and emits its batches; a persistent
// grid of CTAs takes batches from the global list, builds each batch's path
// grid and profile in shared memory and deposits its panels; one CTA per OM
// finishes the bins with the prefix pass. Everything is float64, as the
// deposit's global quadratic coefficients in t cancel strongly.
#include <algorithm>

#include "lh_common.cuh"
#include "lh_timing.cuh"

namespace lh {

constexpr int kO1MaxNodes = 2048;
constexpr int kO1MaxMono = 10;
constexpr int kO1MaxValues = 2 * kO1MaxMono + 6;
constexpr int kO1MaxBands = 8;
constexpr int kO1MaxGauss = 64;
constexpr int kO1Moments = 23;
constexpr int kO1SmemSort = 16384;  // group tables up to this size sort in shared memory
constexpr int kO1BatchThreads = 128;

LH_DEVICE uint64_t o1_mix(uint64_t v) {
  v = (v ^ (v >> 30)) * 0xbf58476d1ce4e5b9ull;
  v = (v ^ (v >> 27)) * 0x94d049bb133111ebull;
  return v ^ (v >> 31);
}

// A slot whose claiming thread is still zeroing its row holds its key with
// this bit set (keys stay below 2^62).
constexpr long long kO1Busy = 1ll << 62;
constexpr long long kO1ClaimWaitNs = 100000000ll;  // a wait for a claimed row gives up after 0.1 s

// Insert `key` (>= 0) into an open-addressing table of `capacity` (power of
// two) slots holding -1 when free, whose rows of `n` doubles at `rows` are
// not cleared beforehand: the thread that claims a free slot marks it busy,
// zeroes the slot's row, then publishes the key; a thread that finds its key
// still busy waits for the publication (bounded: past kO1ClaimWaitNs it sets
// LH_STATUS_TIMEOUT and returns -1). Returns the slot, or -1 when the table
// is full (LH_STATUS_OVERFLOW); `fresh` tells whether this call claimed it.
// Only the rows of published slots are ever read.
LH_DEVICE int64_t o1_insert(long long* keys, int64_t capacity, long long key, double* rows,
                            int n, bool& fresh, int32_t* status, bool ordered = false) {
  const uint64_t mask = (uint64_t)capacity - 1;
  uint64_t slot = (ordered ? (uint64_t)key : o1_mix((uint64_t)key)) & mask;
  fresh = false;
  unsigned long long* word = reinterpret_cast<unsigned long long*>(keys);
  for (int64_t probe = 0; probe < capacity; ++probe) {
    const long long prev = (long long)atomicCAS(word + slot, (unsigned long long)(-1ll),
                                                (unsigned long long)(key | kO1Busy));
    if (prev == -1ll) {
      double* row = rows + (int64_t)slot * n;
      for (int k = 0; k < n; ++k) row[k] = 0.0;
      __threadfence();  // the zeros reach the device before the key does
      atomicExch(word + slot, (unsigned long long)key);
      fresh = true;
      return (int64_t)slot;
    }
    if (prev == key) return (int64_t)slot;
    if (prev == (key | kO1Busy)) {
      const unsigned long long began = global_ns();
      for (int poll = 0;; ++poll) {
        if ((long long)atomicAdd(word + slot, 0ull) == key) {
          __threadfence();  // the row's zeros before this thread's additions
          return (int64_t)slot;
        }
        if ((poll & 63) == 63 && (long long)(global_ns() - began) > kO1ClaimWaitNs) {
          atomicOr(reinterpret_cast<unsigned*>(status), LH_STATUS_TIMEOUT);
          return -1;
        }
      }
    }
    slot = (slot + 1) & mask;
  }
  atomicOr(reinterpret_cast<unsigned*>(status), LH_STATUS_OVERFLOW);
  return -1;
}

// ------------------------------------------------------------------ stage A

// Equi-angular cube-sphere pixel (_prompt_numba.py:1015-1043)
LH_DEVICE int o1_pixel(double sx, double sy, double sz, int n_face) {
  const double ax = fabs(sx), ay = fabs(sy), az = fabs(sz);
  int face;
  double u, v;
  if (ax >= ay && ax >= az) {
    face = sx > 0 ? 0 : 1; u = sy / ax; v = sz / ax;
  } else if (ay >= az) {
    face = sy > 0 ? 2 : 3; u = sx / ay; v = sz / ay;
  } else {
    face = sz > 0 ? 4 : 5; u = sx / az; v = sy / az;
  }
  const double quarter = 0.25 * kPi;
  int i = (int)((atan(u) + quarter) / (2.0 * quarter) * n_face);
  int j = (int)((atan(v) + quarter) / (2.0 * quarter) * n_face);
  i = min(max(i, 0), n_face - 1);
  j = min(max(j, 0), n_face - 1);
  return (face * n_face + i) * n_face + j;
}

struct O1Subseg {
  double px, py, pz, t;
};

LH_DEVICE O1Subseg o1_subseg(const lh_order1_elements& E, int64_t i, int64_t ia, int64_t n_a) {
  const double frac = (ia + 0.5) / n_a;
  O1Subseg s;
  s.px = E.start[3 * i] + frac * E.length[i] * E.direction[3 * i];
  s.py = E.start[3 * i + 1] + frac * E.length[i] * E.direction[3 * i + 1];
  s.pz = E.start[3 * i + 2] + frac * E.length[i] * E.direction[3 * i + 2];
  s.t = E.t0[i] + frac * (E.t1[i] - E.t0[i]);
  return s;
}

constexpr int kO1CoopGroups = 8;  // at most this many groups per warp: summed by the whole warp

// Warp-level sums by key: every lane writes its n values to its row of the
// warp's staging area (`stage`, 32 rows of n doubles in shared memory), and
// each group of lanes with equal keys (`group`, a __match_any_sync mask; its
// lowest lane the `leader`, holding the group's `row`) adds its members' rows
// in lane order with one atomic per value. With few groups the whole warp
// takes one group at a time (lane k sums value k); with many, each leader
// sums its own group's values one after another. Both sum in the same order.
LH_DEVICE void o1_warp_group_add(double* stage, int n, unsigned group, bool leader, double* row) {
  __syncwarp();
  const unsigned full = 0xffffffffu;
  unsigned leaders = __ballot_sync(full, leader && row != nullptr);
  if (__popc(leaders) <= kO1CoopGroups) {
    const int lane = threadIdx.x & 31;
    while (leaders) {
      const int src = __ffs(leaders) - 1;
      leaders &= leaders - 1;
      const unsigned members = __shfl_sync(full, group, src);
      double* target = reinterpret_cast<double*>(
          __shfl_sync(full, reinterpret_cast<unsigned long long>(row), src));
      for (int k = lane; k < n; k += 32) {
        double sum = 0.0;
        for (unsigned g = members; g; g &= g - 1) sum += stage[(__ffs(g) - 1) * n + k];
        atomicAdd(target + k, sum);
      }
    }
  } else if (leader && row) {
    for (int k = 0; k < n; ++k) {
      double sum = 0.0;
      for (unsigned g = group; g; g &= g - 1) sum += stage[(__ffs(g) - 1) * n + k];
      atomicAdd(row + k, sum);
    }
  }
  __syncwarp();
}

constexpr int kO1RingBlock = 4;     // ring nodes per thread
constexpr int kO1RingThreads = 256;

// One thread per (sub-segment, block of kO1RingBlock ring nodes):
// compress_subsegments (_prompt_numba.py:1122-1232) with the ring rotation
// evaluated directly. The lanes of a warp hold consecutive sub-segments and
// take the same ring node together, so nodes that land in the same (cell,
// pixel) (neighbouring steps of a track or shower) are summed in registers
// first: one hash insert and one set of moment atomics per distinct key and warp.
__global__ void __launch_bounds__(kO1RingThreads)
o1_ring_kernel(const lh_order1_config C, const lh_order1_elements E,
                               const int64_t* subseg_offset, int64_t n_subseg,
                               long long* keys, int64_t capacity, double* rows,
                               int32_t* status) {
  const int n_pix = 6 * C.pixel_face * C.pixel_face;
  const double golden = 0.6180339887498949;
  const double two_pi = 2.0 * kPi;
  const int lane = threadIdx.x & 31;
  const int64_t n_pad = (n_subseg + 31) & ~(int64_t)31;  // warps never straddle node blocks
  const int n_blocks = (C.ring_nodes + kO1RingBlock - 1) / kO1RingBlock;
  const int64_t total = n_pad * n_blocks;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  __shared__ double s_stage[kO1RingThreads / 32][32 * kO1Moments];
  double* stage = s_stage[threadIdx.x >> 5];
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < total; k += stride) {
    const int64_t sub = k % n_pad;
    const int q_begin = (int)(k / n_pad) * kO1RingBlock;
    const int q_end = min(q_begin + kO1RingBlock, C.ring_nodes);
    const bool live = sub < n_subseg;
    double ux = 0, uy = 0, uz = 1, e1x = 1, e1y = 0, e1z = 0, e2x = 0, e2y = 1, e2z = 0;
    double cc = 0, cs = 0, arc2 = 0, sub2 = 0, w0 = 0, w2 = 0, offset = 0;
    O1Subseg P{};
    long long cell = 0;
    if (live) {
      // element of this sub-segment: last i with subseg_offset[i] <= sub
      int64_t lo = 0, hi = E.n_el;
      while (hi - lo > 1) {
        int64_t mid = (lo + hi) >> 1;
        if (subseg_offset[mid] <= sub) lo = mid; else hi = mid;
      }
      const int64_t i = lo;
      const int64_t ia = sub - subseg_offset[i];
      const int64_t n_a = subseg_offset[i + 1] - subseg_offset[i];
      ux = E.direction[3 * i]; uy = E.direction[3 * i + 1]; uz = E.direction[3 * i + 2];
      double hx, hy, hz;
      if (fabs(uz) < 0.9) { hx = 0.0; hy = 0.0; hz = 1.0; } else { hx = 1.0; hy = 0.0; hz = 0.0; }
      e1x = uy * hz - uz * hy; e1y = uz * hx - ux * hz; e1z = ux * hy - uy * hx;
      const double norm = sqrt(e1x * e1x + e1y * e1y + e1z * e1z);
      e1x /= norm; e1y /= norm; e1z /= norm;
      e2x = uy * e1z - uz * e1y; e2y = uz * e1x - ux * e1z; e2z = ux * e1y - uy * e1x;
      cc = E.cone_cos[i];
      cs = sqrt(fmax(1.0 - cc * cc, 0.0));
      const double share = 1.0 / ((double)n_a * C.ring_nodes);
      const double arc = two_pi * cs / C.ring_nodes;
      arc2 = arc * arc / 12.0;
      const double sl = E.length[i] / n_a;
      sub2 = sl * sl / 12.0;
      w0 = E.c0[i] * share;
      w2 = E.c2[i] * share;
      const double ig = (double)i * golden;
      offset = (ig - floor(ig)) * two_pi / C.ring_nodes;
      P = o1_subseg(E, i, ia, n_a);
      const long long cx = min(max((long long)floor((P.px - E.grid_origin[0]) / C.cell_m), 0ll), (long long)E.grid_dims[0] - 1);
      const long long cy = min(max((long long)floor((P.py - E.grid_origin[1]) / C.cell_m), 0ll), (long long)E.grid_dims[1] - 1);
      const long long cz = min(max((long long)floor((P.pz - E.grid_origin[2]) / C.cell_m), 0ll), (long long)E.grid_dims[2] - 1);
      cell = (cx * E.grid_dims[1] + cy) * E.grid_dims[2] + cz;
    }
    const double px = P.px, py = P.py, pz = P.pz, t = P.t;
    for (int q = q_begin; q < q_end; ++q) {
      double sp, cp;
      sincos(offset + two_pi * q / C.ring_nodes, &sp, &cp);
      const double sx = cc * ux + cs * (cp * e1x + sp * e2x);
      const double sy = cc * uy + cs * (cp * e1y + sp * e2y);
      const double sz = cc * uz + cs * (cp * e1z + sp * e2z);
      const long long key = live ? cell * n_pix + o1_pixel(sx, sy, sz, C.pixel_face) : -1ll;
      const unsigned group = __match_any_sync(0xffffffffu, key);
      const bool leader = live && lane == __ffs(group) - 1;
      double* row = nullptr;
      if (leader) {
        bool fresh;
        // slots in key order (keys of one cell are contiguous) so that the
        // compacted pencils come out spatially ordered
        const int64_t slot = o1_insert(keys, capacity, key, rows, kO1Moments, fresh, status, true);
        if (slot >= 0) row = rows + slot * kO1Moments;
      }
      const double tx = -sp * e1x + cp * e2x, ty = -sp * e1y + cp * e2y, tz = -sp * e1z + cp * e2z;
      const double m[kO1Moments] = {
          w0, w2, w0 * px, w0 * py, w0 * pz, w0 * t, w0 * sx, w0 * sy, w0 * sz,
          w0 * (px * px + py * py + pz * pz + sub2), w0 * t * t,
          w0 * (sx * sx + arc2 * tx * tx), w0 * (sy * sy + arc2 * ty * ty),
          w0 * (sz * sz + arc2 * tz * tz), w0 * (sx * sy + arc2 * tx * ty),
          w0 * (sx * sz + arc2 * tx * tz), w0 * (sy * sz + arc2 * ty * tz),
          w0 * (px * px + sub2 * ux * ux), w0 * (py * py + sub2 * uy * uy),
          w0 * (pz * pz + sub2 * uz * uz), w0 * (px * py + sub2 * ux * uy),
          w0 * (px * pz + sub2 * ux * uz), w0 * (py * pz + sub2 * uy * uz)};
      double* mine = stage + lane * kO1Moments;
#pragma unroll
      for (int k = 0; k < kO1Moments; ++k) mine[k] = m[k];
      o1_warp_group_add(stage, kO1Moments, group, leader, row);
    }
  }
}

constexpr int kO1Tile = 4096;          // ring-table slots per compaction CTA
constexpr int kO1FinishThreads = 256;  // kO1Tile / kO1FinishThreads consecutive slots each

LH_DEVICE bool o1_slot_used(const long long* keys, const double* rows, int64_t slot) {
  return keys[slot] != -1ll && rows[slot * kO1Moments] > 0.0;
}

// Exclusive prefix sum of `v` over the CTA (blockDim a multiple of 32, at most
// 1024); `total` receives the CTA's sum.
LH_DEVICE int o1_block_exclusive_scan(int v, int& total) {
  __shared__ int warp_sums[32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, n_warps = blockDim.x >> 5;
  int inclusive = v;
  for (int off = 1; off < 32; off <<= 1) {
    const int up = __shfl_up_sync(0xffffffffu, inclusive, off);
    if (lane >= off) inclusive += up;
  }
  __syncthreads();  // warp_sums may still be read by a previous call
  if (lane == 31) warp_sums[warp] = inclusive;
  __syncthreads();
  if (warp == 0) {
    int w = lane < n_warps ? warp_sums[lane] : 0;
    for (int off = 1; off < 32; off <<= 1) {
      const int up = __shfl_up_sync(0xffffffffu, w, off);
      if (lane >= off) w += up;
    }
    warp_sums[lane] = w;  // inclusive over warps
  }
  __syncthreads();
  total = warp_sums[n_warps - 1];
  return inclusive - v + (warp ? warp_sums[warp - 1] : 0);
}

// The slot of `key` in an ordered-start table, or -1 when absent.
LH_DEVICE int64_t o1_find(const long long* keys, int64_t capacity, long long key) {
  const uint64_t mask = (uint64_t)capacity - 1;
  uint64_t slot = (uint64_t)key & mask;
  for (int64_t probe = 0; probe < capacity; ++probe) {
    const long long k = keys[slot];
    if (k == key) return (int64_t)slot;
    if (k == -1ll) return -1;
    slot = (slot + 1) & mask;
  }
  return -1;
}

// parent_keys (_prompt_screen.py:44-54): the pixel of the nested parent face
// in the same position cell.
LH_DEVICE long long o1_parent_key(long long key, int face, int parent_face) {
  const long long per_cell = 6ll * face * face;
  const long long cell = key / per_cell, pixel = key % per_cell;
  const long long cube = pixel / ((long long)face * face), ij = pixel % ((long long)face * face);
  const long long i = ij / face, j = ij % face, factor = face / parent_face;
  return cell * (6ll * parent_face * parent_face) + (cube * parent_face + i / factor) * parent_face +
         j / factor;
}

// compress_screen's parents (_prompt_screen.py:56-85): every occupied child
// slot adds its moments to its parent pixel's slot (the parents of one cell
// are the sums of its children, as finish_pencils sums them).
__global__ void __launch_bounds__(kO1FinishThreads)
o1_parent_kernel(const long long* keys, const double* rows, int64_t capacity, int face,
                 int parent_face, long long* parent_keys, double* parent_rows,
                 int64_t parent_capacity, int32_t* status) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t slot = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; slot < capacity;
       slot += stride) {
    const long long key = keys[slot];
    if (key == -1ll) continue;
    bool fresh;
    const int64_t ps = o1_insert(parent_keys, parent_capacity,
                                 o1_parent_key(key, face, parent_face), parent_rows, kO1Moments,
                                 fresh, status, true);
    if (ps < 0) continue;
    for (int k = 0; k < kO1Moments; ++k)
      atomicAdd(parent_rows + ps * kO1Moments + k, rows[slot * kO1Moments + k]);
  }
}

// Pencils of a screen table: parents plus children.
__global__ void o1_total_kernel(const int32_t* children, const int32_t* parents, int32_t* total) {
  if (threadIdx.x == 0 && blockIdx.x == 0) *total = *children + *parents;
}

// Used slots per tile of the ring table. Thread t takes slots t, t + 256, ...
// of its tile, so that a warp's key loads are contiguous.
__global__ void __launch_bounds__(kO1FinishThreads)
o1_tile_count_kernel(const long long* keys, const double* rows, int64_t capacity,
                     int32_t* tile_count) {
  constexpr int per = kO1Tile / kO1FinishThreads;
  const int64_t tile0 = blockIdx.x * (int64_t)kO1Tile + threadIdx.x;
  int mine = 0;
#pragma unroll
  for (int j = 0; j < per; ++j) {
    const int64_t slot = tile0 + (int64_t)j * kO1FinishThreads;
    if (slot < capacity && o1_slot_used(keys, rows, slot)) ++mine;
  }
  int total;
  o1_block_exclusive_scan(mine, total);
  if (threadIdx.x == 0) tile_count[blockIdx.x] = total;
}

// Exclusive tile offsets (in place) and the pencil count, in one CTA.
__global__ void __launch_bounds__(1024)
o1_tile_scan_kernel(int32_t* tile, int64_t n_tiles, int32_t* count) {
  int carry = 0;
  for (int64_t base = 0; base < n_tiles; base += blockDim.x) {
    const int64_t i = base + threadIdx.x;
    const int v = i < n_tiles ? tile[i] : 0;
    int total;
    const int before = o1_block_exclusive_scan(v, total);
    if (i < n_tiles) tile[i] = carry + before;
    carry += total;
  }
  if (threadIdx.x == 0) *count = carry;
}

LH_DEVICE void o1_write_pencil(const double* a, lh_order1_pencil_table& Pn, int q);

// finish_pencils (_prompt_numba.py:2247-2354) for slots with a positive weight,
// compacted into the pencil table in slot order: one CTA per tile, each thread
// over kO1Tile / kO1FinishThreads consecutive slots, ranks by a CTA scan plus
// the tile's offset. Slot order follows the keys, so pencils of a cell are
// neighbours in the table.
// Screen tables (the coarse charge screen) take their parents first: parent
// rows [0, n_parents) record their row per slot in `slot_row`; child rows
// follow from `base_count` and look up their parent's row by its key.
__global__ void __launch_bounds__(kO1FinishThreads)
o1_finish_kernel(const long long* keys, int64_t capacity, const double* rows,
                 lh_order1_pencil_table Pn, const int32_t* tile_offset, const int32_t* count,
                 const int32_t* base_count, int32_t* slot_row, const long long* parent_keys,
                 int64_t parent_capacity, const int32_t* parent_row, int face, int parent_face,
                 int32_t* status) {
  constexpr int per = kO1Tile / kO1FinishThreads;  // rounds of 256 consecutive slots
  constexpr int warps = kO1FinishThreads / 32;
  static_assert(per <= 32 && per * warps == 128, "one 32-bit mask per thread, 4 counts per lane");
  __shared__ int before[per * warps];  // used slots ahead of each (round, warp) in the tile
  const int64_t n = *count;
  const int64_t base = base_count ? *base_count : 0;
  if (base + n > Pn.capacity) {  // the caller redoes the stage with a larger table
    if (blockIdx.x == 0 && threadIdx.x == 0)
      atomicOr(reinterpret_cast<unsigned*>(status), LH_STATUS_OVERFLOW);
    return;
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t tile0 = blockIdx.x * (int64_t)kO1Tile + threadIdx.x;
  unsigned used = 0;  // bit j: this thread's slot of round j holds a pencil
#pragma unroll
  for (int j = 0; j < per; ++j) {
    const int64_t slot = tile0 + (int64_t)j * kO1FinishThreads;
    if (slot < capacity && o1_slot_used(keys, rows, slot)) used |= 1u << j;
  }
#pragma unroll
  for (int j = 0; j < per; ++j) {
    const unsigned b = __ballot_sync(0xffffffffu, (used >> j) & 1u);
    if (lane == 0) before[j * warps + warp] = __popc(b);
  }
  __syncthreads();
  if (warp == 0) {  // exclusive scan of the 128 (round, warp) counts in slot order
    int v[4], sum = 0;
    for (int i = 0; i < 4; ++i) {
      v[i] = before[4 * lane + i];
      sum += v[i];
    }
    int inclusive = sum;
    for (int off = 1; off < 32; off <<= 1) {
      const int up = __shfl_up_sync(0xffffffffu, inclusive, off);
      if (lane >= off) inclusive += up;
    }
    int running = inclusive - sum;
    for (int i = 0; i < 4; ++i) {
      before[4 * lane + i] = running;
      running += v[i];
    }
  }
  __syncthreads();
  if (!used) return;
  const unsigned lower = (1u << lane) - 1u;
  for (int j = 0; j < per; ++j) {
    const unsigned b = __ballot_sync(__activemask(), (used >> j) & 1u);
    if (!((used >> j) & 1u)) continue;
    const int64_t slot = tile0 + (int64_t)j * kO1FinishThreads;
    // rank order = slot order: a cell's pencils are neighbours in the table, so
    // that the 32 pencils of a stage-B warp share their groups (about four items
    // per group against one for a random order) and the warp sums them before
    // the atomics
    const int row = (int)(base + tile_offset[blockIdx.x] + before[j * warps + warp] +
                          __popc(b & lower));
    o1_write_pencil(rows + slot * kO1Moments, Pn, row);
    if (slot_row) slot_row[slot] = row;
    if (Pn.parent) {
      int32_t parent = -1;
      if (parent_keys) {
        const int64_t ps = o1_find(parent_keys, parent_capacity,
                                   o1_parent_key(keys[slot], face, parent_face));
        if (ps < 0) atomicOr(reinterpret_cast<unsigned*>(status), LH_STATUS_OVERFLOW);
        else parent = parent_row[ps];
      }
      Pn.parent[row] = parent;
    }
  }
}

LH_DEVICE void o1_write_pencil(const double* a, lh_order1_pencil_table& Pn, int q) {
  {
    const double w = a[0];
    const double mx = a[2] / w, my = a[3] / w, mz = a[4] / w;
    Pn.position[3 * q] = mx; Pn.position[3 * q + 1] = my; Pn.position[3 * q + 2] = mz;
    Pn.time[q] = a[5] / w;
    Pn.w0[q] = w;
    Pn.w2[q] = a[1];
    const double rx = a[6] / w, ry = a[7] / w, rz = a[8] / w;
    const double norm = sqrt(rx * rx + ry * ry + rz * rz);
    const double dx = rx / norm, dy = ry / norm, dz = rz / norm;
    Pn.direction[3 * q] = dx; Pn.direction[3 * q + 1] = dy; Pn.direction[3 * q + 2] = dz;
    const double cxx = a[11] / w - rx * rx, cyy = a[12] / w - ry * ry, czz = a[13] / w - rz * rz;
    const double cxy = a[14] / w - rx * ry, cxz = a[15] / w - rx * rz, cyz = a[16] / w - ry * rz;
    double hx, hy, hz;
    if (fabs(dz) < 0.9) { hx = 0.0; hy = 0.0; hz = 1.0; } else { hx = 1.0; hy = 0.0; hz = 0.0; }
    double e1x = dy * hz - dz * hy, e1y = dz * hx - dx * hz, e1z = dx * hy - dy * hx;
    const double nn = sqrt(e1x * e1x + e1y * e1y + e1z * e1z);
    e1x /= nn; e1y /= nn; e1z /= nn;
    const double e2x = dy * e1z - dz * e1y, e2y = dz * e1x - dx * e1z, e2z = dx * e1y - dy * e1x;
    const double c11 = e1x * (cxx * e1x + cxy * e1y + cxz * e1z) + e1y * (cxy * e1x + cyy * e1y + cyz * e1z) +
                       e1z * (cxz * e1x + cyz * e1y + czz * e1z);
    const double c22 = e2x * (cxx * e2x + cxy * e2y + cxz * e2z) + e2y * (cxy * e2x + cyy * e2y + cyz * e2z) +
                       e2z * (cxz * e2x + cyz * e2y + czz * e2z);
    const double c12 = e1x * (cxx * e2x + cxy * e2y + cxz * e2z) + e1y * (cxy * e2x + cyy * e2y + cyz * e2z) +
                       e1z * (cxz * e2x + cyz * e2y + czz * e2z);
    const double half = 0.5 * (c11 + c22);
    const double disc = sqrt(fmax(0.25 * (c11 - c22) * (c11 - c22) + c12 * c12, 0.0));
    Pn.var_major[q] = fmax(half + disc, 0.0);
    Pn.var_minor[q] = fmax(half - disc, 0.0);
    double sa, ca;
    sincos(0.5 * atan2(2.0 * c12, c11 - c22), &sa, &ca);
    Pn.major[3 * q] = ca * e1x + sa * e2x;
    Pn.major[3 * q + 1] = ca * e1y + sa * e2y;
    Pn.major[3 * q + 2] = ca * e1z + sa * e2z;
    Pn.pos_cov[6 * q] = fmax(a[17] / w - mx * mx, 0.0);
    Pn.pos_cov[6 * q + 1] = fmax(a[18] / w - my * my, 0.0);
    Pn.pos_cov[6 * q + 2] = fmax(a[19] / w - mz * mz, 0.0);
    Pn.pos_cov[6 * q + 3] = a[20] / w - mx * my;
    Pn.pos_cov[6 * q + 4] = a[21] / w - mx * mz;
    Pn.pos_cov[6 * q + 5] = a[22] / w - my * mz;
  }
}

// ------------------------------------------------------------------ stage B

// Node sums of the Gaussian inverse-radius measure shared by
// gauss_inverse_mean_prepared (_prompt_numba.py:115-129) and
// inverse_radius_rule (_prompt_screen.py:101-140), for every lane of `need`
// (arguments u, v, var_u, var_v): the warp evaluates one lane's nodes at a
// time, lane j taking nodes j, j + 32, ..., and a butterfly reduction adds
// them, so a lane that needs the 48-node sum does not run it alone while the
// rest of its warp waits. Each lane of `need` receives s0 = 1 / sqrt(scale),
// scale = 2 (var_u + var_v) + u^2 + v^2 (its sums stay 0 when scale <= 0),
// the sum of the node masses and of mass x the radial second moment. Call
// with the whole warp.
LH_DEVICE void o1_node_sums(unsigned need, double u, double v, double var_u, double var_v,
                            const double* tangent, const double* wsec2, int n, double& s0_out,
                            double& mass_out, double& radial_out) {
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  s0_out = mass_out = radial_out = 0.0;
  while (need) {
    const int src = __ffs(need) - 1;
    need &= need - 1;
    const double bu = __shfl_sync(full, u, src), bv = __shfl_sync(full, v, src);
    const double bvu = __shfl_sync(full, var_u, src), bvv = __shfl_sync(full, var_v, src);
    const double scale = 2.0 * (bvu + bvv) + bu * bu + bv * bv;
    if (scale <= 0.0) continue;  // the same for the whole warp
    const double s0 = 1.0 / sqrt(scale);
    double mass = 0.0, radial = 0.0;
    for (int k = lane; k < n; k += 32) {
      const double t = s0 * tangent[k];
      const double a = 1.0 + 2.0 * t * t * bvu, b = 1.0 + 2.0 * t * t * bvv;
      const double m = wsec2[k] * exp(-t * t * (bu * bu / a + bv * bv / b)) / sqrt(a * b);
      mass += m;
      radial += m * (bvu / a + bvv / b + bu * bu / (a * a) + bv * bv / (b * b));
    }
    for (int off = 16; off; off >>= 1) {
      mass += __shfl_xor_sync(full, mass, off);
      radial += __shfl_xor_sync(full, radial, off);
    }
    if (lane == src) {
      s0_out = s0;
      mass_out = mass;
      radial_out = radial;
    }
  }
}

// gauss_inverse_mean_prepared from its node sums.
LH_DEVICE double o1_gauss_inverse_mean(double u, double v, double var_u, double var_v, double s0,
                                       double mass) {
  if (2.0 * (var_u + var_v) + u * u + v * v <= 0.0) return 1e300;
  return 2.0 / sqrt(kPi) * s0 * mass;
}

// inverse_radius_rule from its node sums: a positive two-node rule for the
// Gaussian measure over the radius (w0, t0, w1, t1).
LH_DEVICE void o1_inverse_radius_rule(double u, double v, double var_u, double var_v, double s0,
                                      double mass, double radial, double& w0, double& t0,
                                      double& w1, double& t1) {
  w0 = t0 = w1 = t1 = 0.0;
  if (2.0 * (var_u + var_v) + u * u + v * v <= 0.0) return;
  const double multiplier = 2.0 / sqrt(kPi) * s0;
  const double inverse = mass * multiplier;
  radial *= multiplier;
  if (inverse <= 0.0) return;
  const double mean = 1.0 / inverse, second = radial / inverse;
  const double variance = second - mean * mean;
  if (variance <= 0.0) {
    w0 = inverse; t0 = mean; t1 = mean;
    return;
  }
  const double third = (u * u + v * v + var_u + var_v) / inverse;
  const double other = (third - 2.0 * mean * second + mean * mean * mean) / variance;
  const double disc = sqrt((mean - other) * (mean - other) + 4.0 * variance);
  const double low = 0.5 * (mean + other - disc), high = 0.5 * (mean + other + disc);
  const double low_weight = inverse * (high - mean) / (high - low);
  w0 = low_weight; t0 = low; w1 = inverse - low_weight; t1 = high;
}

// The coarse screen's refinement test (_prompt_screen.py:233-240): the OM
// looks into pencil x's angular extent (forward, theta^2 < s^2 extent^2).
LH_DEVICE bool o1_refined(const lh_order1_config& C, const lh_order1_pencil_table& Pn, int x,
                          double rx, double ry, double rz) {
  const double dx = rx - Pn.position[3 * x], dy = ry - Pn.position[3 * x + 1],
               dz = rz - Pn.position[3 * x + 2];
  const double r = sqrt(dx * dx + dy * dy + dz * dz);
  const double hx = dx / r, hy = dy / r, hz = dz / r;
  const double sx = Pn.direction[3 * x], sy = Pn.direction[3 * x + 1], sz = Pn.direction[3 * x + 2];
  const double cosine = hx * sx + hy * sy + hz * sz;
  const double qx = hx - cosine * sx, qy = hy - cosine * sy, qz = hz - cosine * sz;
  const double theta = atan2(sqrt(qx * qx + qy * qy + qz * qz), cosine);
  const double* cov = Pn.pos_cov + 6 * x;
  const double extent2 = Pn.var_major[x] + (cov[0] + cov[1] + cov[2]) / (r * r);
  const double sf = C.smoothing_factor;
  return theta < 0.5 * kPi && theta * theta < sf * sf * extent2;
}

constexpr int kO1GroupOms = 8;       // work OMs per warp chunk of the group stage
constexpr int kO1PencilFields = 20;  // float64 fields of a pencil read by the group stage

struct O1GroupShared {
  double tangent[kO1MaxGauss], wsec2[kO1MaxGauss];
  double coef[kO1MaxMono];
  int ipow[kO1MaxMono], jpow[kO1MaxMono];
};

// One thread per (work OM, pencil): _grouped_pencils_order1_block's pencil
// loop (_prompt_numba.py:1827-1921) with the generic moment layout. kScreen
// (kScreen): the coarse screen's instance; the fine instance carries none of
// the screen's code (a smaller loop for the instruction cache).
template <bool kScreen>
__global__ void __launch_bounds__(256, 2)
o1_group_kernel(const lh_order1_config C, const lh_order1_pencil_table Pn,
                                int32_t n_pencils_bound, const int32_t* n_pencils_device,
                                const int32_t* work, int32_t n_work,
                                const double* origins, long long* gkeys, double* grows,
                                int32_t* gcount, int32_t* status, unsigned long long* units) {
  __shared__ O1GroupShared S;
  for (int k = threadIdx.x; k < C.n_gauss; k += blockDim.x) {
    const double t = tan(C.gauss_tau[k]);
    S.tangent[k] = t;
    S.wsec2[k] = C.gauss_w[k] * (1.0 + t * t);
  }
  for (int k = threadIdx.x; k < C.n_mono; k += blockDim.x) {
    S.coef[k] = C.coef[k];
    S.ipow[k] = C.ipow[k];
    S.jpow[k] = C.jpow[k];
  }
  __syncthreads();
  const int n_values = 2 * C.n_mono + 6;
  const double log_theta_ratio = log(1.0 + C.theta_ratio);
  const int theta_bins = C.theta_bins;
  const int64_t cap = C.group_capacity;
  // the pencil count is read on the device when given (no host round trip)
  const int32_t n_pencils =
      n_pencils_device ? min(*n_pencils_device, n_pencils_bound) : n_pencils_bound;
  const int64_t total = (int64_t)n_work * n_pencils;
  if (units && blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(units, (unsigned long long)total);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  // [warp][32][n_values] group staging, then [warp][field][32] pencil fields
  extern __shared__ double o1g_stage[];
  double* stage = o1g_stage + warp * 32 * n_values;
  double* pen = o1g_stage + (blockDim.x >> 5) * 32 * n_values + warp * 32 * kO1PencilFields + lane;
  // A warp takes 32 consecutive pencils (neighbours in space) and kO1GroupOms
  // consecutive work OMs: each lane reads its pencil once (into shared memory)
  // and evaluates it against every OM of the chunk in turn. Chunks take the OM
  // blocks fastest and the pencil blocks in a fixed permutation
  // ((q (2^31 - 1)) mod blocks, 2^31 - 1 prime), so that the warps running at
  // once work on different OMs and distant parts of the shower rather than
  // competing for the same group rows. Lanes past the last pencil compute on
  // pencil 0 and take no part in any group.
  const int64_t pblocks = ((int64_t)n_pencils + 31) / 32;
  const int64_t oblocks = (n_work + kO1GroupOms - 1) / kO1GroupOms;
  const int64_t chunks = pblocks * oblocks;
  const int64_t warps_total = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t chunk = blockIdx.x * (int64_t)(blockDim.x >> 5) + warp; chunk < chunks;
       chunk += warps_total) {
    const int64_t p_raw = (((chunk / oblocks) * 2147483647ll) % pblocks) * 32 + lane;
    const int w_first = (int)(chunk % oblocks) * kO1GroupOms;
    const bool p_ok = p_raw < n_pencils;
    const int p = p_ok ? (int)p_raw : 0;
    pen[0] = Pn.position[3 * p]; pen[32] = Pn.position[3 * p + 1]; pen[64] = Pn.position[3 * p + 2];
    pen[96] = Pn.time[p];
    pen[128] = Pn.direction[3 * p]; pen[160] = Pn.direction[3 * p + 1];
    pen[192] = Pn.direction[3 * p + 2];
    pen[224] = Pn.major[3 * p]; pen[256] = Pn.major[3 * p + 1]; pen[288] = Pn.major[3 * p + 2];
    pen[320] = Pn.var_major[p]; pen[352] = Pn.var_minor[p];
    for (int f = 0; f < 6; ++f) pen[(12 + f) * 32] = Pn.pos_cov[6 * p + f];
    pen[576] = Pn.w0[p]; pen[608] = Pn.w2[p];
    const int parent = kScreen ? Pn.parent[p] : -1;
    for (int k = 0; k < kO1GroupOms; ++k) {
    const int w = w_first + k;
    if (w >= n_work) break;  // the same for the whole warp
    bool live = p_ok;
    const int d = work[w];
    const double rx = C.om_pos[3 * d], ry = C.om_pos[3 * d + 1], rz = C.om_pos[3 * d + 2];
    const double nx = C.om_look[3 * d], ny = C.om_look[3 * d + 1], nz = C.om_look[3 * d + 2];
    // _prepare_receiver_geometry (_prompt_numba.py:1590-1612)
    const double dx = rx - pen[0], dy = ry - pen[32], dz = rz - pen[64];
    const double r = sqrt(dx * dx + dy * dy + dz * dz);
    const double hx = dx / r, hy = dy / r, hz = dz / r;
    // the screen's charge batches ignore emission time (_prompt_screen.py:220-229)
    const double t_emit = kScreen ? 0.0 : pen[96] - origins[d];
    const double tau = kScreen ? 0.0 : t_emit + r / C.speed_ref;
    const double log_r = log(r);
    const long long key0 = (long long)floor(log_r / C.log_r_step) + (1ll << 20);
    const long long key1 =
        min(max((long long)floor(tau / C.tau_step) + (1ll << 20), 0ll), (1ll << 21) - 1);
    const long long base = kScreen ? key0 * 2 * theta_bins : ((key1 << 21) + key0) * 2 * theta_bins;
    if (kScreen && live) {  // a parent unless the OM looks into it, else its children
      // rows of a table whose stage A overflowed are not written (the caller
      // redoes it): an index outside the table is never followed
      if (parent >= n_pencils || parent < -1) live = false;
      else live = parent < 0 ? !o1_refined(C, Pn, p, rx, ry, rz)
                             : o1_refined(C, Pn, parent, rx, ry, rz);
    }
    // children stand in for their parent only where the OM looks into it, so
    // most screen warps over children have nothing to add
    if (kScreen && !__any_sync(0xffffffffu, live)) continue;
    // _pencil_frame_from_ray_cached_look (_prompt_numba.py:594-606)
    const double sx = pen[128], sy = pen[160], sz = pen[192];
    const double c1 = sx * nx + sy * ny + sz * nz;
    const double cosine = hx * sx + hy * sy + hz * sz;
    const double qx = hx - cosine * sx, qy = hy - cosine * sy, qz = hz - cosine * sz;
    const double sine = sqrt(qx * qx + qy * qy + qz * qz);
    const double c3 = sine > 1e-300 ? (qx * nx + qy * ny + qz * nz) / sine : 0.0;
    double theta = atan2(sine, cosine);
    const bool backward = theta > 0.5 * kPi;
    double weight = 0.0, weight2 = 0.0, theta2 = theta;
    bool averaged = false;
    const double ax = pen[224], ay = pen[256], az = pen[288];
    const double cov[6] = {pen[384], pen[416], pen[448], pen[480], pen[512], pen[544]};
    // _prepare_pencil_shape (_prompt_numba.py:1347-1370)
    const double bx = sy * az - sz * ay, by = sz * ax - sx * az, bz = sx * ay - sy * ax;
    const double trace = cov[0] + cov[1] + cov[2];
    const double sf = C.smoothing_factor;
    // How this lane's weight is formed: 0 done; 1 the screen's two-node radial
    // rule; 2 the Gauss inverse mean; 3 the far-field expansion. Modes 1 and 2
    // need a 48-node sum, which the whole warp evaluates for each such lane.
    int mode = 0;
    bool far = true;
    double m11 = 0.0, m22 = 0.0, m12 = 0.0, mu1 = 0.0, mu2 = 0.0, extent = 0.0;
    double u_ = 0.0, v_ = 0.0, r_extent = 0.0;
    double arg_u = 0.0, arg_v = 0.0, arg_var_u = 0.0, arg_var_v = 0.0;  // of the node sums
    if (backward) {
      weight = 1.0 / r;
    } else {
      const double bound = pen[320] + pen[352] + trace / (r * r);
      if (sine > 1e-300 && bound < 1e-4 * sine * sine) {
        weight = (1.0 / sine) / r;
      } else {
        // _pencil_shape_factor_from_ray (_prompt_numba.py:1389-1436)
        const double caa = ax * (cov[0] * ax + cov[3] * ay + cov[4] * az) +
                           ay * (cov[3] * ax + cov[1] * ay + cov[5] * az) +
                           az * (cov[4] * ax + cov[5] * ay + cov[2] * az);
        const double cbb = bx * (cov[0] * bx + cov[3] * by + cov[4] * bz) +
                           by * (cov[3] * bx + cov[1] * by + cov[5] * bz) +
                           bz * (cov[4] * bx + cov[5] * by + cov[2] * bz);
        const double cab = ax * (cov[0] * bx + cov[3] * by + cov[4] * bz) +
                           ay * (cov[3] * bx + cov[1] * by + cov[5] * bz) +
                           az * (cov[4] * bx + cov[5] * by + cov[2] * bz);
        const double inv_r2 = 1.0 / (r * r);
        m11 = pen[320] + caa * inv_r2;
        m22 = pen[352] + cbb * inv_r2;
        m12 = cab * inv_r2;
        const double upper = fmax(m11, m22) + fabs(m12);
        far = fmax(fmax(fabs(m11), fabs(m22)), fabs(m12)) < 1e150 &&
              theta * theta > sf * sf * fmax(upper, 0.0) * (1.0 + 1e-12);
        if (!far) {
          const double half_tr = 0.5 * (m11 + m22);
          const double disc = sqrt(fmax(0.25 * (m11 - m22) * (m11 - m22) + m12 * m12, 0.0));
          mu1 = half_tr + disc;
          mu2 = fmax(half_tr - disc, 1e-16 * mu1 + 1e-300);
          extent = sqrt(fmax(mu1, 0.0));
        }
        u_ = hx * ax + hy * ay + hz * az;
        v_ = hx * bx + hy * by + hz * bz;
        mode = (!far && extent > 0.0 && theta < sf * extent) ? 2 : 3;
        if (kScreen) {
          // pencil_radial_rule (_prompt_screen.py:143-169): two radial nodes where the
          // OM lies within the pencil's angular smoothing extent
          const double half_tr = 0.5 * (m11 + m22);
          const double disc = sqrt(fmax(0.25 * (m11 - m22) * (m11 - m22) + m12 * m12, 0.0));
          const double r_mu1 = half_tr + disc;
          const double r_mu2 = fmax(half_tr - disc, 1e-16 * r_mu1 + 1e-300);
          r_extent = sqrt(fmax(r_mu1, 0.0));
          if (r_extent > 0.0 && theta < sf * r_extent) {
            const double st = sine > 0.0 ? theta / sine : 1.0;
            const double uu = u_ * st, vv = v_ * st;
            double sa, ca;
            sincos(0.5 * atan2(2.0 * m12, m11 - m22), &sa, &ca);
            arg_u = ca * uu + sa * vv;
            arg_v = -sa * uu + ca * vv;
            arg_var_u = r_mu1;
            arg_var_v = r_mu2;
            mode = 1;
          }
        }
      }
    }
    if (!live) mode = 0;  // nothing of this lane is added
    const unsigned full = 0xffffffffu;
    double s0n, mass, radial;
    const unsigned need_rule = __ballot_sync(full, mode == 1);
    if (need_rule) {
      o1_node_sums(need_rule, arg_u, arg_v, arg_var_u, arg_var_v, S.tangent, S.wsec2, C.n_gauss,
                   s0n, mass, radial);
      if (mode == 1) {
        double w0r, t0r, w1r, t1r;
        o1_inverse_radius_rule(arg_u, arg_v, arg_var_u, arg_var_v, s0n, mass, radial, w0r, t0r,
                               w1r, t1r);
        if (t0r > 0.0 && t1r < 0.5 * kPi && w0r > 0.0 && w1r >= 0.0) {
          averaged = theta < r_extent;
          weight = (w0r * t0r / sin(t0r)) / r;
          weight2 = (w1r * t1r / sin(t1r)) / r;
          theta = t0r;
          theta2 = t1r;
          mode = 0;
        } else {
          mode = (!far && extent > 0.0 && theta < sf * extent) ? 2 : 3;
        }
      }
    }
    if (mode == 2) {
      double sa, ca;
      sincos(0.5 * atan2(2.0 * m12, m11 - m22), &sa, &ca);
      arg_u = ca * u_ + sa * v_;
      arg_v = -sa * u_ + ca * v_;
      arg_var_u = mu1;
      arg_var_v = mu2;
    }
    const unsigned need_mean = __ballot_sync(full, mode == 2);
    if (need_mean) {
      o1_node_sums(need_mean, arg_u, arg_v, arg_var_u, arg_var_v, S.tangent, S.wsec2, C.n_gauss,
                   s0n, mass, radial);
      if (mode == 2) {
        const double mean = o1_gauss_inverse_mean(arg_u, arg_v, arg_var_u, arg_var_v, s0n, mass);
        const double factor = mean * (sine > 1e-300 ? theta / sine : 1.0);
        averaged = theta < extent;
        theta = factor > 1.0 ? asin(fmin(1.0, 1.0 / factor)) : theta;
        weight = factor / r;
      }
    }
    if (mode == 3) {
      if (sine <= 1e-300) live = false;
      const double d2 = u_ * u_ + v_ * v_;
      double factor = 1.0 / sine;
      if (d2 > 0.0) {
        const double qf = m11 * u_ * u_ + 2.0 * m12 * u_ * v_ + m22 * v_ * v_;
        factor *= 1.0 + 0.5 * (3.0 * qf / d2 - (m11 + m22)) / d2;
      }
      weight = factor / r;
    }
    // _fill_moments_averaged_pair (_prompt_numba.py:1260-1277): the angular powers
    double cpw[5], spw[5];
    cpw[0] = 1.0;
    spw[0] = 1.0;
    const double perp2 = fmax(1.0 - c1 * c1, 0.0);
    for (int q = 1; q <= C.max_power; ++q) {
      cpw[q] = cpw[q - 1] * c1;
      if (averaged) spw[q] = (q & 1) ? 0.0 : spw[q - 2] * perp2 * (q - 1.0) / q;
      else spw[q] = spw[q - 1] * c3;
    }
    const int nm = C.n_mono;
    // one group entry per radial node: the screen's two-node rule adds a second
    // (_prompt_screen.py:281-336); every lane of the warp takes both rounds
    const int nodes = kScreen ? 2 : 1;
    for (int node = 0; node < nodes; ++node) {
      const bool live_n = live && (node == 0 || weight2 > 0.0);
      const double wn = node == 0 ? weight : weight2;
      const double th = node == 0 ? theta : theta2;
      // theta index (scalar_theta_index, _prompt_numba.py:1628-1631)
      int i_theta;
      if (!(th >= C.theta_lo)) i_theta = 0;
      else i_theta = min(1 + (int)(log(th / C.theta_lo) / log_theta_ratio), theta_bins - 1);
      const long long key = base + (backward ? theta_bins : 0) + i_theta;
      // lanes with the same (OM, group key) sum their moments in registers; the
      // group's lowest lane inserts the key and adds the sums
      const unsigned group = __match_any_sync(0xffffffffu, live_n ? key : -1ll) &
                             __match_any_sync(0xffffffffu, live_n ? w : -1);
      const bool leader = live_n && lane == __ffs(group) - 1;
      double* row = nullptr;
      if (leader) {
        bool fresh;
        long long* keys = gkeys + (int64_t)w * cap;
        const int64_t slot = o1_insert(keys, cap, key, grows + (int64_t)w * cap * kO1MaxValues,
                                       kO1MaxValues, fresh, status);
        if (slot >= 0) {
          if (fresh) atomicAdd(gcount + w, 1);
          row = grows + ((int64_t)w * cap + slot) * kO1MaxValues;
        }
      }
      const double field0 = wn * pen[576], field2 = wn * pen[608];
      double omega = 0.0;
      double* mine = stage + lane * n_values;
      for (int m = 0; m < nm; ++m) {
        const double basis = cpw[S.ipow[m]] * spw[S.jpow[m]];
        const double v0 = field0 * basis;
        if (m == 0) omega = fabs(v0);
        mine[m] = v0;
        mine[nm + m] = field2 * basis;
      }
      mine[2 * nm] = omega;
      mine[2 * nm + 1] = omega * th;
      mine[2 * nm + 2] = omega * r;
      mine[2 * nm + 3] = omega * t_emit;
      mine[2 * nm + 4] = omega * tau;
      mine[2 * nm + 5] = omega * tau * tau;
      o1_warp_group_add(stage, n_values, group, leader, row);
    }
    }  // OMs of the chunk
  }
}

// One CTA per work OM: sort the OM's group keys and list its (tau, r) batches.
__global__ void __launch_bounds__(1024)
o1_batches_kernel(const lh_order1_config C, int32_t n_work, const long long* gkeys,
                  int32_t* sorted_slots, int32_t* batch_list, int32_t* batch_total,
                  unsigned long long* sort_keys, int32_t* sort_slots, int32_t* status) {
  // Tables up to kO1SmemSort slots sort (key << 14 | slot) in shared memory;
  // larger ones (steps whose pencils mix times, e.g. delayed light) sort keys
  // and slots side by side in the workspace.
  extern __shared__ __align__(16) unsigned char o1b_smem[];
  __shared__ int n_used;
  const int w = blockIdx.x;
  const int64_t cap = C.group_capacity;
  const bool packed = cap <= kO1SmemSort;
  unsigned long long* v =
      packed ? reinterpret_cast<unsigned long long*>(o1b_smem) : sort_keys + (int64_t)w * cap;
  int32_t* vs = packed ? nullptr : sort_slots + (int64_t)w * cap;
  const long long* keys = gkeys + (int64_t)w * cap;
  if (threadIdx.x == 0) n_used = 0;
  __syncthreads();
  for (int64_t slot = threadIdx.x; slot < cap; slot += blockDim.x) {
    const long long key = keys[slot];
    if (key == -1ll) continue;
    const int k = atomicAdd(&n_used, 1);
    if (packed) {
      v[k] = ((unsigned long long)key << 14) | (unsigned long long)slot;
    } else {
      v[k] = (unsigned long long)key;
      vs[k] = (int32_t)slot;
    }
  }
  __syncthreads();
  const int used = n_used;
  int n = 1;
  while (n < used) n <<= 1;
  for (int k = used + threadIdx.x; k < n; k += blockDim.x) {
    v[k] = ~0ull;
    if (!packed) vs[k] = -1;
  }
  __syncthreads();
  // bitonic sort, ascending (shared or, for large tables, global memory: the
  // barrier makes the block's global writes visible to the block)
  for (int size = 2; size <= n; size <<= 1) {
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      for (int k = threadIdx.x; k < n; k += blockDim.x) {
        const int partner = k ^ stride;
        if (partner > k) {
          const bool up = (k & size) == 0;
          const unsigned long long a = v[k], b = v[partner];
          if ((a > b) == up) {
            v[k] = b;
            v[partner] = a;
            if (!packed) {
              const int32_t t = vs[k];
              vs[k] = vs[partner];
              vs[partner] = t;
            }
          }
        }
      }
      __syncthreads();
    }
  }
  int32_t* out = sorted_slots + (int64_t)w * cap;
  const long long tb = C.theta_bins;
  auto key_of = [&](int k) { return packed ? (long long)(v[k] >> 14) : (long long)v[k]; };
  for (int k = threadIdx.x; k < used; k += blockDim.x) {
    out[k] = packed ? (int32_t)(v[k] & 0x3fffull) : vs[k];
    const long long bk = key_of(k) / tb;
    if (k == 0 || key_of(k - 1) / tb != bk) {
      int stop = k + 1;
      while (stop < used && key_of(stop) / tb == bk) ++stop;
      const int b = atomicAdd(batch_total, 1);
      batch_list[3 * b] = w;
      batch_list[3 * b + 1] = k;
      batch_list[3 * b + 2] = stop;
    }
  }
  (void)status;
}

// _ifuncs (_prompt_numba.py:139-154): I_k(z) = int_0^1 x^k e^{z x} dx, k = 0, 1, 2
LH_DEVICE void o1_ifuncs(double z, double ez, double& i0, double& i1, double& i2) {
  if (fabs(z) < 1.0) {
    // Taylor coefficients 1 / (n! (n + j + 1)), Horner from n = 23
    double f = 1.0;  // 1/n!
    double c0[24], c1[24], c2[24];
    for (int n = 0; n < 24; ++n) {
      if (n > 0) f /= n;
      c0[n] = f / (n + 1.0);
      c1[n] = f / (n + 2.0);
      c2[n] = f / (n + 3.0);
    }
    i0 = c0[23]; i1 = c1[23]; i2 = c2[23];
    for (int n = 22; n >= 0; --n) {
      i0 = i0 * z + c0[n];
      i1 = i1 * z + c1[n];
      i2 = i2 * z + c2[n];
    }
    return;
  }
  i0 = (ez - 1.0) / z;
  i1 = (ez * (z - 1.0) + 1.0) / (z * z);
  i2 = (ez * (z * z - 2.0 * z + 2.0) - 2.0) / (z * z * z);
}

// _quad_integral (_prompt_numba.py:158-163)
LH_DEVICE double o1_quad(double e_start, double alpha, double beta, double gamma, double width,
                         double kappa, double e_end) {
  const double z = kappa * width;
  const double ez = e_start > 0.0 ? e_end / e_start : exp(z);
  double i0, i1, i2;
  o1_ifuncs(z, ez, i0, i1, i2);
  return e_start * width * (alpha * i0 + width * (beta * i1 + width * gamma * i2));
}

// _find_bin (_prompt_numba.py:167-182)
LH_DEVICE int o1_find_bin(const double* edges, int nb, double t) {
  if (t < edges[0]) return -1;
  if (t >= edges[nb]) return nb;
  int low = 0, high = nb;
  while (high - low > 1) {
    const int middle = (low + high) / 2;
    if (t < edges[middle]) high = middle; else low = middle;
  }
  return low;
}

// _deposit_panel (_prompt_numba.py:186-254) into the OM's accumulators
// pre[3] and acc[nb][4] of one band.
LH_DEVICE void o1_deposit_panel(double t_a, double t_b, double e_a, double e_b, double alpha,
                                double beta, double gamma, double kappa, const double* edges,
                                const double* eedge, int nb, double* pre, double* acc,
                                int direct_bins) {
  const double lo = t_a > edges[0] ? t_a : edges[0];
  const double hi = t_b < edges[nb] ? t_b : edges[nb];
  if (hi <= lo) return;
  const int k_lo = o1_find_bin(edges, nb, lo);
  int k_hi = o1_find_bin(edges, nb, hi);
  if (k_hi >= nb || (k_hi > k_lo && hi <= edges[k_hi])) k_hi -= 1;
  if (k_hi - k_lo + 1 <= direct_bins) {
    for (int k = k_lo; k <= k_hi; ++k) {
      const double s_lo = lo > edges[k] ? lo : edges[k];
      const double s_hi = hi < edges[k + 1] ? hi : edges[k + 1];
      if (s_hi <= s_lo) continue;
      double e_lo = s_lo == t_a ? e_a : eedge[k];
      if (s_lo != t_a && s_lo != edges[k]) e_lo = exp(kappa * s_lo);
      double e_hi = s_hi == t_b ? e_b : eedge[k + 1];
      if (s_hi != t_b && s_hi != edges[k + 1]) e_hi = exp(kappa * s_hi);
      const double shift = s_lo - t_a;
      const double a_loc = alpha + shift * (beta + shift * gamma);
      const double b_loc = beta + 2.0 * gamma * shift;
      atomicAdd(acc + 4 * k + 3, o1_quad(e_lo, a_loc, b_loc, gamma, s_hi - s_lo, kappa, e_hi));
    }
    return;
  }
  const double big_a = alpha - t_a * (beta - gamma * t_a);
  const double big_b = beta - 2.0 * gamma * t_a;
  const double big_c = gamma;
  if (t_a < edges[0]) {
    atomicAdd(pre + 0, big_a);
    atomicAdd(pre + 1, big_b);
    atomicAdd(pre + 2, big_c);
  } else {
    const int k = k_lo;
    atomicAdd(acc + 4 * k + 0, big_a);
    atomicAdd(acc + 4 * k + 1, big_b);
    atomicAdd(acc + 4 * k + 2, big_c);
    atomicAdd(acc + 4 * k + 3, o1_quad(e_a, alpha, beta, gamma, edges[k + 1] - t_a, kappa, eedge[k + 1]));
  }
  if (t_b < edges[nb]) {
    const int k = o1_find_bin(edges, nb, t_b);
    atomicAdd(acc + 4 * k + 0, -big_a);
    atomicAdd(acc + 4 * k + 1, -big_b);
    atomicAdd(acc + 4 * k + 2, -big_c);
    const double shift = t_b - t_a;
    const double a_loc = alpha + shift * (beta + shift * gamma);
    const double b_loc = beta + 2.0 * gamma * shift;
    atomicAdd(acc + 4 * k + 3,
              -o1_quad(e_b, a_loc, b_loc, gamma, edges[k + 1] - t_b, kappa, eedge[k + 1]));
  }
}

struct O1BandDeposit {
  double v, kappa, spread, t_base, e_emit, w0, w2, h_front, total;
  int last, pairs, panels;
  bool outside;
};

// NODES: the path-grid nodes a CTA holds in shared memory (kO1SmallNodes for
// the common short grids, kO1MaxNodes for the rest).
constexpr int kO1SmallNodes = 512;

template <int NODES>
struct O1BatchShared {
  double s[NODES];
  double g0[NODES];
  double g2[NODES];
  double mom[kO1MaxValues * 128];  // moments of the batch's theta groups (<= 128)
  double sin_q[128], cos_q[128];   // per group: sin, cos of its mean angle (0, 0: empty)
  double coef[kO1MaxMono];
  int ipow[kO1MaxMono], jpow[kO1MaxMono];
  double red[kO1BatchThreads / 32];
  double stats[8];
  O1BandDeposit band[kO1MaxBands];
  int n, last;
};

// Persistent CTAs over the batch list: _grouped_pencils_order1_block's batch
// loop (_prompt_numba.py:1934-1993) with _batch_grid, _batch_add_moments and
// _batch_deposit (_prompt_numba.py:258-551).
// The small-grid instance (NODES < kO1MaxNodes, 42 KB of shared memory, five
// CTAs per SM) takes the whole list and hands each batch whose path grid needs
// more than NODES nodes to `deferred`; the full-size instance (two CTAs per
// SM) then takes only those.
template <int NODES>
__global__ void __launch_bounds__(kO1BatchThreads)
o1_batch_kernel(const lh_order1_config C, const int32_t* work, const long long* gkeys,
                const double* grows, const int32_t* sorted_slots, const int32_t* batch_list,
                const int32_t* batch_total, int32_t* deferred, int32_t* n_deferred,
                double* accum, int32_t* status) {
  constexpr bool kSmall = NODES < kO1MaxNodes;
  extern __shared__ __align__(16) unsigned char o1_smem[];
  O1BatchShared<NODES>& S = *reinterpret_cast<O1BatchShared<NODES>*>(o1_smem);
  const int tid = threadIdx.x;
  const int nm = C.n_mono;
  const int nv = 2 * nm + 6;
  const int nb = C.n_edges - 1;
  const int NL = C.n_bands;
  const int64_t cap = C.group_capacity;
  for (int k = tid; k < nm; k += blockDim.x) {
    S.coef[k] = C.coef[k];
    S.ipow[k] = C.ipow[k];
    S.jpow[k] = C.jpow[k];
  }
  double mut_min = C.mut[0], speed_max = C.speed[0];
  for (int l = 1; l < NL; ++l) {
    mut_min = fmin(mut_min, C.mut[l]);
    speed_max = fmax(speed_max, C.speed[l]);
  }
  const double g = C.g;
  const double y_g = g != 0.0 ? (1.0 - fabs(g)) / (1.0 + fabs(g)) : 1.0;
  const int total = kSmall ? *batch_total : *n_deferred;
  const int64_t per_om = (int64_t)NL * (3 + 4 * nb + 1);
  for (int i = blockIdx.x; i < total; i += gridDim.x) {
    const int b = kSmall ? i : deferred[i];
    __syncthreads();
    const int w = batch_list[3 * b], start = batch_list[3 * b + 1], stop = batch_list[3 * b + 2];
    const int count = stop - start;
    const int32_t* slots = sorted_slots + (int64_t)w * cap + start;
    const double* rows = grows + (int64_t)w * cap * kO1MaxValues;
    if (count > 128) {
      if (tid == 0) atomicOr(reinterpret_cast<unsigned*>(status), LH_STATUS_OVERFLOW);
      continue;
    }
    for (int k = tid; k < count * nv; k += blockDim.x) {
      const int q = k / nv, c = k - q * nv;
      S.mom[q * kO1MaxValues + c] = rows[(int64_t)slots[q] * kO1MaxValues + c];
    }
    const long long key0 = gkeys[(int64_t)w * cap + slots[0]];
    const bool backward = ((key0 / C.theta_bins) & 1) == 1;
    __syncthreads();
    if (tid == 0) {
      double omega_sum = 0, r_sum = 0, t_sum = 0, tau_sum = 0, tau2_sum = 0, theta_small = kPi;
      for (int q = 0; q < count; ++q) {
        const double* row = S.mom + q * kO1MaxValues;
        const double omega = row[2 * nm];
        if (omega > 0.0) {
          omega_sum += omega;
          r_sum += row[2 * nm + 2];
          t_sum += row[2 * nm + 3];
          tau_sum += row[2 * nm + 4];
          tau2_sum += row[2 * nm + 5];
          theta_small = fmin(theta_small, row[2 * nm + 1] / omega);
        }
      }
      S.n = 0;
      if (omega_sum > 0.0) {
        const double r_b = r_sum / omega_sum;
        const double t_b = t_sum / omega_sum;
        const double tau_mean = tau_sum / omega_sum;
        const double tau_var = fmax(tau2_sum / omega_sum - tau_mean * tau_mean, 0.0);
        theta_small = fmax(theta_small, 1e-9);
        double sigma;
        if (backward) {
          sigma = fmax(0.5 * r_b * sin(theta_small) * y_g, 0.25 * r_b * (1.0 - cos(theta_small)));
        } else {
          // _batch_sigma (_prompt_numba.py:290-292)
          sigma = fmax(0.5 * r_b * sin(theta_small) * fmax(y_g, 0.5 * tan(0.5 * theta_small)),
                       1e-9 * r_b);
        }
        // _batch_grid (_prompt_numba.py:258-286): node counts
        const double ext_end = C.tail_exponent / mut_min;
        // the screen's grids run to the tail without a window edge
        // (_prompt_screen.py:413: edge_end = inf)
        double ext_win = C.screen ? ext_end : speed_max * (C.edges[nb] - t_b) - r_b;
        ext_win = fmin(fmax(ext_win, 0.0), ext_end);
        const double u_end = asinh(ext_end / sigma), u_win = asinh(ext_win / sigma);
        if (!(u_win >= 0.0) || !(u_end >= u_win) || !(u_end < 1e6)) {
          atomicOr(reinterpret_cast<unsigned*>(status), LH_STATUS_OVERFLOW);
          S.n = 0;
          goto stats_done;
        }
        long long n_in = u_win > 0.0 ? (long long)ceil(u_win / C.path_step) : 0;
        long long n_out = u_end > u_win ? (long long)ceil((u_end - u_win) / C.path_step_tail) : 0;
        const int capacity = C.max_path_nodes;
        if (n_in + n_out + 1 > capacity) {
          const double scale = (capacity - 1.0) / (double)(n_in + n_out);
          n_in = (long long)(n_in * scale);
          n_out = capacity - 1 - n_in;
        }
        S.n = (int)(n_in + n_out + 1);
        if (S.n > NODES) {  // a long path grid: the full-size instance takes this batch
          deferred[atomicAdd(n_deferred, 1)] = b;
          S.n = 0;
          goto stats_done;
        }
        S.stats[0] = r_b; S.stats[1] = t_b; S.stats[2] = sqrt(12.0 * tau_var);
        S.stats[3] = sigma; S.stats[4] = u_win; S.stats[5] = u_end;
        S.stats[6] = (double)n_in; S.stats[7] = (double)n_out;
      }
    }
  stats_done:
    __syncthreads();
    const int n = S.n;
    if (n == 0) continue;
    const double r_b = S.stats[0], t_b = S.stats[1], front_extra = S.stats[2];
    const double sigma = S.stats[3], u_win = S.stats[4], u_end = S.stats[5];
    const int n_in = (int)S.stats[6], n_out = (int)S.stats[7];
    // the groups' mean angles, once per batch (the profile loop below reads them
    // for every path node)
    for (int q = tid; q < count; q += blockDim.x) {
      const double* row = S.mom + q * kO1MaxValues;
      const double omega = row[2 * nm];
      double sin_t = 0.0, cos_t = 0.0;
      if (omega > 0.0) sincos(fmax(row[2 * nm + 1] / omega, 1e-9), &sin_t, &cos_t);
      S.sin_q[q] = sin_t;
      S.cos_q[q] = cos_t;
    }
    for (int k = tid; k < n; k += blockDim.x) {
      double s;
      if (k == 0) s = r_b;
      else if (k <= n_in) s = r_b + sigma * sinh(u_win * k / n_in);
      else s = r_b + sigma * sinh(u_win + (u_end - u_win) * (k - n_in) / n_out);
      S.s[k] = s;
    }
    __syncthreads();
    // profile: _batch_add_moments (_prompt_numba.py:394-447), generic monomials
    // With few path nodes (typically ~33) the groups are split into `parts`
    // contiguous ranges so that every thread works: each (node, part) sum goes
    // to the unused upper part of g0/g2 and the parts are added in order.
    const double g1 = 1.0 + g * g, gg = 2.0 * g, norm = (1.0 - g * g) / (4.0 * kPi);
    constexpr int kSplitNodes = NODES / 4;
    const int parts = n <= kSplitNodes ? max(1, min(3, (int)blockDim.x / n)) : 1;
    for (int it = tid; it < n * parts; it += blockDim.x) {
      const int k = it % n, part = it / n;
      const int q0 = part * count / parts, q1 = (part + 1) * count / parts;
      double a0s = 0.0, a2s = 0.0;
      for (int q = q0; q < q1; ++q) {
        const double* row = S.mom + q * kO1MaxValues;
        const double omega = row[2 * nm];
        if (omega <= 0.0) continue;
        const double sin_t = S.sin_q[q], cos_t = S.cos_q[q];
        const double rs = r_b * sin_t;
        double c, s, path_jacobian;
        if (backward) {
          const double shift = S.s[k] - r_b * cos_t;
          const double den = rs * rs + shift * shift;
          c = (rs * rs - shift * shift) / den;
          s = 2.0 * rs * shift / den;
          path_jacobian = 2.0 * r_b / den;
        } else {
          const double y = (S.s[k] - r_b) / rs + sin_t / (1.0 + cos_t);
          const double inv = 1.0 / (1.0 + y * y);
          c = (1.0 - y * y) * inv;
          s = 2.0 * y * inv;
          path_jacobian = 2.0 / (r_b * sin_t) * inv;
        }
        double cpw[5], spw[5];
        cpw[0] = 1.0;
        spw[0] = 1.0;
        for (int pw = 1; pw <= C.max_power; ++pw) {
          cpw[pw] = cpw[pw - 1] * c;
          spw[pw] = spw[pw - 1] * s;
        }
        double a0 = 0.0, a2 = 0.0;
        for (int m = 0; m < nm; ++m) {
          const double basis = S.coef[m] * cpw[S.ipow[m]] * spw[S.jpow[m]];
          a0 += basis * row[m];
          a2 += basis * row[nm + m];
        }
        const double den = g1 - gg * c;
        const double value = path_jacobian * norm / (den * sqrt(den));
        a0s += a0 * value;
        a2s += a2 * value;
      }
      if (parts == 1) {
        S.g0[k] = a0s;
        S.g2[k] = a2s;
      } else {
        S.g0[kSplitNodes * (part + 1) + k] = a0s;
        S.g2[kSplitNodes * (part + 1) + k] = a2s;
      }
    }
    if (parts > 1) {
      __syncthreads();
      for (int k = tid; k < n; k += blockDim.x) {
        double a0s = 0.0, a2s = 0.0;
        for (int part = 0; part < parts; ++part) {
          a0s += S.g0[kSplitNodes * (part + 1) + k];
          a2s += S.g2[kSplitNodes * (part + 1) + k];
        }
        S.g0[k] = a0s;
        S.g2[k] = a2s;
      }
    }
    __syncthreads();
    // _batch_deposit (_prompt_numba.py:451-551) for every band at once: the
    // band constants in shared memory, node times and profile values evaluated
    // from the path grid on the fly, (band, panel) items over the whole CTA,
    // then each band's front ramp by its own thread
    const int d = work[w];
    double* accw = accum + (int64_t)w * per_om;
    const bool bins = C.compute_bins != 0;
    if (tid < NL) {
      const int lam = tid;
      O1BandDeposit& B = S.band[lam];
      B.panels = 0;
      B.total = 0.0;
      if (C.mus[lam] != 0.0) {
        const double v = C.speed[lam];
        int last = n - 1;
        const double limit = r_b + C.tail_exponent / C.mut[lam];
        while (last > 2 && S.s[last - 1] > limit) last -= 1;
        if (last >= 2) {
          B.v = v;
          B.kappa = -C.mut[lam] * v;
          B.last = last;
          B.spread = fmin(front_extra, (S.s[last] - r_b) / v);
          const double front_time = t_b + r_b / v;
          const double end_time = t_b + S.s[last] / v;
          B.outside = front_time - 0.5 * B.spread >= C.edges[nb] ||
                      end_time + 0.5 * B.spread <= C.edges[0];
          B.t_base = B.outside ? 0.0 : t_b;
          B.e_emit = exp(B.kappa * B.t_base);
          const double h_scale = C.mus[lam] * v / B.e_emit;
          B.w0 = C.s0w[lam] * h_scale;
          B.w2 = C.s2w[lam] * h_scale;
          B.h_front = B.w0 * S.g0[0] + B.w2 * S.g2[0];
          // panels start at even nodes with step 2; an odd `last` ends with one step
          B.pairs = last / 2;
          B.panels = B.pairs + (last & 1);
        }
      }
    }
    __syncthreads();
    int n_items = 0;
    for (int lam = 0; lam < NL; ++lam) n_items += S.band[lam].panels;
    for (int item = tid; item < n_items; item += blockDim.x) {
      int lam = 0, pi = item;
      while (pi >= S.band[lam].panels) pi -= S.band[lam].panels, ++lam;
      const O1BandDeposit& B = S.band[lam];
      const double v = B.v, mut = C.mut[lam];
      auto node_t = [&](int j) { return B.t_base + S.s[j] / v; };
      auto node_h = [&](int j) { return (B.w0 * S.g0[j] + B.w2 * S.g2[j]) - B.h_front; };
      double t_a, t_b2, alpha, beta, gamma, e_a, e_b;
      if (pi < B.pairs) {
        const int j = 2 * pi;
        t_a = node_t(j);
        const double t_m = node_t(j + 1);
        t_b2 = node_t(j + 2);
        const double h0 = node_h(j), h1 = node_h(j + 1), h2 = node_h(j + 2);
        const double u_m = t_m - t_a, u_b = t_b2 - t_a;
        const double d1 = (h1 - h0) / u_m;
        const double d2 = ((h2 - h1) / (t_b2 - t_m) - d1) / u_b;
        alpha = h0;
        beta = d1 - d2 * u_m;
        gamma = d2;
        e_a = B.e_emit * exp(-mut * S.s[j]);
        e_b = B.e_emit * exp(-mut * S.s[j + 2]);
      } else {
        const int j = B.last - 1;
        const double t_p = node_t(j - 1);
        t_a = node_t(j);
        t_b2 = node_t(j + 1);
        const double hp = node_h(j - 1), h0 = node_h(j), h1 = node_h(j + 1);
        const double u_m = t_a - t_p, u_b = t_b2 - t_p;
        const double d1 = (h0 - hp) / u_m;
        const double d2 = ((h1 - h0) / (t_b2 - t_a) - d1) / u_b;
        alpha = h0;
        beta = d1 - d2 * u_m + 2.0 * d2 * u_m;
        gamma = d2;
        e_a = B.e_emit * exp(-mut * S.s[j]);
        e_b = B.e_emit * exp(-mut * S.s[j + 1]);
      }
      atomicAdd(&S.band[lam].total, o1_quad(e_a, alpha, beta, gamma, t_b2 - t_a, B.kappa, e_b));
      if (bins && !B.outside) {
        double* pre = accw + (int64_t)lam * (3 + 4 * nb + 1);
        o1_deposit_panel(t_a, t_b2, e_a, e_b, alpha, beta, gamma, B.kappa, C.edges,
                         C.eedge + (int64_t)lam * C.n_edges, nb, pre, pre + 3, C.direct_bins);
      }
    }
    __syncthreads();
    if (tid < NL && S.band[tid].panels > 0) {
      const int lam = tid;
      const O1BandDeposit& B = S.band[lam];
      const double* eedge = C.eedge + (int64_t)lam * C.n_edges;
      double* pre = accw + (int64_t)lam * (3 + 4 * nb + 1);
      double* acc = pre + 3;
      double* chg = acc + 4 * nb;
      double sum = B.total;
      // front step as a mass-normalised ramp of width `spread`
      const double e_first = B.e_emit * exp(-C.mut[lam] * S.s[0]);
      const double e_last = B.e_emit * exp(-C.mut[lam] * S.s[B.last]);
      const double t_f = B.t_base + S.s[0] / B.v, t_end = B.t_base + S.s[B.last] / B.v;
      const double h_front = B.h_front, spread = B.spread, kappa = B.kappa;
      const double exact = o1_quad(e_first, h_front, 0.0, 0.0, t_end - t_f, kappa, e_last);
      sum += exact;
      if (bins && spread > 0.0 && !B.outside) {
        const double t_1 = t_f - 0.5 * spread, t_2 = t_f + 0.5 * spread;
        const double e_1 = exp(kappa * t_1), e_2 = exp(kappa * t_2);
        const double ramp = o1_quad(e_1, 0.0, 1.0 / spread, 0.0, spread, kappa, e_2);
        const double flat = t_end > t_2 ? o1_quad(e_2, 1.0, 0.0, 0.0, t_end - t_2, kappa, e_last) : 0.0;
        const double height = ramp + flat != 0.0 ? exact / (ramp + flat) : 0.0;
        o1_deposit_panel(t_1, t_2, e_1, e_2, 0.0, height / spread, 0.0, kappa, C.edges, eedge,
                         nb, pre, acc, C.direct_bins);
        if (t_end > t_2)
          o1_deposit_panel(t_2, t_end, e_2, e_last, height, 0.0, 0.0, kappa, C.edges, eedge, nb,
                           pre, acc, C.direct_bins);
      } else if (bins && t_end > t_f && !B.outside) {
        o1_deposit_panel(t_f, t_end, e_first, e_last, h_front, 0.0, 0.0, kappa, C.edges, eedge,
                         nb, pre, acc, C.direct_bins);
      }
      atomicAdd(chg, sum);
    }
    (void)d;
  }
}

// _finalize (_prompt_numba.py:610-632): one CTA per work OM.
__global__ void o1_finalize_kernel(const lh_order1_config C, const int32_t* work, int32_t n_work,
                                   const double* accum, double* charge, double* bins) {
  const int w = blockIdx.x;
  const int d = work[w];
  const int nb = C.n_edges - 1;
  const int NL = C.n_bands;
  const int64_t per_om = (int64_t)NL * (3 + 4 * nb + 1);
  const double* accw = accum + (int64_t)w * per_om;
  const double area = C.om_area[d];
  if (threadIdx.x == 0) {
    double total = 0.0;
    for (int lam = 0; lam < NL; ++lam) total += accw[(int64_t)lam * (3 + 4 * nb + 1) + 3 + 4 * nb];
    charge[d] = area * total;
  }
  if (!C.compute_bins || !bins) return;
  // one thread per band runs the prefix; the bands are summed in order
  extern __shared__ __align__(16) unsigned char o1f_smem[];
  double* band_bins = reinterpret_cast<double*>(o1f_smem);
  for (int lam = threadIdx.x; lam < NL; lam += blockDim.x) {
    const double* pre = accw + (int64_t)lam * (3 + 4 * nb + 1);
    const double* acc = pre + 3;
    const double* eedge = C.eedge + (int64_t)lam * C.n_edges;
    const double* itab = C.itab + (int64_t)lam * nb * 3;
    double a = pre[0], b = pre[1], c = pre[2];
    for (int k = 0; k < nb; ++k) {
      const double e_k = C.edges[k];
      const double width = C.edges[k + 1] - e_k;
      const double a_loc = a + e_k * (b + c * e_k);
      const double b_loc = b + 2.0 * c * e_k;
      const double value = eedge[k] * width *
                           (a_loc * itab[3 * k] + width * (b_loc * itab[3 * k + 1] + width * c * itab[3 * k + 2]));
      band_bins[(int64_t)lam * nb + k] = area * (value + acc[4 * k + 3]);
      a += acc[4 * k];
      b += acc[4 * k + 1];
      c += acc[4 * k + 2];
    }
  }
  __syncthreads();
  for (int k = threadIdx.x; k < nb; k += blockDim.x) {
    double sum = 0.0;
    for (int lam = 0; lam < NL; ++lam) sum += band_bins[(int64_t)lam * nb + k];
    bins[(int64_t)d * nb + k] = sum;
  }
}

// ------------------------------------------------------------------ host side

struct O1Workspace {
  long long* pkeys;
  double* prows;
  int32_t* pcount;
  int32_t* tiles;
  long long* parent_keys;  // screen tables: parent pixels (same capacity as pkeys)
  double* parent_rows;
  int32_t* parent_tiles;
  int32_t* parent_row;     // row of each parent slot in the pencil table
  long long* gkeys;
  double* grows;
  int32_t* gcount;
  int32_t* sorted;
  int32_t* batch_list;
  int32_t* batch_total;  // [4]: batches, then batches deferred to the full-size grid
  int32_t* deferred;     // batches whose path grid exceeds kO1SmallNodes
  double* accum;
  unsigned long long* sort_keys;  // tables above kO1SmemSort only
  int32_t* sort_slots;
  size_t bytes;
};

static size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

static O1Workspace o1_layout(const lh_order1_config& C, int64_t pencil_capacity, int64_t ring_capacity,
                             int32_t n_work, unsigned char* base) {
  O1Workspace W{};
  size_t off = 0;
  auto take = [&](size_t bytes) {
    unsigned char* p = base ? base + off : nullptr;
    off += align256(bytes);
    return p;
  };
  const int nb = C.n_edges - 1;
  W.pkeys = reinterpret_cast<long long*>(take(sizeof(long long) * ring_capacity));
  W.prows = reinterpret_cast<double*>(take(sizeof(double) * kO1Moments * ring_capacity));
  W.pcount = reinterpret_cast<int32_t*>(take(sizeof(int32_t) * 4));
  W.tiles = reinterpret_cast<int32_t*>(take(sizeof(int32_t) * (ring_capacity / kO1Tile + 1)));
  const int64_t parent_cap = C.screen ? ring_capacity : 0;
  W.parent_keys = reinterpret_cast<long long*>(take(sizeof(long long) * parent_cap));
  W.parent_rows = reinterpret_cast<double*>(take(sizeof(double) * kO1Moments * parent_cap));
  W.parent_tiles = reinterpret_cast<int32_t*>(take(sizeof(int32_t) * (parent_cap / kO1Tile + 1)));
  W.parent_row = reinterpret_cast<int32_t*>(take(sizeof(int32_t) * parent_cap));
  W.gkeys = reinterpret_cast<long long*>(take(sizeof(long long) * (size_t)n_work * C.group_capacity));
  W.grows = reinterpret_cast<double*>(
      take(sizeof(double) * kO1MaxValues * (size_t)n_work * C.group_capacity));
  W.gcount = reinterpret_cast<int32_t*>(take(sizeof(int32_t) * (size_t)n_work));
  W.sorted = reinterpret_cast<int32_t*>(take(sizeof(int32_t) * (size_t)n_work * C.group_capacity));
  W.batch_list =
      reinterpret_cast<int32_t*>(take(sizeof(int32_t) * 3 * (size_t)n_work * C.group_capacity));
  W.batch_total = reinterpret_cast<int32_t*>(take(sizeof(int32_t) * 4));
  W.deferred = reinterpret_cast<int32_t*>(take(sizeof(int32_t) * (size_t)n_work * C.group_capacity));
  W.accum = reinterpret_cast<double*>(take(sizeof(double) * (size_t)n_work * C.n_bands * (3 + 4 * nb + 1)));
  const size_t sort_n = C.group_capacity > kO1SmemSort ? (size_t)n_work * C.group_capacity : 0;
  W.sort_keys = reinterpret_cast<unsigned long long*>(take(sizeof(unsigned long long) * sort_n));
  W.sort_slots = reinterpret_cast<int32_t*>(take(sizeof(int32_t) * sort_n));
  (void)pencil_capacity;
  W.bytes = off;
  return W;
}

static int64_t next_pow2(int64_t x) {
  int64_t p = 1;
  while (p < x) p <<= 1;
  return p;
}

int64_t o1_ring_capacity(int64_t n_subseg, int32_t ring_nodes) {
  return next_pow2(std::max<int64_t>(4096, n_subseg * ring_nodes));
}

static int grid_for(int64_t items, int threads) {
  int64_t blocks = (items + threads - 1) / threads;
  if (blocks < 1) blocks = 1;
  if (blocks > 148 * 64) blocks = 148 * 64;
  return (int)blocks;
}

}  // namespace lh

namespace {
bool o1_config_valid(const lh_order1_config* C) {
  if (!C) return false;
  if (C->n_om < 1 || !C->om_pos || !C->om_look || !C->om_area) return false;
  if (C->n_bands < 1 || C->n_bands > lh::kO1MaxBands || !C->mus || !C->mut || !C->speed ||
      !C->s0w || !C->s2w)
    return false;
  if (C->n_mono < 1 || C->n_mono > lh::kO1MaxMono || C->max_power < 0 || C->max_power > 4 ||
      !C->coef || !C->ipow || !C->jpow)
    return false;
  if (C->n_edges < 2 || !C->edges || !C->eedge || !C->itab) return false;
  if (C->max_path_nodes < 4 || C->max_path_nodes > lh::kO1MaxNodes) return false;
  if (C->n_gauss < 1 || C->n_gauss > lh::kO1MaxGauss || !C->gauss_tau || !C->gauss_w) return false;
  if (C->group_capacity < 1024 || C->group_capacity > (1 << 20) ||
      (C->group_capacity & (C->group_capacity - 1)))
    return false;
  if (C->theta_bins < 2 || C->theta_bins > 128 || !(C->theta_lo > 0) || !(C->theta_ratio > 0) ||
      !(C->tau_step > 0) || !(C->log_r_step > 0))
    return false;
  if (C->pixel_face < 1 || C->ring_nodes < 1 || !(C->cell_m > 0)) return false;
  if (C->screen && (C->parent_face < 1 || C->pixel_face % C->parent_face || C->compute_bins))
    return false;
  return true;
}
}  // namespace

extern "C" size_t lh_order1_workspace_bytes(const lh_order1_config* C, int64_t n_subseg,
                                            int32_t n_work) {
  if (!o1_config_valid(C) || n_subseg < 0 || n_work < 0) return 0;
  const int64_t ring_cap = lh::o1_ring_capacity(n_subseg, C->ring_nodes);
  return lh::o1_layout(*C, 0, ring_cap, n_work, nullptr).bytes;
}

extern "C" int lh_order1_pencils(const lh_order1_config* C, const lh_order1_elements* E,
                                 const lh_order1_pencil_table* P, int32_t* n_pencils_device,
                                 void* workspace, size_t workspace_bytes, int32_t* status,
                                 void* stream) {
  if (!o1_config_valid(C) || !E || !P || !n_pencils_device || !status) return LH_EINVAL;
  if (C->screen && !P->parent) return LH_EINVAL;
  if (E->n_el < 0 || E->n_subseg < 0 || (E->n_el && (!E->subseg_offset || !E->start ||
                                                     !E->direction || !E->length || !E->c0 ||
                                                     !E->c2 || !E->cone_cos || !E->t0 || !E->t1)))
    return LH_EINVAL;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int64_t ring_cap = lh::o1_ring_capacity(E->n_subseg, C->ring_nodes);
  lh::O1Workspace W = lh::o1_layout(*C, 0, ring_cap, 0, static_cast<unsigned char*>(workspace));
  if (!workspace || workspace_bytes < W.bytes) return LH_ENOMEM;
  cudaMemsetAsync(n_pencils_device, 0, sizeof(int32_t), s);
  if (E->n_el == 0 || E->n_subseg == 0) return cudaGetLastError() == cudaSuccess ? LH_OK : LH_ECUDA;
  cudaMemsetAsync(W.pkeys, 0xff, sizeof(long long) * ring_cap, s);  // rows: zeroed on claim
  const int64_t ring_threads = ((E->n_subseg + 31) / 32) * 32 *
                               ((C->ring_nodes + lh::kO1RingBlock - 1) / lh::kO1RingBlock);
  {
    lh::TimedLaunch timed_launch(LH_KT_O1_RING, s);
    lh::o1_ring_kernel<<<lh::grid_for(ring_threads, lh::kO1RingThreads), lh::kO1RingThreads, 0, s>>>(
        *C, *E, E->subseg_offset, E->n_subseg, W.pkeys, ring_cap, W.prows, status);
  }
  const int64_t n_tiles = (ring_cap + lh::kO1Tile - 1) / lh::kO1Tile;
  if (!C->screen) {
    lh::o1_tile_count_kernel<<<(unsigned)n_tiles, lh::kO1FinishThreads, 0, s>>>(
        W.pkeys, W.prows, ring_cap, W.tiles);
    lh::o1_tile_scan_kernel<<<1, 1024, 0, s>>>(W.tiles, n_tiles, n_pencils_device);
    lh::o1_finish_kernel<<<(unsigned)n_tiles, lh::kO1FinishThreads, 0, s>>>(
        W.pkeys, ring_cap, W.prows, *P, W.tiles, n_pencils_device, nullptr, nullptr, nullptr, 0,
        nullptr, 0, 0, status);
    return cudaGetLastError() == cudaSuccess ? LH_OK : LH_ECUDA;
  }
  // the coarse screen: parents (sums of their children) take rows [0, n_parents),
  // children follow with their parent's row
  cudaMemsetAsync(W.parent_keys, 0xff, sizeof(long long) * ring_cap, s);
  cudaMemsetAsync(W.parent_row, 0xff, sizeof(int32_t) * ring_cap, s);
  lh::o1_parent_kernel<<<lh::grid_for(ring_cap, lh::kO1FinishThreads), lh::kO1FinishThreads, 0, s>>>(
      W.pkeys, W.prows, ring_cap, C->pixel_face, C->parent_face, W.parent_keys, W.parent_rows,
      ring_cap, status);
  lh::o1_tile_count_kernel<<<(unsigned)n_tiles, lh::kO1FinishThreads, 0, s>>>(
      W.parent_keys, W.parent_rows, ring_cap, W.parent_tiles);
  lh::o1_tile_scan_kernel<<<1, 1024, 0, s>>>(W.parent_tiles, n_tiles, W.pcount + 1);
  lh::o1_finish_kernel<<<(unsigned)n_tiles, lh::kO1FinishThreads, 0, s>>>(
      W.parent_keys, ring_cap, W.parent_rows, *P, W.parent_tiles, W.pcount + 1, nullptr,
      W.parent_row, nullptr, 0, nullptr, 0, 0, status);
  lh::o1_tile_count_kernel<<<(unsigned)n_tiles, lh::kO1FinishThreads, 0, s>>>(
      W.pkeys, W.prows, ring_cap, W.tiles);
  lh::o1_tile_scan_kernel<<<1, 1024, 0, s>>>(W.tiles, n_tiles, W.pcount);
  lh::o1_finish_kernel<<<(unsigned)n_tiles, lh::kO1FinishThreads, 0, s>>>(
      W.pkeys, ring_cap, W.prows, *P, W.tiles, W.pcount, W.pcount + 1, nullptr, W.parent_keys,
      ring_cap, W.parent_row, C->pixel_face, C->parent_face, status);
  lh::o1_total_kernel<<<1, 32, 0, s>>>(W.pcount, W.pcount + 1, n_pencils_device);
  return cudaGetLastError() == cudaSuccess ? LH_OK : LH_ECUDA;
}

extern "C" int lh_order1_grouped(const lh_order1_config* C, const lh_order1_pencil_table* P,
                                 int32_t n_pencils, const int32_t* n_pencils_device,
                                 const int32_t* work, int32_t n_work,
                                 const double* origins, double* charge, double* bins,
                                 void* workspace, size_t workspace_bytes, int32_t* status,
                                 void* stream) {
  if (!o1_config_valid(C) || !P || n_pencils < 0 || n_work < 0 || !status || !charge) return LH_EINVAL;
  if (C->screen && !P->parent) return LH_EINVAL;
  if (n_work && (!work || !origins)) return LH_EINVAL;
  if (C->compute_bins && !bins) return LH_EINVAL;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // the grouped stage reuses the workspace from its start (pencils live elsewhere)
  lh::O1Workspace W = lh::o1_layout(*C, 0, 0, n_work, static_cast<unsigned char*>(workspace));
  if (!workspace || workspace_bytes < W.bytes) return LH_ENOMEM;
  const int nb = C->n_edges - 1;
  cudaMemsetAsync(charge, 0, sizeof(double) * C->n_om, s);
  if (C->compute_bins) cudaMemsetAsync(bins, 0, sizeof(double) * (size_t)C->n_om * nb, s);
  if (n_work == 0 || n_pencils == 0) return cudaGetLastError() == cudaSuccess ? LH_OK : LH_ECUDA;
  const int64_t cap = C->group_capacity;
  cudaMemsetAsync(W.gkeys, 0xff, sizeof(long long) * (size_t)n_work * cap, s);  // rows: zeroed on claim
  cudaMemsetAsync(W.gcount, 0, sizeof(int32_t) * (size_t)n_work, s);
  cudaMemsetAsync(W.batch_total, 0, sizeof(int32_t) * 4, s);
  cudaMemsetAsync(W.accum, 0, sizeof(double) * (size_t)n_work * C->n_bands * (3 + 4 * nb + 1), s);
  const size_t group_smem =
      sizeof(double) * 32 * (256 / 32) * (2 * C->n_mono + 6 + lh::kO1PencilFields);
  if (group_smem > 48 * 1024 &&
      cudaFuncSetAttribute(C->screen ? lh::o1_group_kernel<true> : lh::o1_group_kernel<false>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)group_smem) != cudaSuccess)
    return LH_ECUDA;
  {
    lh::TimedLaunch timed_launch(LH_KT_O1_GROUP, s);
    // persistent: two resident CTAs per SM take the warp chunks in turn (the
    // host's pencil count is the table's capacity, far above the pencils a
    // shower makes, so a grid sized from it would mostly launch idle CTAs)
    const int group_grid = std::min(lh::grid_for((int64_t)n_work * n_pencils, 256), 148 * 2);
    unsigned long long* units = lh::kernel_units() ? lh::kernel_units() + LH_KT_O1_GROUP : nullptr;
    if (C->screen)
      lh::o1_group_kernel<true><<<group_grid, 256, group_smem, s>>>(
          *C, *P, n_pencils, n_pencils_device, work, n_work, origins, W.gkeys, W.grows,
          W.gcount, status, units);
    else
      lh::o1_group_kernel<false><<<group_grid, 256, group_smem, s>>>(
          *C, *P, n_pencils, n_pencils_device, work, n_work, origins, W.gkeys, W.grows,
          W.gcount, status, units);
  }
  const size_t sort_smem =
      cap <= lh::kO1SmemSort ? sizeof(unsigned long long) * (size_t)cap : 0;
  if (sort_smem > 48 * 1024 &&
      cudaFuncSetAttribute(lh::o1_batches_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)sort_smem) != cudaSuccess)
    return LH_ECUDA;
  lh::o1_batches_kernel<<<n_work, 1024, sort_smem, s>>>(*C, n_work, W.gkeys, W.sorted, W.batch_list,
                                                        W.batch_total, W.sort_keys, W.sort_slots,
                                                        status);
  const size_t small_smem = sizeof(lh::O1BatchShared<lh::kO1SmallNodes>);
  const size_t full_smem = sizeof(lh::O1BatchShared<lh::kO1MaxNodes>);
  if (cudaFuncSetAttribute(lh::o1_batch_kernel<lh::kO1SmallNodes>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)small_smem) != cudaSuccess ||
      cudaFuncSetAttribute(lh::o1_batch_kernel<lh::kO1MaxNodes>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)full_smem) != cudaSuccess)
    return LH_ECUDA;
  {
    lh::TimedLaunch timed_launch(LH_KT_O1_BATCH, s);
    lh::o1_batch_kernel<lh::kO1SmallNodes><<<148 * 5, lh::kO1BatchThreads, small_smem, s>>>(
        *C, work, W.gkeys, W.grows, W.sorted, W.batch_list, W.batch_total, W.deferred,
        W.batch_total + 1, W.accum, status);
    lh::o1_batch_kernel<lh::kO1MaxNodes><<<148 * 2, lh::kO1BatchThreads, full_smem, s>>>(
        *C, work, W.gkeys, W.grows, W.sorted, W.batch_list, W.batch_total, W.deferred,
        W.batch_total + 1, W.accum, status);
  }
  const size_t fin_smem = sizeof(double) * C->n_bands * nb;
  if (fin_smem > 200 * 1024) return LH_EUNSUPPORTED;
  if (cudaFuncSetAttribute(lh::o1_finalize_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)fin_smem) != cudaSuccess)
    return LH_ECUDA;
  lh::o1_finalize_kernel<<<n_work, 128, fin_smem, s>>>(*C, work, n_work, W.accum, charge, bins);
  return cudaGetLastError() == cudaSuccess ? LH_OK : LH_ECUDA;
}

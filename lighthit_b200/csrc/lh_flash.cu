// Isotropic calibration flashes, all scattering orders, on the device.
//
// Reference: TransportKernel._transport_isotropic (transport.py:1061-1164) with
// ResponseCache.acceptance_spectrum / moments_at (cache.py:294-436) and
// readout_bins (readout.py:43-72), for a monochromatic flash and the
// centre-ray receiver.
//
// Work decomposition: a tile is 64 (flash, OM) pairs = 128 readout rows
// (orders 1 and 2 of each pair).
//  1. pair setup (float64, one thread per pair): distance, head-on cosine,
//     acceptance, the OM clock time_origin_ns, the order-0 bin, the radial
//     interval of the log-r spline and the safety bound of transport.py:1115;
//  2. spectrum (float32, one thread per (pair, omega)): cubic in log r of the
//     detrended multipole moments, contracted with alpha_l P_l(cos)/(4 pi),
//     times attenuation and the flight phase; writes the absolute spectrum and
//     the demodulated (relative) spectrum of orders 1 and 2 as readout rows;
//  3. readout of the rows (see lh_readout.cu) and the order-0 bin rows,
//     charge (spectrum at the first frequency) and the active mask.
// flash_tc_kernel fuses 1-3 in one persistent kernel: the readout rows are
// written straight into shared memory as the tensor-core A tile.
#include "lh_common.cuh"
#include "lh_readout.cuh"

namespace lh {

constexpr int kFlashPairs = 64;  // pairs per tile -> 128 readout rows
constexpr int kMaxAcc = 8;       // highest acceptance degree handled
constexpr int kFlashThreads = 256;    // plain path
constexpr int kFlashTcThreads = 512;  // fused path: 16 warps hide the table-load latency
// A tile of the fused path: K-major, no swizzle, [k/8][row][k%8] with each
// 8-column chunk of the 128 rows padded by 16 bytes (2064 B apart, the MMA's
// leading byte offset). A warp stores 32 consecutive columns of one row: the
// padding puts their four chunks in different banks (2048 B apart they shared
// four banks: 4-way conflicts on every A-tile store).
constexpr int kAChunk = 128 * 8 + 8;   // elements per 8-column chunk
LH_DEVICE int a_offset(int row, int k) { return (k >> 3) * kAChunk + row * 8 + (k & 7); }

struct FlashPair {
  double origin;  // time_origin_ns of the OM for this flash
  double t12;     // r / speed: flight time of the spectrum phase (orders 1, 2)
  double t0;      // absolute order-0 phase time (r / speed inside, t + r / speed outside)
  double q0;      // order-0 bin weight
  double c12, c0, cr;  // t12, t0 and t12 - origin in turns per (rad/ns): t / (2 pi)
  float tt;       // offset in the log-r interval
  float amp12;    // photons * area * efficiency * exp(-mu_a r) / (4 pi r^2)
  float amp0;     // order-0 amplitude
  int j;          // log-r interval, -1 outside the table's radial range
  int bin0;       // order-0 bin, -1 outside the window
  int valid;      // pair exists
  int inside;
  int flags;      // bit 1: unsafe (outside range, bound above threshold); bit 2: coincident
  float w[kMaxAcc + 1];  // alpha_l P_l(cos) / (4 pi)
  float charge[3];
};

// Flashes in this launch: the device count when given (graph replay), else n_flash.
LH_DEVICE int flash_count(const lh_flash_batch& b) {
  if (b.n_flash_device) {
    const int n = *b.n_flash_device;
    return n < 0 ? 0 : (n > b.n_flash ? b.n_flash : n);
  }
  return b.n_flash;
}

// Step 1 for one pair.
LH_DEVICE void flash_pair_setup(const lh_flash_problem& p, const lh_flash_batch& b, int64_t pair,
                                FlashPair& s) {
  const int n_om = p.n_om;
  const int64_t f = pair / n_om;
  const int d = (int)(pair % n_om);
  const double sx = b.pos[3 * f], sy = b.pos[3 * f + 1], sz = b.pos[3 * f + 2];
  const double px = p.om_pos[3 * d], py = p.om_pos[3 * d + 1], pz = p.om_pos[3 * d + 2];
  // displacement = positions - source; radii = |displacement| (transport.py:1069-1070)
  const double dx = __dsub_rn(px, sx), dy = __dsub_rn(py, sy), dz = __dsub_rn(pz, sz);
  const double r = sqrt(dot3_rn(dx, dy, dz, dx, dy, dz));
  s.flags = 0;
  if (r == 0.0) {
    atomicOr(reinterpret_cast<unsigned*>(b.status), LH_STATUS_COINCIDENT);
    s.flags |= 4;
  }
  // head_on_cosine (model.py:158-162): toward = (source - position) / |.|
  const double tx = __dsub_rn(sx, px), ty = __dsub_rn(sy, py), tz = __dsub_rn(sz, pz);
  const double tn = sqrt(dot3_rn(tx, ty, tz, tx, ty, tz));
  const double cosine = dot3_rn(p.om_look[3 * d], p.om_look[3 * d + 1], p.om_look[3 * d + 2],
                                tx / tn, ty / tn, tz / tn);
  // Legendre P_l(cos): acceptance A = sum alpha_l (2l+1) P_l / (4 pi) (cache.py:509-521)
  // and contraction weights alpha_l P_l / (4 pi) (cache.py:416-418)
  double pl_prev = 1.0, pl = cosine, acc = 0.0;
  for (int l = 0; l <= p.acc_top; ++l) {
    double P;
    if (l == 0) P = 1.0;
    else if (l == 1) P = cosine;
    else {
      P = ((2 * l - 1) * cosine * pl - (l - 1) * pl_prev) / l;
      pl_prev = pl;
      pl = P;
    }
    acc += p.alpha[l] * (2 * l + 1) * P / (4 * kPi);
    s.w[l] = (float)(P * p.alpha[l] / (4 * kPi));
  }
  const double area = p.om_area[d];
  const double photons = b.photons[f];
  const double t_src = b.time_ns[f];
  const double scale = photons * area * p.efficiency;
  const double four_pi_r2 = 4 * kPi * r * r;
  s.q0 = scale * acc * exp(-p.mu_t * r) / four_pi_r2;
  s.inside = (r >= p.r_low) && (r <= p.r_high);
  const double upper = photons * area * p.efficiency * acc * exp(-p.mu_a * r) / four_pi_r2;
  if (!s.inside && 10 * upper >= p.threshold) {
    s.flags |= 2;
    atomicOr(reinterpret_cast<unsigned*>(b.status), LH_STATUS_UNSAFE);
    atomicAdd(b.status + 1, 1);
    atomicMax(reinterpret_cast<unsigned long long*>(b.status + 2),
              (unsigned long long)__double_as_longlong(r));
  }
  const double arrival = t_src + r / p.speed;
  s.origin = t_src + r / p.origin_speed;
  const int bin = bin_right(p.edges, p.n_edges, arrival - s.origin);
  s.bin0 = (bin >= 0 && bin < p.n_edges - 1) ? bin : -1;
  if (s.inside) {
    const double logr = log(r);
    int j = bin_right(p.log_r, p.n_radii, logr);
    j = j < 0 ? 0 : (j > p.n_radii - 2 ? p.n_radii - 2 : j);
    s.j = j;
    s.tt = (float)(logr - p.log_r[j]);
    s.amp12 = (float)(scale * (exp(-p.mu_a * r) / four_pi_r2));
    s.amp0 = (float)(scale * acc * (exp(-p.mu_t * r) / four_pi_r2));
    s.t12 = r / p.speed;
    s.t0 = r / p.speed;
  } else {
    s.j = -1;
    s.tt = 0.f;
    s.amp12 = 0.f;
    s.amp0 = (float)s.q0;
    s.t12 = 0.0;
    s.t0 = arrival;
  }
  const double inv2pi = 1.0 / (2 * kPi);
  s.c12 = s.t12 * inv2pi;
  s.c0 = s.t0 * inv2pi;
  s.cr = (s.t12 - s.origin) * inv2pi;
  s.valid = 1;
}

// exp(2 pi i turns): the turns reduced in float64 to (-1/2, 1/2], the angle in
// float32 on the SFU (absolute error ~1e-6, far inside the 1e-4 bar of the
// spectra and bins).
LH_DEVICE float2 phase_turns(double turns) {
  const float frac = (float)(turns - rint(turns));
  float sv, cv;
  __sincosf((float)(2 * kPi) * frac, &sv, &cv);
  return make_float2(cv, sv);
}

LH_DEVICE float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// Step 2 for one (pair, omega). Returns the relative spectra of orders 1, 2
// through rel1/rel2 and writes the absolute spectrum of all orders.
LH_DEVICE void flash_item(const lh_flash_problem& p, const lh_flash_batch& b, int64_t pair,
                          int w, FlashPair& s, float2& rel1, float2& rel2) {
  const double om = p.omega[w];
  float2 s1 = make_float2(0.f, 0.f), s2 = make_float2(0.f, 0.f);
  if (s.j >= 0) {
    const int L = p.acc_top + 1;
    const int W = p.n_omega;
    // [interval][degree][order][power][omega]: the lanes of a warp (consecutive
    // omega) read consecutive float2, one coalesced segment per coefficient
    const float2* c = reinterpret_cast<const float2*>(p.coef) + (int64_t)s.j * L * 8 * W + w;
    const float t = s.tt;
    for (int l = 0; l < L; ++l) {
      const float2* cl = c + (int64_t)l * 8 * W;
      const float2 a0 = __ldg(cl), a1 = __ldg(cl + W), a2 = __ldg(cl + 2 * W),
                   a3 = __ldg(cl + 3 * W);  // order 1: c0..c3
      const float2 b0 = __ldg(cl + 4 * W), b1 = __ldg(cl + 5 * W), b2 = __ldg(cl + 6 * W),
                   b3 = __ldg(cl + 7 * W);  // order 2
      float vr = fmaf(fmaf(fmaf(a0.x, t, a1.x), t, a2.x), t, a3.x);
      float vi = fmaf(fmaf(fmaf(a0.y, t, a1.y), t, a2.y), t, a3.y);
      const float wl = s.w[l];
      s1.x = fmaf(wl, vr, s1.x);
      s1.y = fmaf(wl, vi, s1.y);
      vr = fmaf(fmaf(fmaf(b0.x, t, b1.x), t, b2.x), t, b3.x);
      vi = fmaf(fmaf(fmaf(b0.y, t, b1.y), t, b2.y), t, b3.y);
      s2.x = fmaf(wl, vr, s2.x);
      s2.y = fmaf(wl, vi, s2.y);
    }
    s1.x *= s.amp12; s1.y *= s.amp12;
    s2.x *= s.amp12; s2.y *= s.amp12;
  }
  const float2 e12 = phase_turns(om * s.c12);
  const float2 e0 = (s.t0 == s.t12) ? e12 : phase_turns(om * s.c0);
  const float2 r12 = s.j >= 0 ? phase_turns(om * s.cr) : make_float2(1.f, 0.f);
  const float2 o0 = make_float2(s.amp0 * e0.x, s.amp0 * e0.y);
  const float2 o1 = cmul(s1, e12), o2 = cmul(s2, e12);
  if (s.valid) {
    float2* out = reinterpret_cast<float2*>(b.spectrum) + (pair * p.n_omega + w) * 3;
    out[0] = o0;
    out[1] = o1;
    out[2] = o2;
    if (w == 0) {
      s.charge[0] = o0.x;
      s.charge[1] = o1.x;
      s.charge[2] = o2.x;
    }
  }
  rel1 = cmul(s1, r12);
  rel2 = cmul(s2, r12);
}

// Step 3 (order 0 and the mask) for the tile's pairs.
// `threads`: the first threads of the CTA that take part (0: all).
LH_DEVICE void flash_tile_order0(const lh_flash_problem& p, const lh_flash_batch& b,
                                 const FlashPair* sp, int64_t base, int n_bins, int threads = 0) {
  const int stride = threads ? threads : (int)blockDim.x;
  if ((n_bins & 3) == 0) {  // rows are 16-byte aligned: four bins per store
    const int quads = n_bins >> 2;
    for (int i = threadIdx.x; i < kFlashPairs * quads; i += stride) {
      const int lp = i / quads, bin = (i % quads) * 4;
      const FlashPair& s = sp[lp];
      if (!s.valid) continue;
      const float q = (float)s.q0;
      const float4 v = make_float4(bin == s.bin0 ? q : 0.f, bin + 1 == s.bin0 ? q : 0.f,
                                   bin + 2 == s.bin0 ? q : 0.f, bin + 3 == s.bin0 ? q : 0.f);
      *reinterpret_cast<float4*>(b.components + ((base + lp) * 3) * n_bins + bin) = v;
    }
  } else {
    for (int i = threadIdx.x; i < kFlashPairs * n_bins; i += stride) {
      const int lp = i / n_bins, bin = i % n_bins;
      const FlashPair& s = sp[lp];
      if (!s.valid) continue;
      b.components[((base + lp) * 3) * n_bins + bin] = (bin == s.bin0) ? (float)s.q0 : 0.f;
    }
  }
  if (threadIdx.x < kFlashPairs) {
    const FlashPair& s = sp[threadIdx.x];
    if (s.valid) {
      const int64_t pair = base + threadIdx.x;
      const double q = ((double)s.charge[0] + (double)s.charge[1]) + (double)s.charge[2];
      for (int o = 0; o < 3; ++o) b.charge[pair * 3 + o] = (double)s.charge[o];
      b.origin[pair] = s.origin;
      const bool active = p.threshold == 0.0 ? s.inside : (s.inside && q >= p.threshold);
      b.active[pair] = (uint8_t)((active ? 1 : 0) | s.flags);
    }
  }
}

LH_DEVICE void flash_slot_setup(const lh_flash_problem& p, const lh_flash_batch& b, FlashPair& s,
                                int64_t pair, int64_t n_pairs) {
  if (pair < n_pairs) {
    flash_pair_setup(p, b, pair, s);
  } else {
    s.valid = 0;
    s.j = -1;
    s.amp12 = s.amp0 = 0.f;
    s.t12 = s.t0 = s.origin = 0.0;
    s.c12 = s.c0 = s.cr = 0.0;
    s.inside = 0;
    s.flags = 0;
  }
  s.charge[0] = s.charge[1] = s.charge[2] = 0.f;
}

LH_DEVICE void flash_tile_setup(const lh_flash_problem& p, const lh_flash_batch& b, FlashPair* sp,
                                int64_t base, int64_t n_pairs) {
  if (threadIdx.x < kFlashPairs)
    flash_slot_setup(p, b, sp[threadIdx.x], base + threadIdx.x, n_pairs);
}

// ---------------------------------------------------------------- plain path
// One block per tile; readout rows go to a row-major fp32 workspace that
// readout_fp32_kernel consumes.
__global__ void __launch_bounds__(kFlashThreads)
flash_plain_kernel(lh_flash_problem p, lh_flash_batch b, int kpad, int n_bins, float* a_rows) {
  __shared__ FlashPair sp[kFlashPairs];
  const int64_t n_pairs = (int64_t)flash_count(b) * p.n_om;
  const int64_t base = (int64_t)blockIdx.x * kFlashPairs;
  flash_tile_setup(p, b, sp, base, n_pairs);
  __syncthreads();
  const int nw = p.n_omega;
  // Every row the readout reads (2 per pair of the host count, whose grid
  // follows) is written in full here: pairs past the device count get zero
  // rows (flash_item yields zero spectra for them), and the padding columns
  // 2 nw .. kpad-1 are zeroed whatever their number.
  const int64_t host_pairs = (int64_t)b.n_flash * p.n_om;
  for (int i = threadIdx.x; i < kFlashPairs * nw; i += blockDim.x) {
    const int lp = i / nw, w = i % nw;
    float2 r1, r2;
    flash_item(p, b, base + lp, w, sp[lp], r1, r2);
    if (base + lp < host_pairs) {
      float* row1 = a_rows + (2 * (base + lp)) * (int64_t)kpad;
      float* row2 = row1 + kpad;
      row1[w] = r1.x;
      row1[nw + w] = r1.y;
      row2[w] = r2.x;
      row2[nw + w] = r2.y;
      for (int c = 2 * nw + w; c < kpad; c += nw) {
        row1[c] = 0.f;
        row2[c] = 0.f;
      }
    }
  }
  __syncthreads();
  flash_tile_order0(p, b, sp, base, n_bins);
}

// ---------------------------------------------------------------- fused tcgen05 path
// 256 threads, one CTA per SM, persistent over tiles. B (the readout operator,
// hi and lo parts) is loaded once per CTA. Per tile: setup -> spectrum items
// writing A (bf16 hi/lo) into shared memory -> one thread issues the MMAs ->
// order-0 rows and mask while the tensor core runs -> TMEM drain.
__global__ void __launch_bounds__(kFlashTcThreads, 1)
flash_tc_kernel(lh_flash_problem p, lh_flash_batch b, const __nv_bfloat16* __restrict__ g_bhi,
                const __nv_bfloat16* __restrict__ g_blo, int kpad, int n_bins, int n_tile,
                int passes) {
  extern __shared__ __align__(1024) uint8_t smem[];
  const uint32_t a_bytes = (uint32_t)(kpad / 8) * kAChunk * 2u;
  const uint32_t b_bytes = (uint32_t)n_tile * kpad * 2u;
  __nv_bfloat16* s_ahi = reinterpret_cast<__nv_bfloat16*>(smem);
  __nv_bfloat16* s_alo = reinterpret_cast<__nv_bfloat16*>(smem + a_bytes);
  __nv_bfloat16* s_bhi = reinterpret_cast<__nv_bfloat16*>(smem + 2 * a_bytes);
  __nv_bfloat16* s_blo = reinterpret_cast<__nv_bfloat16*>(smem + 2 * a_bytes + b_bytes);
  // two pair buffers: the next tile's setup runs while this tile's MMA is in flight
  FlashPair* sp_buf = reinterpret_cast<FlashPair*>(smem + 2 * a_bytes + 2 * b_bytes);
  uint64_t* bars = reinterpret_cast<uint64_t*>(sp_buf + 2 * kFlashPairs);
  uint32_t* s_tmem = reinterpret_cast<uint32_t*>(bars + 2);
  uint64_t* bar_b = bars;
  uint64_t* bar_mma = bars + 1;

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const bool need_lo_b = passes >= 2;
  if (tid == 0) {
    mbar_init(bar_b, 1);
    mbar_init(bar_mma, 1);
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
  if (tid == 0) {
    mbar_expect_tx(bar_b, b_bytes * (need_lo_b ? 2u : 1u));
    bulk_g2s(s_bhi, g_bhi, b_bytes, bar_b);
    if (need_lo_b) bulk_g2s(s_blo, g_blo, b_bytes, bar_b);
  }
  const uint32_t idesc = instr_desc_bf16_f32(128, n_tile);
  const int64_t n_pairs = (int64_t)flash_count(b) * p.n_om;
  const int64_t n_tiles = (n_pairs + kFlashPairs - 1) / kFlashPairs;
  const int nw = p.n_omega;
  const int padw = kpad - 2 * nw;
  uint32_t ph_mma = 0;
  bool b_ready = false, failed = false, mma_pending = false;

  if (blockIdx.x < n_tiles) flash_tile_setup(p, b, sp_buf, blockIdx.x * kFlashPairs, n_pairs);
  __syncthreads();
  int cur = 0;
  for (int64_t tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {
    const int64_t base = tile * kFlashPairs;
    FlashPair* sp = sp_buf + cur * kFlashPairs;  // set up before the barrier closing the last tile
    for (int i = tid; i < 128 * padw; i += blockDim.x) {
      const int off = a_offset(i / padw, 2 * nw + i % padw);
      s_ahi[off] = __float2bfloat16_rn(0.f);
      s_alo[off] = __float2bfloat16_rn(0.f);
    }
    // The last warp sets up the next tile's pairs (float64, two per lane) while
    // the other warps compute this tile's spectra, then issues the MMAs while
    // they write the order-0 rows: neither waits behind the other.
    const int64_t next = tile + gridDim.x;
    const int workers = blockDim.x - 32;
    if (tid >= workers) {
      if (next < n_tiles)
        for (int k = lane; k < kFlashPairs; k += 32)
          flash_slot_setup(p, b, sp_buf[(cur ^ 1) * kFlashPairs + k], next * kFlashPairs + k,
                           n_pairs);
    } else {
      for (int i = tid; i < kFlashPairs * nw; i += workers) {
        const int lp = i / nw, w = i % nw;
        float2 r1, r2;
        flash_item(p, b, base + lp, w, sp[lp], r1, r2);
        // K columns (Re, Im) per frequency: one bf16x2 store per row and part
        const __nv_bfloat162 h1 = __floats2bfloat162_rn(r1.x, r1.y);
        const __nv_bfloat162 l1 = __floats2bfloat162_rn(r1.x - __low2float(h1),
                                                        r1.y - __high2float(h1));
        const __nv_bfloat162 h2 = __floats2bfloat162_rn(r2.x, r2.y);
        const __nv_bfloat162 l2 = __floats2bfloat162_rn(r2.x - __low2float(h2),
                                                        r2.y - __high2float(h2));
        const int o1 = a_offset(2 * lp, 2 * w), o2 = a_offset(2 * lp + 1, 2 * w);
        *reinterpret_cast<__nv_bfloat162*>(s_ahi + o1) = h1;
        *reinterpret_cast<__nv_bfloat162*>(s_alo + o1) = l1;
        *reinterpret_cast<__nv_bfloat162*>(s_ahi + o2) = h2;
        *reinterpret_cast<__nv_bfloat162*>(s_alo + o2) = l2;
      }
    }
    fence_proxy_async();  // generic-proxy smem writes -> visible to the tensor core
    __syncthreads();
    if (tid == workers) {
      bool ok = true;
      if (!b_ready) {
        ok = mbar_wait(bar_b, 0);
        b_ready = true;
      }
      if (ok) {
        tc_fence_after();
        const int ksteps = kpad / 16;
        const uint32_t lbo_a = kAChunk * 2u, lbo_b = (uint32_t)n_tile * 16u;
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
      } else {
        failed = true;
      }
    }
    if (tid < workers) flash_tile_order0(p, b, sp, base, n_bins, workers);
    if (__syncthreads_or(failed)) { failed = true; break; }
    const bool ok = mbar_wait(bar_mma, ph_mma);
    ph_mma ^= 1u;
    if (__syncthreads_or(!ok)) { failed = true; mma_pending = true; break; }
    tc_fence_after();
    // drain: warp w reads TMEM lanes 32*(w%4).. (rows); the warps with the same
    // lane quarter split the 16-column chunks between them
    const int q = warp & 3, h = warp >> 2, groups = (int)blockDim.x / 128;
    const int row = q * 32 + lane;
    const int lp = row >> 1, order = 1 + (row & 1);
    const bool valid = sp[lp].valid;
    const int chunks = n_tile / 16;
    const int per = (chunks + groups - 1) / groups;
    const int c_begin = h * per, c_end = min(chunks, (h + 1) * per);
    const uint32_t lane_addr = tmem + ((uint32_t)(q * 32) << 16);
    float* dst = b.components + ((base + lp) * 3 + order) * (int64_t)n_bins;
    const bool vec = (n_bins & 3) == 0;
    // The A tile is free once the MMA has completed: each warp transposes its
    // 32 rows x 16 bins through a 32 x 20-float slice of it, so that four
    // lanes store one row's 64 bytes and a store instruction covers eight rows
    // (full 32-byte sectors) instead of 32 rows at a 16-byte stride.
    float* stage = reinterpret_cast<float*>(smem) + warp * 32 * 20;
    const bool staged = vec && 2u * a_bytes >= (blockDim.x / 32) * 32u * 20u * sizeof(float);
    for (int c = c_begin; c < c_end; ++c) {
      float v[16];
      tmem_ld16(lane_addr + (uint32_t)(c * 16), v);
      if (staged && c * 16 + 16 <= n_bins) {
#pragma unroll
        for (int i = 0; i < 4; ++i)
          *reinterpret_cast<float4*>(stage + lane * 20 + 4 * i) =
              make_float4(v[4 * i], v[4 * i + 1], v[4 * i + 2], v[4 * i + 3]);
        __syncwarp();
#pragma unroll
        for (int it = 0; it < 4; ++it) {
          const int r = it * 8 + (lane >> 2), part = lane & 3;
          const int trow = q * 32 + r;
          const int tlp = trow >> 1, torder = 1 + (trow & 1);
          if (sp[tlp].valid) {
            const float4 x = *reinterpret_cast<const float4*>(stage + r * 20 + 4 * part);
            *reinterpret_cast<float4*>(b.components + ((base + tlp) * 3 + torder) * (int64_t)n_bins +
                                       c * 16 + 4 * part) = x;
          }
        }
        __syncwarp();
      } else if (valid) {
#pragma unroll
        for (int i = 0; i < 16; ++i)
          if (c * 16 + i < n_bins) dst[c * 16 + i] = v[i];
      }
    }
    tc_fence_before();
    __syncthreads();
    cur ^= 1;
  }
  if (failed && tid == 0) atomicOr(reinterpret_cast<unsigned*>(b.status), LH_STATUS_TIMEOUT);
  if (mma_pending) mbar_wait(bar_mma, ph_mma ^ 1u);
  if (tid == blockDim.x - 32 && !b_ready) mbar_wait(bar_b, 0);  // no bulk copy left in flight
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, 256);
}

// ---------------------------------------------------------------- broadband
// Sum of the node runs of a broadband flash and the mask and range check of
// the sum (transport.py:1088-1164). Grid-stride over the spectrum and bins
// (node order fixed: identical results alone or in a batch), then one thread
// per pair: charge, the absorption-only estimate over the nodes, flags.
__global__ void flash_combine_kernel(lh_flash_problem p, lh_flash_nodes nd, lh_flash_batch b) {
  const int64_t n_pairs = (int64_t)flash_count(b) * p.n_om;
  const int nb = p.n_edges - 1;
  const int64_t first = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const int64_t n_spec = n_pairs * p.n_omega * 6;  // floats
  for (int64_t i = first; i < n_spec; i += stride) {
    float v = 0.f;
    for (int n = 0; n < nd.n_nodes; ++n) v += nd.spectrum[n][i];
    b.spectrum[i] = v;
  }
  const int64_t n_comp = n_pairs * 3 * nb;
  for (int64_t i = first; i < n_comp; i += stride) {
    float v = 0.f;
    for (int n = 0; n < nd.n_nodes; ++n) v += nd.components[n][i];
    b.components[i] = v;
  }
  for (int64_t pair = first; pair < n_pairs; pair += stride) {
    double q[3] = {0.0, 0.0, 0.0};
    for (int n = 0; n < nd.n_nodes; ++n)
      for (int o = 0; o < 3; ++o) q[o] += nd.charge[n][pair * 3 + o];
    for (int o = 0; o < 3; ++o) b.charge[pair * 3 + o] = q[o];
    // geometry and acceptance as flash_pair_setup
    const int64_t f = pair / p.n_om;
    const int d = (int)(pair % p.n_om);
    const double sx = b.pos[3 * f], sy = b.pos[3 * f + 1], sz = b.pos[3 * f + 2];
    const double px = p.om_pos[3 * d], py = p.om_pos[3 * d + 1], pz = p.om_pos[3 * d + 2];
    const double dx = __dsub_rn(px, sx), dy = __dsub_rn(py, sy), dz = __dsub_rn(pz, sz);
    const double r = sqrt(dot3_rn(dx, dy, dz, dx, dy, dz));
    int flags = 0;
    if (r == 0.0) {
      atomicOr(reinterpret_cast<unsigned*>(b.status), LH_STATUS_COINCIDENT);
      flags |= 4;
    }
    const double tx = __dsub_rn(sx, px), ty = __dsub_rn(sy, py), tz = __dsub_rn(sz, pz);
    const double tn = sqrt(dot3_rn(tx, ty, tz, tx, ty, tz));
    const double cosine = dot3_rn(p.om_look[3 * d], p.om_look[3 * d + 1], p.om_look[3 * d + 2],
                                  tx / tn, ty / tn, tz / tn);
    double pl_prev = 1.0, pl = cosine, acc = 0.0;
    for (int l = 0; l <= p.acc_top; ++l) {
      double P;
      if (l == 0) P = 1.0;
      else if (l == 1) P = cosine;
      else {
        P = ((2 * l - 1) * cosine * pl - (l - 1) * pl_prev) / l;
        pl_prev = pl;
        pl = P;
      }
      acc += p.alpha[l] * (2 * l + 1) * P / (4 * kPi);
    }
    const double four_pi_r2 = 4 * kPi * r * r;
    double upper = 0.0;
    for (int n = 0; n < nd.n_nodes; ++n)
      upper += nd.photons[n][f] * p.om_area[d] * nd.efficiency[n] * acc *
               exp(-nd.absorption[n] * r) / four_pi_r2;
    const bool inside = (r >= p.r_low) && (r <= p.r_high);
    if (!inside && 10 * upper >= p.threshold) {
      flags |= 2;
      atomicOr(reinterpret_cast<unsigned*>(b.status), LH_STATUS_UNSAFE);
      atomicAdd(b.status + 1, 1);
      atomicMax(reinterpret_cast<unsigned long long*>(b.status + 2),
                (unsigned long long)__double_as_longlong(r));
    }
    const double total = (q[0] + q[1]) + q[2];
    const bool active = p.threshold == 0.0 ? inside : (inside && total >= p.threshold);
    b.active[pair] = (uint8_t)((active ? 1 : 0) | flags);
  }
}

size_t flash_tc_smem_bytes(int kpad, int n_tile) {
  return 2ull * (kpad / 8) * kAChunk * 2 + 2ull * n_tile * kpad * 2 +
         2 * sizeof(FlashPair) * kFlashPairs + 64;
}

}  // namespace lh

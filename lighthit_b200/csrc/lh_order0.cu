// Order 0: direct Cherenkov light of spectral elements to the first glass
// entry of each OM sphere, summed over elements, OMs and the continuous
// wavelength spectrum.
//
// Reference: PreparedBallistic (_surface_ballistic.py:20-353) integrates this
// with control variates; its direct form, used there for the geometry the
// control variates cannot invert, is _surface_ballistic_rays.evaluate
// (_surface_ballistic_rays.py:36-156) over the pairs of interval_candidates
// (_ballistic_interval_numba.py:449-519). This file evaluates that direct
// form for every pair at a fixed Gauss order:
//
//   q_d = sum_pairs sum_panels sum_lambda w_l  S(lambda) A / (pi R^2)
//         int ds int dphi/(2 pi) [acc(+) + acc(-)] exp(-mu_t(lambda) d_entry)
//
// with the element's Cherenkov cone at the spectral phase index n(lambda),
// s along the element where the cone meets the sphere, phi the azimuth of the
// cone ray about the element axis and d_entry the distance to the first glass
// entry. Bins split the s and phi ranges at the bin edges (arrival time).
//
// Precision: the pair, wavelength-node and s-node geometry (cone, sphere
// window, arrival times, bin cuts and the bin index) are float64; the
// innermost azimuth quadrature (acceptance, entry distance, attenuation) is
// float32 with the entry distance written without cancellation:
//   d = B / (dot + sqrt(R^2 - |w x k|^2)),  |w x k|^2 = sin^2(th) sin^2(phi) |w|^2
//       + (E0 - along sin(th) 2 sin^2(phi/2))^2,
// E0 = along sin(th) - rho cos(th) formed in float64.
//
// Launch: a candidate pass (one thread per (OM, element), warp-aggregated
// counts per (event, OM)), a scan into per-(event, OM) pair segments and a
// list of 32-pair chunks, a second candidate pass listing the pairs, then a
// persistent grid over the chunks: warp 0 forms each pair's frame, the CTA
// lists the (pair, panel, piece) work, spreads (piece x wavelength node) over
// its threads, accumulates bins in shared memory and the charge by a block
// reduction, and adds both to the outputs once per chunk.
#include <algorithm>

#include "lh_common.cuh"
#include "lh_timing.cuh"

namespace lh {

constexpr int kO0Chunk = 32;
constexpr int kO0Threads = 256;
constexpr int kO0MaxOrder = 64;
constexpr int kO0MaxPanels = 128;
constexpr int kO0MaxSCuts = 64;
constexpr int kO0MaxPhiCuts = 32;
constexpr int kO0MaxAlpha = 8;

struct O0Pair {
  double z, rho, axial, across, side, nmin, nmax, cut0, cut1, tau;
  int el;
};

LH_DEVICE double o0_clamp1(double x) { return x < -1.0 ? -1.0 : (x > 1.0 ? 1.0 : x); }

// _ballistic_interval_numba.py:151-185 (_support): phase-index window of the
// cone rays that meet the sphere, and the two inner cuts.
LH_DEVICE bool o0_support(double z, double rho, double length, double beta, double radius,
                          double& nmin, double& nmax, double& cut0, double& cut1) {
  if (radius == 0.0) {
    if (z <= 0.0) return false;
    nmin = hypot(z, rho) / (beta * z);
    nmax = INFINITY;
    if (z > length) {
      double rz = z - length;
      nmax = hypot(rz, rho) / (beta * rz);
    }
    cut0 = cut1 = INFINITY;
    return true;
  }
  const double quarter = 0.5 * kPi;
  double psi0 = atan2(rho, z), psi1 = atan2(rho, z - length);
  double r0 = radius / hypot(z, rho), r1 = radius / hypot(z - length, rho);
  double a0 = asin(r0 < 1.0 ? r0 : 1.0), a1 = asin(r1 < 1.0 ? r1 : 1.0);
  double low = psi0 - a0, high = psi1 + a1;
  if (low >= quarter) return false;
  double floor_n = (1.0 + 1e-9) / beta;
  if (low <= 0.0) {
    nmin = floor_n;
  } else {
    double v = 1.0 / (beta * cos(low));
    nmin = floor_n > v ? floor_n : v;
  }
  nmax = high >= quarter ? INFINITY : 1.0 / (beta * cos(high));
  double inner0 = psi0 + a0, inner1 = psi1 - a1;
  cut0 = inner0 >= quarter ? INFINITY : 1.0 / (beta * cos(inner0));
  cut1 = (inner1 <= 0.0 || inner1 >= quarter) ? INFINITY : 1.0 / (beta * cos(inner1));
  return true;
}

// _ballistic_interval_numba.py:226-251 (_cone_can_reach_sphere)
LH_DEVICE bool o0_cone_reaches(double z, double rho, double length, double beta, double radius,
                               double pmin, double pmax) {
  if (z <= -radius || beta * pmax <= 1.0) return false;
  double c_hi = 1.0 / (beta * pmax);
  double t = (1.0 - c_hi) * (1.0 + c_hi);
  double s_hi = sqrt(t > 0.0 ? t : 0.0);
  double c_lo = 1.0 / (beta * pmin);
  if (c_lo > 1.0) c_lo = 1.0;
  t = (1.0 - c_lo) * (1.0 + c_lo);
  double s_lo = sqrt(t > 0.0 ? t : 0.0);
  double q_hi = rho * c_hi - z * s_hi;
  double other = rho * c_lo - z * s_lo;
  double minimum = z >= 0.0 ? q_hi : (q_hi < other ? q_hi : other);
  double rounding = 16 * 2.220446049250313e-16 * (fabs(z) + rho + length + radius);
  if (minimum > radius + rounding) return false;
  double end_z = z - length;
  if (end_z >= 0.0 && rho * c_lo - end_z * s_lo < -radius - rounding) return false;
  return true;
}

// _surface_ballistic_rays.py:14-30: real roots of a s^2 + b s + c inside (low, high)
LH_DEVICE int o0_quadratic_cuts(double* cuts, int count, double a, double b, double c, double low,
                                double high) {
  double r[2];
  int nr = 0;
  if (a == 0.0) {
    if (b != 0.0) r[nr++] = -c / b;
  } else {
    double disc = b * b - 4 * a * c;
    if (disc < 0.0) return count;
    double q = -0.5 * (b + copysign(sqrt(disc), b));
    if (q == 0.0) {
      r[nr++] = -b / (2 * a);
    } else {
      r[nr++] = q / a;
      r[nr++] = c / q;
    }
  }
  for (int k = 0; k < nr; ++k)
    if (low < r[k] && r[k] < high) {
      if (count < kO0MaxSCuts) cuts[count] = r[k];
      ++count;
    }
  return count;
}

LH_DEVICE double o0_entry(double B, double dot) {
  double t = dot * dot - B;
  return B / (dot + sqrt(t > 0.0 ? t : 0.0));
}

LH_DEVICE int o0_search_right(const double* e, int n, double x) {
  int lo = 0, hi = n;
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if (e[mid] > x) hi = mid; else lo = mid + 1;
  }
  return lo;
}

LH_DEVICE int o0_search_left(const double* e, int n, double x) {
  int lo = 0, hi = n;
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if (e[mid] >= x) hi = mid; else lo = mid + 1;
  }
  return lo;
}

template <typename T>
LH_DEVICE void o0_sort(T* v, int count) {
  for (int k = 1; k < count; ++k) {
    T value = v[k];
    int m = k - 1;
    while (m >= 0 && v[m] > value) {
      v[m + 1] = v[m];
      --m;
    }
    v[m + 1] = value;
  }
}

// Legendre acceptance sum_l (2l+1) alpha_l P_l(x) / (4 pi), clipped at zero
// (_ballistic_interval_numba.py:21-37); `bad` is raised below -1e-12 max(1, sum|alpha|).
LH_DEVICE float o0_acceptance(const float* alpha, int n_alpha, float x, float alpha_abs,
                              bool& bad) {
  constexpr float inv4pi = 0.0795774715459476679f;
  float result = alpha[0] * inv4pi;
  float previous = 1.0f, current = x;
  if (n_alpha > 1) result += 3.0f * alpha[1] * current * inv4pi;
  for (int ell = 2; ell < n_alpha; ++ell) {
    float value = ((2 * ell - 1) * x * current - (ell - 1) * previous) * (1.0f / ell);
    result += (2 * ell + 1) * alpha[ell] * value * inv4pi;
    previous = current;
    current = value;
  }
  if (result < 0.0f) {
    // float32 rounding of a zero of the polynomial is not a negative response
    if (result < -1e-6f * alpha_abs) bad = true;
    return 0.0f;
  }
  return result;
}


// interval_candidates (_ballistic_interval_numba.py:449-519) with the sphere
// always in reach and the axis included: does element i light OM om at all?
LH_DEVICE bool o0_is_candidate(const lh_order0_optics& O, const lh_order0_batch& B, int om,
                               int64_t i, double pmin, double pmax, uint32_t& flags) {
  const double radius = O.om_radius[om];
  const double beta = B.beta[i], len = B.length[i];
  const double ux = B.direction[3 * i], uy = B.direction[3 * i + 1], uz = B.direction[3 * i + 2];
  const double wx = O.om_pos[3 * om] - B.start[3 * i], wy = O.om_pos[3 * om + 1] - B.start[3 * i + 1],
               wz = O.om_pos[3 * om + 2] - B.start[3 * i + 2];
  const double z = wx * ux + wy * uy + wz * uz;
  const bool sphere = radius > 0.0;
  if (B.c0[i] == 0.0 || beta * pmax <= 1.0 || (z <= 0.0 && (!sphere || z <= -radius))) return false;
  const double cx = wy * uz - wz * uy, cy = wz * ux - wx * uz, cz = wx * uy - wy * ux;
  const double rho_c = sqrt(cx * cx + cy * cy + cz * cz);
  const double rad = sphere ? radius : 0.0;
  if (z <= 0.0 && rad == 0.0) return false;
  if (rho_c == 0.0) {
    if (rad == 0.0) {
      if (0.0 < z && z < len) flags |= LH_STATUS_ON_TRACK;
      return false;
    }
    return true;
  }
  if (rad == 0.0) return false;  // a point receiver has no first-entry window: no light here
  if (!o0_cone_reaches(z, rho_c, len, beta, rad, pmin, pmax)) return false;
  double a, b, c, d;
  return o0_support(z, rho_c, len, beta, rad, a, b, c, d) && !(a > pmax || b <= pmin);
}

LH_DEVICE void o0_phase_range(const lh_order0_optics& O, double& pmin, double& pmax) {
  pmin = O.phase[0];
  pmax = O.phase[0];
  for (int k = 1; k < O.n_panel_edges; ++k) {
    pmin = fmin(pmin, O.phase[k]);
    pmax = fmax(pmax, O.phase[k]);
  }
}

LH_DEVICE int o0_event_of(const lh_order0_batch& B, int64_t i) {
  int lo = 0, hi = B.n_events;  // last event with element_offset[ev] <= i
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (B.element_offset[mid] <= i) lo = mid; else hi = mid;
  }
  return lo;
}

struct O0Work {
  int32_t* counts;    // [n_events * n_om] candidate pairs
  int32_t* offsets;   // [n_events * n_om] first pair of each (event, OM)
  int32_t* cursor;    // [n_events * n_om]
  int32_t* pairs;     // [pair capacity] global element index
  int2* chunks;       // [chunk capacity] (event * n_om + om, chunk)
  uint32_t* mask;     // [pair capacity / 32] candidate bits of the counting pass
  int32_t* n_chunks;  // [2]: the chunk count, then the next chunk to take
  int64_t pair_capacity, chunk_capacity;
};

// Candidate pairs counted (fill = false) or listed (fill = true) per (event, OM):
// one thread per (OM, element); a warp's elements are consecutive, so the
// lanes of one (event, OM) add their count once (warp-aggregated atomics). The
// counting pass keeps each warp's candidate mask, which the listing pass reads
// instead of testing the pair again.
template <bool fill>
__global__ void order0_candidates_kernel(const lh_order0_optics O, const lh_order0_batch B,
                                         O0Work W) {
  double pmin, pmax;
  o0_phase_range(O, pmin, pmax);
  const int64_t n_el = B.n_elements;
  const int64_t total = n_el * O.n_om;
  uint32_t flags = 0;
  for (int64_t base = (int64_t)blockIdx.x * blockDim.x; base < total;
       base += (int64_t)gridDim.x * blockDim.x) {
    const int64_t item = base + threadIdx.x;
    const int64_t word = item >> 5;  // blockDim and base are multiples of 32
    bool keep = false;
    int key = -1;
    int64_t i = 0;
    if (item < total) {
      const int om = (int)(item / n_el);
      i = item - (int64_t)om * n_el;
      keep = fill ? ((W.mask[word] >> (threadIdx.x & 31)) & 1u)
                  : o0_is_candidate(O, B, om, i, pmin, pmax, flags);
      if (keep) key = o0_event_of(B, i) * O.n_om + om;
    }
    const unsigned active = __ballot_sync(0xffffffffu, keep);
    if (!fill && (threadIdx.x & 31) == 0 && item < total) W.mask[word] = active;
    if (keep) {
      const unsigned peers = __match_any_sync(active, key);
      const int leader = __ffs(peers) - 1;
      const int lane = threadIdx.x & 31;
      const int rank = __popc(peers & ((1u << lane) - 1u));
      int first = 0;
      if (lane == leader) first = atomicAdd(fill ? W.cursor + key : W.counts + key, __popc(peers));
      first = __shfl_sync(peers, first, leader);
      if (fill && first + rank < W.pair_capacity) W.pairs[first + rank] = (int32_t)i;
    }
  }
  if (!fill && flags) atomicOr(reinterpret_cast<unsigned*>(B.status), flags);
}

// Single CTA: pair offsets per (event, OM) and the list of 32-pair chunks.
__global__ void __launch_bounds__(1024) order0_scan_kernel(int32_t n_keys, O0Work W) {
  __shared__ int32_t warp_sum[32], warp_chunks[32];
  __shared__ int32_t carry, carry_chunks;
  if (threadIdx.x == 0) {
    carry = 0;
    carry_chunks = 0;
  }
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int base = 0; base < n_keys; base += blockDim.x) {
    const int key = base + threadIdx.x;
    const int32_t c = key < n_keys ? W.counts[key] : 0;
    const int32_t ch = (c + kO0Chunk - 1) / kO0Chunk;
    int32_t v = c, h = ch;
    for (int off = 1; off < 32; off <<= 1) {
      const int32_t a = __shfl_up_sync(0xffffffffu, v, off);
      const int32_t b = __shfl_up_sync(0xffffffffu, h, off);
      if (lane >= off) {
        v += a;
        h += b;
      }
    }
    if (lane == 31) {
      warp_sum[warp] = v;
      warp_chunks[warp] = h;
    }
    __syncthreads();
    if (warp == 0) {
      int32_t sv = lane < (int)(blockDim.x >> 5) ? warp_sum[lane] : 0;
      int32_t sh = lane < (int)(blockDim.x >> 5) ? warp_chunks[lane] : 0;
      for (int off = 1; off < 32; off <<= 1) {
        const int32_t a = __shfl_up_sync(0xffffffffu, sv, off);
        const int32_t b = __shfl_up_sync(0xffffffffu, sh, off);
        if (lane >= off) {
          sv += a;
          sh += b;
        }
      }
      warp_sum[lane] = sv;
      warp_chunks[lane] = sh;
    }
    __syncthreads();
    const int32_t before = (warp ? warp_sum[warp - 1] : 0) + v - c + carry;
    const int32_t before_ch = (warp ? warp_chunks[warp - 1] : 0) + h - ch + carry_chunks;
    if (key < n_keys) {
      W.offsets[key] = before;
      W.cursor[key] = before;
      for (int j = 0; j < ch; ++j)
        if (before_ch + j < W.chunk_capacity) W.chunks[before_ch + j] = make_int2(key, j);
    }
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) {
      carry = before + c;
      carry_chunks = before_ch + ch;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    W.n_chunks[0] = carry_chunks;
    W.n_chunks[1] = 0;
  }
}

// One Gauss rule: nodes, weights and the s-node map sin/cos(pi/2 x).
struct O0Rule {
  double x[kO0MaxOrder], w[kO0MaxOrder];
  double sin_psi[kO0MaxOrder], cos_psi[kO0MaxOrder];
};

// A (piece, wavelength node) item as its s-nodes read it.
struct O0Item {
  double cosine, sine, velocity, scale, t0;
  float absorption;
  int code;  // pair | 0x100 for the check rule
};

constexpr int kO0CutPool = 1536;  // s cuts staged per batch of items

struct O0Shared {
  O0Rule rule[2];  // the quadrature order and the lower check order
  float alpha[kO0MaxAlpha];
  O0Pair pair[kO0Chunk];
  O0Item item[kO0Threads];   // the batch's items, one per thread
  int unit_end[kO0Threads];  // inclusive prefix of the items' s-node counts
  int cut_at[kO0Threads];    // each item's first s cut in `cuts`
  double cuts[kO0CutPool];
  double warp_charge[kO0Threads / 32];
  double warp_check[kO0Threads / 32];
  double bin_stage[kO0Threads / 32][32];  // per warp: the lanes' bin values before one add per bin
  int scan[32];
  int chunk;
  int n_pairs;
  int n_combos;
};

// Exclusive prefix sum of `v` over the CTA (blockDim a multiple of 32, at most
// 1024) through `warp_sums` (32 ints of shared memory); `total` gets the sum.
LH_DEVICE int o0_block_scan(int v, int& total, int* warp_sums) {
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

__global__ void __launch_bounds__(kO0Threads, 4)
order0_kernel(const lh_order0_optics O, const lh_order0_batch B, const O0Work W,
              unsigned long long* units) {
  extern __shared__ __align__(16) unsigned char o0_smem[];
  O0Shared& S = *reinterpret_cast<O0Shared*>(o0_smem);
  const int n_panels = O.n_panel_edges - 1;
  const int nb = B.n_edges - 1;
  const bool want_bins = B.bins != nullptr;
  double* sbins = reinterpret_cast<double*>(o0_smem + sizeof(O0Shared));
  uint32_t* combos = reinterpret_cast<uint32_t*>(sbins + (want_bins ? nb : 0));
  const int tid = threadIdx.x;
  const int order = O.order;
  // the check rule's items follow the main rule's in each (pair, panel, piece)
  const int check = (B.charge_check && O.check_order > 0) ? O.check_order : 0;
  const int rules = order + check;
  for (int k = tid; k < order; k += blockDim.x) {
    S.rule[0].x[k] = O.gauss_x[k];
    S.rule[0].w[k] = O.gauss_w[k];
    sincospi(0.5 * O.gauss_x[k], &S.rule[0].sin_psi[k], &S.rule[0].cos_psi[k]);
  }
  for (int k = tid; k < check; k += blockDim.x) {
    S.rule[1].x[k] = O.check_x[k];
    S.rule[1].w[k] = O.check_w[k];
    sincospi(0.5 * O.check_x[k], &S.rule[1].sin_psi[k], &S.rule[1].cos_psi[k]);
  }
  for (int k = tid; k < O.n_alpha; k += blockDim.x) S.alpha[k] = (float)O.alpha[k];
  double pmin, pmax;
  o0_phase_range(O, pmin, pmax);
  const int total_chunks = min(*W.n_chunks, (int)W.chunk_capacity);
  unsigned long long evaluations = 0;  // float32 integrand nodes of this thread
  // CTAs take chunks from a counter: one that drew a heavy chunk does not
  // hold back the chunks dealt to it after
  for (;;) {
  __syncthreads();
  if (tid == 0) S.chunk = atomicAdd(W.n_chunks + 1, 1);
  __syncthreads();
  const int chunk = S.chunk;
  if (chunk >= total_chunks) break;
  const int2 entry = W.chunks[chunk];
  const int ev = entry.x / O.n_om;
  const int om = entry.x - ev * O.n_om;
  const int p_begin = W.offsets[entry.x] + entry.y * kO0Chunk;
  const int p_end = min(W.offsets[entry.x] + W.counts[entry.x], p_begin + kO0Chunk);
  if (want_bins)
    for (int k = tid; k < nb; k += blockDim.x) sbins[k] = 0.0;
  if (tid == 0) S.n_combos = 0;
  const double ox = O.om_pos[3 * om], oy = O.om_pos[3 * om + 1], oz = O.om_pos[3 * om + 2];
  const double radius = O.om_radius[om];
  uint32_t flags = 0;

  // ---- phase 0: the chunk's candidate pairs (warp 0) and their frames
  if (tid < 32) {
    const int pi = p_begin + tid;
    bool keep = false;
    O0Pair P{};
    if (pi < p_end && pi < W.pair_capacity) {
      const int64_t i = W.pairs[pi];
      const double beta = B.beta[i], len = B.length[i];
      const double ux = B.direction[3 * i], uy = B.direction[3 * i + 1], uz = B.direction[3 * i + 2];
      const double wx = ox - B.start[3 * i], wy = oy - B.start[3 * i + 1], wz = oz - B.start[3 * i + 2];
      const double z = wx * ux + wy * uy + wz * uz;
      keep = true;
      if (keep) {
        // _surface_ballistic_rays.py:52-80: frame and support of the pair
        const double tx = wx - z * ux, ty = wy - z * uy, tz = wz - z * uz;
        const double rho = sqrt(tx * tx + ty * ty + tz * tz);
        double nmin, nmax, cut0, cut1;
        if (!o0_support(z, rho, len, beta, radius, nmin, nmax, cut0, cut1) || nmin > pmax ||
            nmax <= pmin) {
          keep = false;
        } else {
          const double along_min = z < 0.0 ? z : (z > len ? z - len : 0.0);
          if (rho * rho + along_min * along_min <= radius * radius) {
            flags |= LH_STATUS_INSIDE_GLASS;
            keep = false;
          } else {
            double e1x, e1y, e1z;
            if (rho > 0.0) {
              e1x = tx / rho; e1y = ty / rho; e1z = tz / rho;
            } else {
              double ax = 0, ay = 0, az = 0;
              if (fabs(ux) < 0.9) ax = 1.0; else ay = 1.0;
              e1x = uy * az - uz * ay; e1y = uz * ax - ux * az; e1z = ux * ay - uy * ax;
              double nn = sqrt(e1x * e1x + e1y * e1y + e1z * e1z);
              e1x /= nn; e1y /= nn; e1z /= nn;
            }
            const double e2x = uy * e1z - uz * e1y, e2y = uz * e1x - ux * e1z,
                         e2z = ux * e1y - uy * e1x;
            const double lx = O.om_look[3 * om], ly = O.om_look[3 * om + 1], lz = O.om_look[3 * om + 2];
            P.z = z; P.rho = rho;
            P.axial = ux * lx + uy * ly + uz * lz;
            P.across = e1x * lx + e1y * ly + e1z * lz;
            P.side = e2x * lx + e2y * ly + e2z * lz;
            P.nmin = nmin; P.nmax = nmax; P.cut0 = cut0; P.cut1 = cut1;
            P.tau = (B.t1[i] - B.t0[i]) / len;
            P.el = (int)i;
          }
        }
      }
    }
    const unsigned mask = __ballot_sync(0xffffffffu, keep);
    if (keep) S.pair[__popc(mask & ((1u << tid) - 1u))] = P;
    if (tid == 0) S.n_pairs = __popc(mask);
  }
  __syncthreads();
  const int n_pairs = S.n_pairs;
  if (n_pairs == 0) {
    if (flags) atomicOr(reinterpret_cast<unsigned*>(B.status), flags);
    continue;
  }

  // ---- phase 1: (pair, panel, piece) work list
  for (int item = tid; item < n_pairs * n_panels; item += blockDim.x) {
    const int p = item / n_panels, panel = item - p * n_panels;
    const O0Pair& P = S.pair[p];
    const double left = O.panel_edges[panel], width = O.panel_edges[panel + 1] - left;
    const double n0 = O.phase[panel], dn = O.phase[panel + 1] - n0;
    double a = left, b = left + width;
    if (dn == 0.0) {
      if (n0 < P.nmin || n0 >= P.nmax) continue;
    } else {
      double x0 = (P.nmin - n0) / dn, x1 = (P.nmax - n0) / dn;
      double l = fmin(x0, x1), h = fmax(x0, x1);
      a = left + width * fmax(l, 0.0);
      b = left + width * fmin(h, 1.0);
    }
    if (a >= b) continue;
    int pieces = 1;
    if (dn != 0.0) {
      double vals[2] = {P.cut0, P.cut1};
      for (int v = 0; v < 2; ++v)
        if (isfinite(vals[v])) {
          double lam = left + width * (vals[v] - n0) / dn;
          if (a < lam && lam < b) ++pieces;
        }
    }
    const int slot = atomicAdd(&S.n_combos, pieces);
    for (int k = 0; k < pieces; ++k)
      combos[slot + k] = (uint32_t)p | ((uint32_t)panel << 8) | ((uint32_t)k << 24);
  }
  __syncthreads();
  const int n_combos = S.n_combos;

  // ---- phase 2: (piece, wavelength node) items in batches of one per thread.
  // Each thread sets up its item (cone of the wavelength node, s window, the s
  // cuts at the bin-edge crossings) and stages it; the batch's s-nodes (s piece
  // x Gauss node) are then spread evenly over the CTA, so that lanes no longer
  // wait on a neighbour whose item has more s pieces or none at all.
  const double area_scale = O.om_area[om] / (kPi * radius * radius);
  const double origin = B.origins[(int64_t)ev * O.n_om + om];
  const double* edges = B.edges;
  const int n_edges = B.n_edges;
  float alpha_abs = 0.0f;
  for (int k = 0; k < O.n_alpha; ++k) alpha_abs += fabsf(S.alpha[k]);
  alpha_abs = fmaxf(alpha_abs, 1.0f);
  bool bad_acceptance = false;
  double charge = 0.0, charge_check = 0.0;
  double scuts[kO0MaxSCuts];
  double phicuts[kO0MaxPhiCuts];

  // main-rule items first, then the check rule's: a warp's items share a rule
  const int main_items = n_combos * order;
  const int n_items = n_combos * rules;
  for (int first = 0; first < n_items;) {  // the same on every thread
    const int item = first + tid;
    int ns = 0, units = 0;
    O0Item it{};
    if (item < n_items) {
      int ci, r_item;
      if (item < main_items) {
        ci = item / order;
        r_item = item - ci * order;
      } else {
        const int rest = item - main_items;
        ci = rest / check;
        r_item = order + (rest - ci * check);
      }
      const bool is_check = r_item >= order;
      const int ilam = is_check ? r_item - order : r_item;
      const O0Rule& R = S.rule[is_check ? 1 : 0];
      const uint32_t code = combos[ci];
      const int p = code & 0xff, panel = (code >> 8) & 0xffff, piece = code >> 24;
      const O0Pair& P = S.pair[p];
      const int64_t i = P.el;
      const double left = O.panel_edges[panel], width = O.panel_edges[panel + 1] - left;
      const double n0 = O.phase[panel], dn = O.phase[panel + 1] - n0;
      double cuts[4];
      int count = 2;
      if (dn == 0.0) {
        cuts[0] = left; cuts[1] = left + width;
      } else {
        double x0 = (P.nmin - n0) / dn, x1 = (P.nmax - n0) / dn;
        cuts[0] = left + width * fmax(fmin(x0, x1), 0.0);
        cuts[1] = left + width * fmin(fmax(x0, x1), 1.0);
        double vals[2] = {P.cut0, P.cut1};
        const double lo_c = cuts[0], hi_c = cuts[1];
        for (int v = 0; v < 2; ++v)
          if (isfinite(vals[v])) {
            double lam = left + width * (vals[v] - n0) / dn;
            if (lo_c < lam && lam < hi_c) cuts[count++] = lam;
          }
        o0_sort(cuts, count);
      }
      const double low = cuts[piece], high = cuts[piece + 1];
      const double beta = B.beta[i], L = B.length[i];
      const double lam = (low + high) / 2 + (high - low) / 2 * R.x[ilam];
      const double q = (lam - left) / width, n = n0 + dn * q, bn = beta * n;
      const double cosine = 1 / bn, sine = bn > 1.0 ? sqrt(1 - cosine * cosine) : 0.0;
      const double z = P.z, rho = P.rho;
      const double centre = z - rho * cosine / sine, spread = radius / sine;
      const double slo = fmax(centre - spread, 0.0), shi = fmin(centre + spread, L);
      if (bn > 1.0 && slo < shi) {
        const double absorption =
            O.extinction[panel] + q * (O.extinction[panel + 1] - O.extinction[panel]);
        const double group = O.group[panel] + q * (O.group[panel + 1] - O.group[panel]);
        const double velocity = kCVacuumMPerNs / group;
        const double* ef = O.efficiency + (int64_t)panel * O.eff_cols;
        double eta = ((ef[3] * q + ef[2]) * q + ef[1]) * q + ef[0];
        if (O.eff_cols > 4) eta *= exp(ef[4] + q * ef[5]);
        const double spectral = (B.c0[i] + B.c2[i] / (n * n)) / L / (lam * lam) * eta;
        const double t0 = B.t0[i], tau = P.tau;
        it.cosine = cosine;
        it.sine = sine;
        it.velocity = velocity;
        it.scale = (high - low) / 2 * R.w[ilam] * spectral * area_scale;
        it.t0 = t0;
        it.absorption = (float)absorption;
        it.code = p | (is_check ? 0x100 : 0);

        // s cuts where a cone ray's entry time crosses a bin edge
        // (_surface_ballistic_rays.py:96-118)
        scuts[0] = slo;
        scuts[1] = shi;
        ns = 2;
        const double d0 = (z - slo) * (z - slo), d1 = (z - shi) * (z - shi);
        const double rmax = sqrt(rho * rho + fmax(d0, d1));
        const double rmin = sqrt(rho * rho + ((slo < z && z < shi) ? 0.0 : fmin(d0, d1)));
        const double e_lo = t0 + tau * slo, e_hi = t0 + tau * shi;
        const double earliest = fmin(e_lo, e_hi) + (rmin - radius) / velocity - origin;
        const double latest = fmax(e_lo, e_hi) + rmax / velocity - origin;
        const int first_edge = o0_search_right(edges, n_edges, earliest);
        const int last_edge = o0_search_left(edges, n_edges, latest);
        for (int edge = first_edge; edge < last_edge; ++edge) {
          const double A = (origin + edges[edge] - t0) * velocity, Bv = tau * velocity;
          for (int sgn = -1; sgn <= 1; sgn += 2) {
            const double D = cosine * z + sgn * sine * rho;
            ns = o0_quadratic_cuts(scuts, ns, 1 + Bv * Bv - 2 * Bv * cosine,
                                   -2 * z - 2 * A * Bv + 2 * (A * cosine + Bv * D),
                                   z * z + rho * rho - radius * radius + A * A - 2 * A * D, slo,
                                   shi);
          }
          ns = o0_quadratic_cuts(scuts, ns, Bv * Bv - 1., -2 * A * Bv + 2 * z,
                                 A * A - z * z - rho * rho + radius * radius, slo, shi);
        }
        if (ns > kO0MaxSCuts) {
          flags |= LH_STATUS_OVERFLOW;
          ns = 0;
        } else {
          o0_sort(scuts, ns);
          units = (ns - 1) * (is_check ? check : order);
        }
      }
    }
    // stage the cuts; the threads whose cuts do not fit the pool (a suffix of
    // the CTA: the offsets only grow) set their items up again next batch
    int cut_total;
    const int cut_at = o0_block_scan(ns, cut_total, S.scan);
    const bool fits = cut_at + ns <= kO0CutPool;
    const int taken = __syncthreads_count(fits);  // at least thread 0's (ns <= kO0MaxSCuts)
    if (!fits) units = 0;
    else
      for (int k = 0; k < ns; ++k) S.cuts[cut_at + k] = scuts[k];
    int unit_total;
    const int unit_at = o0_block_scan(units, unit_total, S.scan);
    S.unit_end[tid] = unit_at + units;
    S.cut_at[tid] = cut_at;
    S.item[tid] = it;
    __syncthreads();

    // the batch's s-nodes, consecutive ones (one item's) on neighbouring lanes
    const float R2 = (float)(radius * radius);
    for (int u = tid; u < unit_total; u += blockDim.x) {
      int owner = 0;  // the first thread whose s-nodes end past u
      for (int hi = blockDim.x - 1; owner < hi;) {
        const int mid = (owner + hi) >> 1;
        if (S.unit_end[mid] > u) hi = mid; else owner = mid + 1;
      }
      const O0Item& c = S.item[owner];
      const bool is_check = c.code >> 8;
      const int ord = is_check ? check : order;
      const O0Rule& R = S.rule[is_check ? 1 : 0];
      const O0Pair& P = S.pair[c.code & 0xff];
      const int local = u - (owner ? S.unit_end[owner - 1] : 0);
      const int sp = local / ord, j = local - sp * ord;
      const double sa = S.cuts[S.cut_at[owner] + sp], sb = S.cuts[S.cut_at[owner] + sp + 1];
      if (sa >= sb) continue;
      const double cosine = c.cosine, sine = c.sine, velocity = c.velocity;
      const double z = P.z, rho = P.rho, t0 = c.t0, tau = P.tau;
      const float cos_f = (float)cosine, sin_f = (float)sine;
      const float axial = (float)P.axial, across = (float)P.across, side = (float)P.side;
      const float absorption_f = c.absorption;
      const double sin_psi = R.sin_psi[j], cos_psi = R.cos_psi[j];
      const double s = (sa + sb) / 2 + (sb - sa) / 2 * sin_psi;
      const double ds = (sb - sa) / 2 * cos_psi * kPi / 2 * R.w[j];
      const double along = z - s, W2 = rho * rho + along * along, Bq = W2 - radius * radius;
      double half, cos_half = 1.0;  // cos(half): the clamped argument itself (rho > 0)
      if (rho > 0.0) {
        cos_half = o0_clamp1((sqrt(Bq) - cosine * along) / (sine * rho));
        half = acos(cos_half);
      } else {
        half = cosine * along >= sqrt(Bq) ? kPi : 0.0;
      }
      if (half == 0.0) continue;
      const double emission = t0 + tau * s - origin;
      const double tmin = emission + o0_entry(Bq, cosine * along + sine * rho) / velocity;
      const double tmax = emission + o0_entry(Bq, cosine * along + sine * rho * cos_half) / velocity;
      phicuts[0] = 0.0;
      int nphi = 1;
      if (rho > 0.0) {
        const int first_cut = o0_search_right(edges, n_edges, tmin);
        const int last_cut = o0_search_left(edges, n_edges, tmax);
        for (int edge = first_cut; edge < last_cut; ++edge) {
          const double distance = (edges[edge] - emission) * velocity;
          const double dot = (Bq + distance * distance) / (2 * distance);
          const double phi = acos(o0_clamp1((dot - cosine * along) / (sine * rho)));
          const double r = phi / half;
          if (nphi < kO0MaxPhiCuts - 1) phicuts[nphi] = asin(r < 1.0 ? r : 1.0);
          ++nphi;
        }
      }
      if (nphi > kO0MaxPhiCuts - 1) {
        flags |= LH_STATUS_OVERFLOW;
        continue;
      }
      phicuts[nphi++] = kPi / 2;
      // float32 azimuth integrand, entry distance without cancellation
      const float half_f = (float)half;
      const float W2_f = (float)W2, B_f = (float)Bq;
      const float E0 = (float)(along * sine - rho * cosine);
      const float Sa = (float)(along * sine);
      const float along_cos = (float)(cosine * along), rho_sin = (float)(sine * rho);
      const float sin2W2 = sin_f * sin_f * W2_f;
      for (int pp = 0; pp < nphi - 1; ++pp) {
        const double pa = phicuts[pp], pb = phicuts[pp + 1];
        if (pa >= pb) continue;
        const float mid = (float)((pa + pb) / 2), hw = (float)((pb - pa) / 2);
        evaluations += ord;
        float integral = 0.0f;
        for (int jp = 0; jp < ord; ++jp) {
          // arguments lie in [0, pi]: the hardware approximations (absolute error
          // near 2^-21) are well inside the float32 integrand's budget
          float s_eta, c_eta;
          __sincosf(mid + hw * (float)R.x[jp], &s_eta, &c_eta);
          const float phi = half_f * s_eta;
          const float dphi = half_f * c_eta * hw * (float)R.w[jp];
          // sin(phi), cos(phi) from the half angle: 2 sin^2(phi/2) = 1 - cos(phi)
          // without cancellation near phi = 0
          float sh, chh;
          __sincosf(0.5f * phi, &sh, &chh);
          const float ss = 2.0f * sh * chh, cp = 1.0f - 2.0f * sh * sh;
          const float E = E0 - Sa * (2.0f * sh * sh);
          const float D = R2 - (sin2W2 * ss * ss + E * E);
          const float dot = along_cos + rho_sin * cp;
          const float distance = __fdividef(B_f, dot + sqrtf(fmaxf(D, 0.0f)));
          const float x1 = cos_f * axial + sin_f * (cp * across + ss * side);
          const float x2 = cos_f * axial + sin_f * (cp * across - ss * side);
          const float accept = o0_acceptance(S.alpha, O.n_alpha, x1, alpha_abs, bad_acceptance) +
                               o0_acceptance(S.alpha, O.n_alpha, x2, alpha_abs, bad_acceptance);
          integral += dphi * accept * __expf(-absorption_f * distance);
        }
        const double value = c.scale * ds * (double)integral * (1.0 / (2 * kPi));
        if (is_check) {  // the check rule: charge only
          charge_check += value;
          continue;
        }
        charge += value;
        if (want_bins) {
          const double phi_mid = half * sin((pa + pb) / 2);
          const double arrival =
              emission + o0_entry(Bq, cosine * along + sine * rho * cos(phi_mid)) / velocity;
          const int slot = o0_search_right(edges, n_edges, arrival) - 1;
          // the lanes here together that land in one bin (neighbouring s-nodes
          // of one item, mostly) add their sum once: one shared-memory atomic
          // per bin and warp instead of one per lane
          const int key = (slot >= 0 && slot < nb) ? slot : -1;
          const unsigned here = __activemask();
          const unsigned peers = __match_any_sync(here, key);
          const int lane = tid & 31;
          double* stage = S.bin_stage[tid >> 5];
          stage[lane] = value;
          __syncwarp(here);
          if (key >= 0 && lane == __ffs(peers) - 1) {
            double sum = 0.0;
            for (unsigned m = peers; m; m &= m - 1) sum += stage[__ffs(m) - 1];
            atomicAdd(&sbins[key], sum);
          }
          __syncwarp(here);  // the stage is rewritten by the next piece
        }
      }
    }
    first += taken;
    __syncthreads();  // the batch's staging is read before the next batch writes it
  }
  if (bad_acceptance) flags |= LH_STATUS_NEGATIVE_ACCEPTANCE;

  // ---- charge: warp shuffles, then one add per CTA; bins: one add per nonzero bin
  for (int off = 16; off > 0; off >>= 1) {
    charge += __shfl_xor_sync(0xffffffffu, charge, off);
    charge_check += __shfl_xor_sync(0xffffffffu, charge_check, off);
  }
  if ((tid & 31) == 0) {
    S.warp_charge[tid >> 5] = charge;
    S.warp_check[tid >> 5] = charge_check;
  }
  __syncthreads();
  if (tid == 0) {
    double total = 0.0, total_check = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
      total += S.warp_charge[w];
      total_check += S.warp_check[w];
    }
    if (total != 0.0) atomicAdd(&B.charge[(int64_t)ev * O.n_om + om], total);
    if (check && total_check != 0.0)
      atomicAdd(&B.charge_check[(int64_t)ev * O.n_om + om], total_check);
  }
  if (want_bins) {
    double* out = B.bins + ((int64_t)ev * O.n_om + om) * nb;
    for (int k = tid; k < nb; k += blockDim.x)
      if (sbins[k] != 0.0) atomicAdd(&out[k], sbins[k]);
  }
  if (flags) atomicOr(reinterpret_cast<unsigned*>(B.status), flags);
  }  // chunks
  if (units) {
    for (int off = 16; off > 0; off >>= 1)
      evaluations += __shfl_xor_sync(0xffffffffu, evaluations, off);
    if ((tid & 31) == 0 && evaluations) atomicAdd(units, evaluations);
  }
}

size_t order0_shared_bytes(const lh_order0_optics& O, const lh_order0_batch& B) {
  const int n_panels = O.n_panel_edges - 1;
  size_t bytes = sizeof(O0Shared);
  if (B.bins) bytes += sizeof(double) * (size_t)(B.n_edges - 1);
  bytes += sizeof(uint32_t) * (size_t)kO0Chunk * n_panels * 3;
  return bytes;
}

static size_t o0_align(size_t x) { return (x + 255) & ~(size_t)255; }

// Workspace: per (event, OM) counts, offsets, cursors; the pair list (at most
// every (OM, element) combination) and the chunk list.
static O0Work o0_layout(const lh_order0_optics& O, const lh_order0_batch& B, unsigned char* base,
                        size_t* bytes) {
  O0Work W{};
  const int64_t keys = (int64_t)B.n_events * O.n_om;
  W.pair_capacity = B.n_elements * O.n_om;
  W.chunk_capacity = W.pair_capacity / kO0Chunk + keys;
  size_t off = 0;
  auto take = [&](size_t n) {
    unsigned char* p = base ? base + off : nullptr;
    off += o0_align(n);
    return p;
  };
  W.counts = reinterpret_cast<int32_t*>(take(sizeof(int32_t) * keys));
  W.offsets = reinterpret_cast<int32_t*>(take(sizeof(int32_t) * keys));
  W.cursor = reinterpret_cast<int32_t*>(take(sizeof(int32_t) * keys));
  W.pairs = reinterpret_cast<int32_t*>(take(sizeof(int32_t) * W.pair_capacity));
  W.chunks = reinterpret_cast<int2*>(take(sizeof(int2) * W.chunk_capacity));
  W.mask = reinterpret_cast<uint32_t*>(take(sizeof(uint32_t) * ((W.pair_capacity + 31) / 32)));
  W.n_chunks = reinterpret_cast<int32_t*>(take(sizeof(int32_t) * 4));
  if (bytes) *bytes = off;
  return W;
}

int order0_launch(const lh_order0_optics& O, const lh_order0_batch& B, cudaStream_t s) {
  const size_t smem = order0_shared_bytes(O, B);
  if (smem > 200 * 1024) return LH_EUNSUPPORTED;
  size_t need = 0;
  O0Work W = o0_layout(O, B, static_cast<unsigned char*>(B.workspace), &need);
  if (!B.workspace || B.workspace_bytes < need) return LH_ENOMEM;
  if (cudaFuncSetAttribute(order0_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)smem) != cudaSuccess)
    return LH_ECUDA;
  const int64_t keys = (int64_t)B.n_events * O.n_om;
  cudaMemsetAsync(B.charge, 0, sizeof(double) * (size_t)keys, s);
  if (B.charge_check && O.check_order > 0)
    cudaMemsetAsync(B.charge_check, 0, sizeof(double) * (size_t)keys, s);
  if (B.bins) cudaMemsetAsync(B.bins, 0, sizeof(double) * (size_t)keys * (B.n_edges - 1), s);
  if (B.n_elements == 0) return cudaGetLastError() == cudaSuccess ? LH_OK : LH_ECUDA;
  cudaMemsetAsync(W.counts, 0, sizeof(int32_t) * keys, s);
  const int64_t items = B.n_elements * O.n_om;
  const int blocks = (int)std::min<int64_t>((items + 255) / 256, 148 * 16);
  order0_candidates_kernel<false><<<blocks, 256, 0, s>>>(O, B, W);
  order0_scan_kernel<<<1, 1024, 0, s>>>((int32_t)keys, W);
  order0_candidates_kernel<true><<<blocks, 256, 0, s>>>(O, B, W);
  {
    lh::TimedLaunch timed_launch(LH_KT_ORDER0, s);
    order0_kernel<<<148 * 8, kO0Threads, smem, s>>>(
        O, B, W, lh::kernel_units() ? lh::kernel_units() + LH_KT_ORDER0 : nullptr);
  }
  return cudaGetLastError() == cudaSuccess ? LH_OK : LH_ECUDA;
}

bool order0_valid(const lh_order0_optics* O, const lh_order0_batch* B) {
  if (!O || !B) return false;
  if (O->n_om < 1 || O->n_om > 65535 || !O->om_pos || !O->om_look || !O->om_area || !O->om_radius)
    return false;
  if (O->n_alpha < 1 || O->n_alpha > kO0MaxAlpha || !O->alpha) return false;
  if (O->n_panel_edges < 2 || O->n_panel_edges - 1 > kO0MaxPanels || !O->panel_edges ||
      !O->phase || !O->group || !O->extinction || !O->efficiency)
    return false;
  if (O->eff_cols != 4 && O->eff_cols != 6) return false;
  if (O->order < 1 || O->order > kO0MaxOrder || !O->gauss_x || !O->gauss_w) return false;
  if (O->check_order < 0 || O->check_order >= O->order ||
      (O->check_order > 0 && (!O->check_x || !O->check_w)))
    return false;
  if (B->n_events < 1 || !B->element_offset || B->n_elements < 0) return false;
  // pair indices, counts and offsets are 32-bit
  if (B->n_elements * (int64_t)O->n_om >= (1ll << 31)) return false;
  if ((int64_t)B->n_events * O->n_om >= (1ll << 31)) return false;
  if (B->n_edges < 2 || !B->edges || !B->origins || !B->charge || !B->status) return false;
  if (B->n_elements && (!B->start || !B->direction || !B->length || !B->c0 || !B->c2 ||
                        !B->beta || !B->t0 || !B->t1))
    return false;
  return true;
}

}  // namespace lh

extern "C" size_t lh_order0_workspace_bytes(const lh_order0_optics* optics,
                                            const lh_order0_batch* batch) {
  if (!lh::order0_valid(optics, batch)) return 0;
  size_t need = 0;
  lh::o0_layout(*optics, *batch, nullptr, &need);
  return need;
}

extern "C" int lh_order0(const lh_order0_optics* optics, const lh_order0_batch* batch,
                         void* stream) {
  if (!lh::order0_valid(optics, batch)) return LH_EINVAL;
  return lh::order0_launch(*optics, *batch, static_cast<cudaStream_t>(stream));
}

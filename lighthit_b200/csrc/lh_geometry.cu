// Per-OM geometry of an element set, float64 and bit-identical to the
// reference's NumPy/Numba arithmetic (no fused multiply-adds):
//   min_distance_to_segments (_prompt_numba.py:2221-2243): distance from each
//     OM to the nearest point of any element (module selection, prompt.py:603-631);
//   earliest_element_arrival (_shower_basis.py:50-78): the per-OM clock of an
//     extended source, min over elements of start_ns + n_g/c |OM - segment|.
// One CTA per (OM, event); threads stride over the event's elements and the
// minima are reduced by warp shuffles (a minimum is exact in any order).
//   radial window (shower/api.py:322-340, shower_basis.py:408-439): basis points
//     of each (event, node band) inside / outside the table's radial range per OM.
//     One CTA per (128 OMs, event x band) stages the basis points' world
//     coordinates and photons in shared memory; each thread owns one OM and walks
//     the points in order (the far-tail sum in the reference's order).
#include "lh_common.cuh"

namespace lh {

__global__ void om_geometry_kernel(const lh_om_geometry_problem G) {
  const int om = blockIdx.x, ev = blockIdx.y;
  const int64_t begin = G.element_offset[ev], end = G.element_offset[ev + 1];
  const double rx = G.om_pos[3 * om], ry = G.om_pos[3 * om + 1], rz = G.om_pos[3 * om + 2];
  const double flight = G.group_index / 0.299792458;
  double best = 1e300, earliest = INFINITY;
  for (int64_t i = begin + threadIdx.x; i < end; i += blockDim.x) {
    const double ux = G.direction[3 * i], uy = G.direction[3 * i + 1], uz = G.direction[3 * i + 2];
    double ox = __dadd_rn(rx, -G.start[3 * i]);
    double oy = __dadd_rn(ry, -G.start[3 * i + 1]);
    double oz = __dadd_rn(rz, -G.start[3 * i + 2]);
    double along = dot3_rn(ox, oy, oz, ux, uy, uz);
    along = along < 0.0 ? 0.0 : (along > G.length[i] ? G.length[i] : along);
    const double dx = __dadd_rn(ox, -__dmul_rn(along, ux));
    const double dy = __dadd_rn(oy, -__dmul_rn(along, uy));
    const double dz = __dadd_rn(oz, -__dmul_rn(along, uz));
    const double value = dot3_rn(dx, dy, dz, dx, dy, dz);
    best = value < best ? value : best;
    const double arrival = __dadd_rn(G.start_ns[i], __dmul_rn(flight, __dsqrt_rn(value)));
    earliest = arrival < earliest ? arrival : earliest;
  }
  for (int off = 16; off > 0; off >>= 1) {
    best = fmin(best, __shfl_xor_sync(0xffffffffu, best, off));
    earliest = fmin(earliest, __shfl_xor_sync(0xffffffffu, earliest, off));
  }
  __shared__ double sb[32], se[32];
  if ((threadIdx.x & 31) == 0) {
    sb[threadIdx.x >> 5] = best;
    se[threadIdx.x >> 5] = earliest;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) {
      best = fmin(best, sb[w]);
      earliest = fmin(earliest, se[w]);
    }
    const int64_t o = (int64_t)ev * G.n_om + om;
    if (G.min_distance) G.min_distance[o] = __dsqrt_rn(best);
    if (G.earliest_ns) G.earliest_ns[o] = earliest;
  }
}

constexpr int kWindowTile = 128;

// np.interp on an ascending grid: end values outside, linear inside.
LH_DEVICE double interp_clamped(double x, const double* xp, const double* fp, int n) {
  if (x <= xp[0]) return fp[0];
  if (x >= xp[n - 1]) return fp[n - 1];
  int lo = 0, hi = n - 1;  // xp[lo] <= x < xp[hi]
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (xp[mid] <= x) lo = mid;
    else hi = mid;
  }
  const double slope = (fp[hi] - fp[lo]) / (xp[hi] - xp[lo]);
  return slope * (x - xp[lo]) + fp[lo];
}

__global__ void __launch_bounds__(kWindowTile)
radial_window_kernel(const lh_radial_window_problem S, const lh_window_event* events) {
  const int ev = blockIdx.y / S.n_bands, band = blockIdx.y % S.n_bands;
  const lh_window_event& E = events[ev];
  const int om = blockIdx.x * kWindowTile + threadIdx.x;
  const int n = E.n_points[band];
  __shared__ double s_x[kWindowTile], s_y[kWindowTile], s_z[kWindowTile], s_ph[kWindowTile];
  double rx = 0.0, ry = 0.0, rz = 0.0;
  if (om < S.n_om) {
    rx = S.om_pos[3 * om];
    ry = S.om_pos[3 * om + 1];
    rz = S.om_pos[3 * om + 2];
  }
  const double low = S.radial_low, high = S.radial_high;
  int near = 0, far = 0;
  double tail = 0.0;
  for (int base = 0; base < n; base += kWindowTile) {
    const int c = base + threadIdx.x;
    if (c < n) {
      const double* p = E.points + ((int64_t)band * E.capacity + c) * 3;
      const double z = p[0], x = p[1], y = p[2];
      double w[3];
      for (int k = 0; k < 3; ++k)
        w[k] = __dadd_rn(__dadd_rn(__dadd_rn(E.centre[k], __dmul_rn(z, E.axis[k])),
                                   __dmul_rn(x, E.first[k])),
                         __dmul_rn(y, E.second[k]));
      s_x[threadIdx.x] = w[0];
      s_y[threadIdx.x] = w[1];
      s_z[threadIdx.x] = w[2];
      const float* ch = E.channels + ((int64_t)band * E.capacity + c) * E.channel_stride;
      // |channel| rounded to float32 as the reference's complex64 magnitude (the
      // squares are exact in float64, so this is the correctly rounded hypot)
      const double re = ch[0], im = ch[1];
      const double magnitude = (double)(float)__dsqrt_rn(__dadd_rn(__dmul_rn(re, re),
                                                                    __dmul_rn(im, im)));
      s_ph[threadIdx.x] = __dmul_rn(S.photon_scale, magnitude) / S.efficiency[band];
    }
    __syncthreads();
    const int m = n - base < kWindowTile ? n - base : kWindowTile;
    if (om < S.n_om) {
      for (int j = 0; j < m; ++j) {
        const double dx = __dadd_rn(s_x[j], -rx), dy = __dadd_rn(s_y[j], -ry),
                     dz = __dadd_rn(s_z[j], -rz);
        const double r = __dsqrt_rn(
            __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz)));
        near += r < low;
        if (r > high) {
          ++far;
          const double factor = exp(interp_clamped(r, S.att_radius, S.att_log, S.n_att)) /
                                (4.0 * kPi * r * r);
          tail += s_ph[j] * factor;
        }
      }
    }
    __syncthreads();
  }
  if (om < S.n_om) {
    const int64_t o = ((int64_t)ev * S.n_bands + band) * S.n_om + om;
    S.n_near[o] = near;
    S.n_far[o] = far;
    S.far_sum[o] = tail;
  }
}

}  // namespace lh

extern "C" size_t lh_window_slot_bytes(int32_t n_events) {
  return n_events < 1 ? 0 : sizeof(lh_window_event) * (size_t)n_events;
}

extern "C" int lh_radial_window(const lh_radial_window_problem* S, const lh_window_event* events,
                                int32_t n_events, void* workspace, size_t workspace_bytes,
                                void* stream) {
  if (!S || !events || n_events < 1 || S->n_om < 1 || S->n_bands < 1 ||
      S->n_bands > 8 || n_events > 65535 / S->n_bands || !S->om_pos || S->n_att < 2 ||
      !S->att_radius || !S->att_log || !S->n_near || !S->n_far || !S->far_sum)
    return LH_EINVAL;
  for (int e = 0; e < n_events; ++e) {
    const lh_window_event& E = events[e];
    if (E.capacity < 0 || E.channel_stride < 2) return LH_EINVAL;
    for (int b = 0; b < S->n_bands; ++b)
      if (E.n_points[b] < 0 || E.n_points[b] > E.capacity) return LH_EINVAL;
    if (E.capacity > 0 && (!E.points || !E.channels)) return LH_EINVAL;
  }
  const size_t bytes = lh_window_slot_bytes(n_events);
  if (!workspace || workspace_bytes < bytes) return LH_ENOMEM;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (cudaMemcpyAsync(workspace, events, bytes, cudaMemcpyHostToDevice, s) != cudaSuccess)
    return LH_ECUDA;
  dim3 grid((unsigned)((S->n_om + lh::kWindowTile - 1) / lh::kWindowTile),
            (unsigned)(n_events * S->n_bands));
  lh::radial_window_kernel<<<grid, lh::kWindowTile, 0, s>>>(
      *S, static_cast<const lh_window_event*>(workspace));
  return cudaGetLastError() == cudaSuccess ? LH_OK : LH_ECUDA;
}

extern "C" int lh_om_geometry(const lh_om_geometry_problem* G, void* stream) {
  if (!G || G->n_om < 1 || G->n_om > 0x7fffffff || G->n_events < 1 || G->n_events > 65535 ||
      !G->om_pos || !G->element_offset || !G->start || !G->direction || !G->length ||
      !G->start_ns || (!G->min_distance && !G->earliest_ns))
    return LH_EINVAL;
  dim3 grid((unsigned)G->n_om, (unsigned)G->n_events);
  lh::om_geometry_kernel<<<grid, 256, 0, static_cast<cudaStream_t>(stream)>>>(*G);
  return cudaGetLastError() == cudaSuccess ? LH_OK : LH_ECUDA;
}

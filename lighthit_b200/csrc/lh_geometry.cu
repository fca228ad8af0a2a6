// Per-OM geometry of an element set, float64 and bit-identical to the
// reference's NumPy/Numba arithmetic (no fused multiply-adds):
//   min_distance_to_segments (_prompt_numba.py:2221-2243): distance from each
//     OM to the nearest point of any element (module selection, prompt.py:603-631);
//   earliest_element_arrival (_shower_basis.py:50-78): the per-OM clock of an
//     extended source, min over elements of start_ns + n_g/c |OM - segment|.
// One CTA per (OM, event); threads stride over the event's elements and the
// minima are reduced by warp shuffles (a minimum is exact in any order).
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

}  // namespace lh

extern "C" int lh_om_geometry(const lh_om_geometry_problem* G, void* stream) {
  if (!G || G->n_om < 1 || G->n_om > 0x7fffffff || G->n_events < 1 || G->n_events > 65535 ||
      !G->om_pos || !G->element_offset || !G->start || !G->direction || !G->length ||
      !G->start_ns || (!G->min_distance && !G->earliest_ns))
    return LH_EINVAL;
  dim3 grid((unsigned)G->n_om, (unsigned)G->n_events);
  lh::om_geometry_kernel<<<grid, 256, 0, static_cast<cudaStream_t>(stream)>>>(*G);
  return cudaGetLastError() == cudaSuccess ? LH_OK : LH_ECUDA;
}

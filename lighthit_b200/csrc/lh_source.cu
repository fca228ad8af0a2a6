// Order >=2 source compile: axial-slice basis of a shower's node bands.
//
// Reference: node_sources (shower/ge2.py:35-67) -> compile_axial_slices
// (_shower_basis.py:188-645) with the shower basis (0.25 m slices, cubic
// Lagrange axial weights, 5-moment transverse stencil of half-width 0.2 m
// for slices wider than 0.03 m, linear deposit on a 0.02 ns time lattice,
// stencil points on the axis), _cone_harmonics (:81-99) and the harmonics of
// axial_fast._harmonics_into / _layout.
//
// For element node e (chord midpoint, or two Gauss nodes on long chords) at
// axial coordinate z, transverse (x, y), time t, direction u and cone cosine
// mu_C in band b, with slice lattice zl = (z - z0)/h_z and tick lattice
// tl = (t - t_ref)/dt:
//   D[b][zb + j][tb + d][k][c] += w_j(zl - zb) w_d(tl - tb) F_k P_l(mu_C) Y_c(u)
// with F = photons_b (1, x, y, x^2, y^2) x node weight, j = -1..2 (cubic),
// d = 0, 1 (linear). Per slice the time lattice is transformed,
//   V[b][s][k][c](w) = sum_tick D[b][s][tick][k][c] e^{i w tick dt},
// and the slice's points carry V (thin slice, one point at the field-0
// centroid) or the stencil combination of its five moments (wide slice).
//
// B200 layout: nodes are counting-sorted by base lattice key (zb, tb); one
// CTA per occupied base key forms the 8 link x 5 moment x channel products of
// its nodes in shared memory (float64) and adds them to the dense
// (slice, tick) deposit once; one CTA per (slice, band) runs the time-lattice
// transform with a rotating phasor and writes the points' channels.
#include <algorithm>

#include "lh_common.cuh"
#include "lh_timing.cuh"

namespace lh {

constexpr int kSrcMaxBands = 8;
constexpr int kSrcMaxNch = 153;       // degree 16, azimuthal degree 4
constexpr int kSrcChunk = 16;         // nodes staged per pass
constexpr int kSrcThreads = 256;

struct SrcNode {
  double zr, tr, x, y;
  int64_t key;
  int el;
  int pad;
};

// Cubic Lagrange weights of shifts -1, 0, 1, 2 at offset r (_shower_basis.py:112-118)
LH_DEVICE void src_axial_weights(double r, double* w) {
  w[0] = -r * (r - 1) * (r - 2) / 6;
  w[1] = (r + 1) * (r - 1) * (r - 2) / 2;
  w[2] = -(r + 1) * r * (r - 2) / 2;
  w[3] = (r + 1) * r * (r - 1) / 6;
}

// Real orthonormal harmonics of direction (x, y, z) into out[kept channel]
// (axial_fast._harmonics_into)
LH_DEVICE void src_harmonics(double x, double y, double z, const lh_source_problem& P, double* out) {
  const double radius = sqrt(x * x + y * y + z * z);
  const double mu = z / radius;
  const double transverse = sqrt(x * x + y * y);
  const double sine = transverse / radius;
  const double cp = transverse == 0.0 ? 1.0 : x / transverse;
  const double sp = transverse == 0.0 ? 0.0 : y / transverse;
  double cm = 1.0, sm = 0.0;
  double diagonal = 1.0 / sqrt(4 * kPi);
  const int degree = P.degree, max_m = P.max_m;
  for (int m = 0; m <= max_m; ++m) {
    if (m) {
      diagonal *= sqrt((2.0 * m + 1) / (2.0 * m)) * sine;
      const double c2 = cm * cp - sm * sp, s2 = sm * cp + cm * sp;
      cm = c2;
      sm = s2;
    }
    double v0 = diagonal, v1 = 0.0;
    for (int ell = m; ell <= degree; ++ell) {
      double value;
      if (ell == m) {
        value = v0;
      } else if (ell == m + 1) {
        value = sqrt(2.0 * m + 3) * mu * v0;
        v1 = value;
      } else {
        value = P.aa[ell * (max_m + 1) + m] * mu * v1 - P.bb[ell * (max_m + 1) + m] * v0;
        v0 = v1;
        v1 = value;
      }
      const int centre = P.starts[ell] + min(ell, max_m);
      if (m == 0) {
        out[centre] = value;
      } else {
        out[centre - m] = sqrt(2.0) * value * sm;
        out[centre + m] = sqrt(2.0) * value * cm;
      }
    }
  }
}

// One thread per (element, node): lattice coordinates, counts per base key,
// slice occupancy and each slice's tick range.
__global__ void src_nodes_kernel(const lh_source_problem P, SrcNode* nodes, int32_t* counts,
                                 int32_t* slice_lo, int32_t* slice_hi, int32_t* status) {
  const int64_t total = (int64_t)P.n_el * P.element_order;
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < total;
       k += (int64_t)gridDim.x * blockDim.x) {
    const int e = (int)(k / P.element_order);
    const int n = (int)(k - (int64_t)e * P.element_order);
    const double f = P.node_fraction[n];
    const double px = P.start[3 * e] + f * P.length[e] * P.direction[3 * e];
    const double py = P.start[3 * e + 1] + f * P.length[e] * P.direction[3 * e + 1];
    const double pz = P.start[3 * e + 2] + f * P.length[e] * P.direction[3 * e + 2];
    const double ox = px - P.centre[0], oy = py - P.centre[1], oz = pz - P.centre[2];
    const double z = ox * P.axis[0] + oy * P.axis[1] + oz * P.axis[2];
    const double tx = ox - z * P.axis[0], ty = oy - z * P.axis[1], tz = oz - z * P.axis[2];
    const double x = tx * P.first[0] + ty * P.first[1] + tz * P.first[2];
    const double y = tx * P.second[0] + ty * P.second[1] + tz * P.second[2];
    const double t = P.t0[e] + f * (P.t1[e] - P.t0[e]);
    const double zl = (z - P.z_origin) / P.cell_m;
    const double zbf = floor(zl);
    const double tl = (t - P.reference_ns) / P.time_step_ns;
    const double tbf = floor(tl);
    SrcNode N;
    N.zr = zl - zbf;
    N.tr = tl - tbf;
    N.x = x;
    N.y = y;
    N.el = e;
    N.pad = n;  // Gauss node of the chord
    const long long zb = (long long)zbf, tb = (long long)tbf;
    if (zb < 1 || zb + 2 >= P.n_slices || tb < 0 || tb + 1 >= P.kmax) {
      atomicOr(reinterpret_cast<unsigned*>(status), LH_STATUS_OVERFLOW);
      N.key = -1;
      nodes[k] = N;
      continue;
    }
    N.key = zb * P.kmax + tb;
    nodes[k] = N;
    atomicAdd(counts + N.key, 1);
    for (int j = -1; j <= 2; ++j) {
      atomicMin(slice_lo + zb + j, (int)tb);
      atomicMax(slice_hi + zb + j, (int)tb + 1);
    }
  }
}

// Single CTA: exclusive scan of the base-key counts and the list of occupied keys.
__global__ void __launch_bounds__(1024)
src_scan_kernel(int64_t n_keys, const int32_t* counts, int32_t* offsets, int32_t* cursor,
                int64_t* groups, int32_t* n_groups) {
  __shared__ int32_t warp_sum[32];
  __shared__ int32_t carry, carry_groups;
  if (threadIdx.x == 0) {
    carry = 0;
    carry_groups = 0;
  }
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int64_t base = 0; base < n_keys; base += blockDim.x) {
    const int64_t i = base + threadIdx.x;
    const int32_t c = i < n_keys ? counts[i] : 0;
    // inclusive scans of the counts and of the occupied flags
    int32_t v = c, g = c > 0 ? 1 : 0;
    for (int off = 1; off < 32; off <<= 1) {
      const int32_t a = __shfl_up_sync(0xffffffffu, v, off);
      const int32_t b = __shfl_up_sync(0xffffffffu, g, off);
      if (lane >= off) {
        v += a;
        g += b;
      }
    }
    __shared__ int32_t warp_g[32];
    if (lane == 31) {
      warp_sum[warp] = v;
      warp_g[warp] = g;
    }
    __syncthreads();
    if (warp == 0) {
      int32_t s = lane < (int)(blockDim.x >> 5) ? warp_sum[lane] : 0;
      int32_t h = lane < (int)(blockDim.x >> 5) ? warp_g[lane] : 0;
      for (int off = 1; off < 32; off <<= 1) {
        const int32_t a = __shfl_up_sync(0xffffffffu, s, off);
        const int32_t b = __shfl_up_sync(0xffffffffu, h, off);
        if (lane >= off) {
          s += a;
          h += b;
        }
      }
      warp_sum[lane] = s;
      warp_g[lane] = h;
    }
    __syncthreads();
    const int32_t before = (warp ? warp_sum[warp - 1] : 0) + v - c + carry;
    const int32_t before_g = (warp ? warp_g[warp - 1] : 0) + g - (c > 0 ? 1 : 0) + carry_groups;
    if (i < n_keys) {
      offsets[i] = before;
      cursor[i] = before;
      if (c > 0) groups[before_g] = i;
    }
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) {
      carry = before + c;
      carry_groups = before_g + (c > 0 ? 1 : 0);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) *n_groups = carry_groups;
}

__global__ void src_scatter_kernel(const lh_source_problem P, const SrcNode* nodes, int32_t* cursor,
                                   int32_t* order) {
  const int64_t total = (int64_t)P.n_el * P.element_order;
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < total;
       k += (int64_t)gridDim.x * blockDim.x) {
    const int64_t key = nodes[k].key;
    if (key < 0) continue;
    order[atomicAdd(cursor + key, 1)] = (int32_t)k;
  }
}

struct SrcGroupShared {
  double harm[kSrcChunk][kSrcMaxNch];
  double pl[kSrcChunk][kSrcMaxBands][17];
  double link[kSrcChunk][8];
  double axial[kSrcChunk][4];
  double factor[kSrcChunk][kSrcMaxBands][5];
};

// One CTA per occupied base key: sum its nodes' products over
// (band, link, moment, channel) and add them to the deposit.
__global__ void __launch_bounds__(kSrcThreads)
src_group_kernel(const lh_source_problem P, const SrcNode* nodes, const int32_t* offsets,
                 const int32_t* counts, const int32_t* order, const int64_t* groups,
                 const int32_t* n_groups, double* deposit, double* zero) {
  extern __shared__ __align__(16) unsigned char src_smem[];
  SrcGroupShared& S = *reinterpret_cast<SrcGroupShared*>(src_smem);
  double* acc = reinterpret_cast<double*>(src_smem + sizeof(SrcGroupShared));
  const int NB = P.n_bands, nch = P.nch;
  const int entries = NB * 8 * 5 * nch;        // (band, link, moment, channel)
  const int zentries = NB * 4 * 5;             // (band, axial shift, moment)
  const int total_groups = *n_groups;
  for (int gi = blockIdx.x; gi < total_groups; gi += gridDim.x) {
    const int64_t key = groups[gi];
    const int begin = offsets[key], count = counts[key];
    for (int i = threadIdx.x; i < entries + zentries; i += blockDim.x) acc[i] = 0.0;
    for (int c0 = 0; c0 < count; c0 += kSrcChunk) {
      const int nn = min(kSrcChunk, count - c0);
      __syncthreads();
      if (threadIdx.x < nn) {
        const int q = threadIdx.x;
        const SrcNode N = nodes[order[begin + c0 + q]];
        const int e = N.el;
        const double ux = P.direction[3 * e], uy = P.direction[3 * e + 1], uz = P.direction[3 * e + 2];
        // rotate into (first, second, axis)
        const double rx = ux * P.first[0] + uy * P.first[1] + uz * P.first[2];
        const double ry = ux * P.second[0] + uy * P.second[1] + uz * P.second[2];
        const double rz = ux * P.axis[0] + uy * P.axis[1] + uz * P.axis[2];
        src_harmonics(rx, ry, rz, P, S.harm[q]);
        double wz[4];
        src_axial_weights(N.zr, wz);
        const double wt[2] = {1 - N.tr, N.tr};
        for (int j = 0; j < 4; ++j) {
          S.axial[q][j] = wz[j];
          for (int d = 0; d < 2; ++d) S.link[q][2 * j + d] = wz[j] * wt[d];
        }
        for (int b = 0; b < NB; ++b) {
          // signed band field C0/lambda^2 + C2/(lambda n)^2 times the chord node weight
          const double f = (P.c0[e] * P.band_s0[b] + P.c2[e] * P.band_s2[b]) * P.node_weight[N.pad];
          S.factor[q][b][0] = f;
          S.factor[q][b][1] = f * N.x;
          S.factor[q][b][2] = f * N.y;
          S.factor[q][b][3] = f * N.x * N.x;
          S.factor[q][b][4] = f * N.y * N.y;
          const double mu = 1.0 / (P.beta[e] * P.band_phase[b]);
          double prev = 1.0, cur = mu;
          for (int ell = 0; ell <= P.degree; ++ell) {
            double p;
            if (ell == 0) p = 1.0;
            else if (ell == 1) p = cur;
            else {
              p = ((2 * ell - 1) * mu * cur - (ell - 1) * prev) / ell;
              prev = cur;
              cur = p;
            }
            S.pl[q][b][ell] = p;
          }
        }
      }
      __syncthreads();
      for (int i = threadIdx.x; i < entries; i += blockDim.x) {
        const int c = i % nch;
        int rest = i / nch;
        const int k = rest % 5;
        rest /= 5;
        const int link = rest % 8;
        const int b = rest / 8;
        const int ell = P.channel_degree[c];
        double sum = 0.0;
        for (int q = 0; q < nn; ++q)
          sum += S.link[q][link] * S.factor[q][b][k] * (S.harm[q][c] * S.pl[q][b][ell]);
        acc[i] += sum;
      }
      for (int i = threadIdx.x; i < zentries; i += blockDim.x) {
        const int k = i % 5;
        const int j = (i / 5) % 4;
        const int b = i / 20;
        double sum = 0.0;
        for (int q = 0; q < nn; ++q) sum += S.axial[q][j] * S.factor[q][b][k];
        acc[entries + i] += sum;
      }
    }
    __syncthreads();
    const long long zb = key / P.kmax, tb = key - zb * P.kmax;
    for (int i = threadIdx.x; i < entries; i += blockDim.x) {
      const double v = acc[i];
      if (v == 0.0) continue;
      const int c = i % nch;
      int rest = i / nch;
      const int k = rest % 5;
      rest /= 5;
      const int link = rest % 8;
      const int b = rest / 8;
      const long long row = (zb + (link >> 1) - 1) * P.kmax + tb + (link & 1);
      atomicAdd(deposit + ((row * NB + b) * 5 + k) * nch + c, v);
    }
    for (int i = threadIdx.x; i < zentries; i += blockDim.x) {
      const int k = i % 5;
      const int j = (i / 5) % 4;
      const int b = i / 20;
      atomicAdd(zero + ((zb + j - 1) * NB + b) * 5 + k, acc[entries + i]);
    }
    __syncthreads();
  }
}

// Single thread: point layout of every band (_shower_basis.py:375-420, 466-475):
// occupied slices in order, then the +x, -x, +y, -y stencil points of the wide
// slices; thin slices sit at their field-0 centroid, wide ones on the axis.
__global__ void src_layout_kernel(const lh_source_problem P, const int32_t* slice_lo,
                                  const int32_t* slice_hi, const double* zero, int32_t* slice_point,
                                  int32_t* slice_wide, double* centroid, int32_t* n_occ_out,
                                  lh_source_output O) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const int NB = P.n_bands;
  const int64_t S = P.n_slices;
  int n_occ = 0;
  for (int64_t s = 0; s < S; ++s) n_occ += slice_hi[s] >= 0 ? 1 : 0;
  *n_occ_out = n_occ;
  for (int b = 0; b < NB; ++b) {
    int occ = 0, wide_count = 0;
    for (int64_t s = 0; s < S; ++s) {
      slice_point[b * S + s] = -1;
      slice_wide[b * S + s] = -1;
      if (slice_hi[s] < 0) continue;
      const double* zm = zero + (s * NB + b) * 5;
      const double mass = zm[0];
      const double safe = mass != 0.0 ? mass : 1.0;
      // absolute values by comparison: nvcc 12.9 at -O3 dropped fabs() of this
      // select (fabs(safe) came back negative for a negative mass)
      const double num = zm[3] + zm[4];
      const double spread = sqrt((num < 0.0 ? -num : num) / (safe < 0.0 ? -safe : safe));
      const bool wide = spread > P.stencil_threshold_m;
      const double cx = wide ? 0.0 : zm[1] / safe, cy = wide ? 0.0 : zm[2] / safe;
      centroid[(b * S + s) * 2] = cx;
      centroid[(b * S + s) * 2 + 1] = cy;
      slice_point[b * S + s] = occ;
      const double z = P.z_origin + (double)s * P.cell_m;
      double* pt = O.points + ((int64_t)b * O.capacity + occ) * 3;
      pt[0] = z;
      pt[1] = cx;
      pt[2] = cy;
      if (wide) slice_wide[b * S + s] = wide_count++;
      ++occ;
    }
    // stencil points: offsets (h,0), (-h,0), (0,h), (0,-h) in wide-slice order
    const double h = P.stencil_m;
    const double ox[4] = {h, -h, 0.0, 0.0}, oy[4] = {0.0, 0.0, h, -h};
    for (int64_t s = 0; s < S; ++s) {
      const int w = slice_wide[b * S + s];
      if (w < 0) continue;
      const double z = P.z_origin + (double)s * P.cell_m;
      for (int o = 0; o < 4; ++o) {
        double* pt = O.points + ((int64_t)b * O.capacity + occ + o * wide_count + w) * 3;
        pt[0] = z;
        pt[1] = ox[o];
        pt[2] = oy[o];
      }
    }
    O.n_points[b] = occ + 4 * wide_count;
  }
}

// One CTA per (slice, band, block of `w_block` frequencies): time-lattice
// transform and the slice's points (_shower_basis.py:577-611). One thread per
// (channel, frequency) walks the slice's ticks with a rotating phasor; the
// CTA stages the deposit rows of kSrcStageBytes worth of ticks at a time in
// shared memory (coalesced, independent loads) before the threads read them.
constexpr int kSrcOmegaBlock = 8;
constexpr int kSrcStageBytes = 48 * 1024;

__global__ void src_transform_kernel(const lh_source_problem P, const int32_t* slice_lo,
                                     const int32_t* slice_hi, const double* deposit,
                                     const int32_t* slice_point, const int32_t* slice_wide,
                                     const int32_t* n_occ, lh_source_output O, int w_block) {
  extern __shared__ double s_dep[];  // [tick][moment][channel]
  const int64_t s = blockIdx.x;
  const int b = blockIdx.y;
  const int NB = P.n_bands, nch = P.nch, W = P.n_omega;
  if (slice_hi[s] < 0) return;
  const int lo = slice_lo[s], hi = slice_hi[s];
  const int64_t S = P.n_slices;
  const int point = slice_point[b * S + s];
  const int wide = slice_wide[b * S + s];
  const int occ = *n_occ;
  const int wide_count = (O.n_points[b] - occ) / 4;
  const double h = P.stencil_m, h2 = h * h;
  const double scale = P.band_scale[b];
  const int w_begin = blockIdx.z * w_block;
  const int w_count = min(w_block, W - w_begin);
  const int nk = wide >= 0 ? 5 : 1;
  const int row = nk * nch;  // staged doubles per tick
  const int chunk = max(1, min(64, (int)(kSrcStageBytes / sizeof(double)) / row));
  const int i = threadIdx.x;
  const bool mine = i < nch * w_count;
  const int c = mine ? i % nch : 0, w = w_begin + (mine ? i / nch : 0);
  const double om = P.omega[w];
  double ps = 0, pc = 1, ds = 0, dc = 1;
  if (mine) {
    sincos(om * lo * P.time_step_ns, &ps, &pc);
    sincos(om * P.time_step_ns, &ds, &dc);
  }
  double re[5] = {0, 0, 0, 0, 0}, im[5] = {0, 0, 0, 0, 0};
  for (int t0 = lo; t0 <= hi; t0 += chunk) {
    const int n_t = min(chunk, hi - t0 + 1);
    __syncthreads();
    for (int e = threadIdx.x; e < n_t * row; e += blockDim.x) {
      const int tt = e / row, r = e - tt * row;
      s_dep[e] = deposit[(((s * P.kmax + t0 + tt) * NB + b) * 5) * nch + r];
    }
    __syncthreads();
    if (!mine) continue;
    for (int tt = 0; tt < n_t; ++tt) {
      const double* rowp = s_dep + tt * row + c;
      for (int k = 0; k < nk; ++k) {
        const double v = rowp[k * nch];
        re[k] += v * pc;
        im[k] += v * ps;
      }
      const double npc = pc * dc - ps * ds, nps = ps * dc + pc * ds;
      pc = npc;
      ps = nps;
    }
  }
  if (mine) {
    float2* out = reinterpret_cast<float2*>(O.channels);
    auto put = [&](int p, double r, double m) {
      out[(((int64_t)b * O.capacity + p) * nch + c) * W + w] =
          make_float2((float)(scale * r), (float)(scale * m));
    };
    if (wide < 0) {
      put(point, re[0], im[0]);
    } else {
      // m0, mx, my, mxx, myy -> centre, +x, -x, +y, -y
      put(point, re[0] - (re[3] + re[4]) / h2, im[0] - (im[3] + im[4]) / h2);
      put(occ + 0 * wide_count + wide, 0.5 * (re[3] / h2 + re[1] / h), 0.5 * (im[3] / h2 + im[1] / h));
      put(occ + 1 * wide_count + wide, 0.5 * (re[3] / h2 - re[1] / h), 0.5 * (im[3] / h2 - im[1] / h));
      put(occ + 2 * wide_count + wide, 0.5 * (re[4] / h2 + re[2] / h), 0.5 * (im[4] / h2 + im[2] / h));
      put(occ + 3 * wide_count + wide, 0.5 * (re[4] / h2 - re[2] / h), 0.5 * (im[4] / h2 - im[2] / h));
    }
  }
}

struct SrcWorkspace {
  SrcNode* nodes;
  int32_t *counts, *offsets, *cursor, *order, *n_groups, *slice_lo, *slice_hi, *slice_point,
      *slice_wide, *n_occ;
  int64_t* groups;
  double *deposit, *zero, *centroid;
  size_t bytes;
};

static size_t src_align(size_t x) { return (x + 255) & ~(size_t)255; }

static SrcWorkspace src_layout(const lh_source_problem& P, unsigned char* base) {
  SrcWorkspace W{};
  size_t off = 0;
  auto take = [&](size_t bytes) {
    unsigned char* p = base ? base + off : nullptr;
    off += src_align(bytes);
    return p;
  };
  const int64_t n_nodes = (int64_t)P.n_el * P.element_order;
  const int64_t n_keys = P.n_slices * P.kmax;
  const int NB = P.n_bands;
  W.nodes = reinterpret_cast<SrcNode*>(take(sizeof(SrcNode) * n_nodes));
  W.counts = reinterpret_cast<int32_t*>(take(sizeof(int32_t) * n_keys));
  W.offsets = reinterpret_cast<int32_t*>(take(sizeof(int32_t) * n_keys));
  W.cursor = reinterpret_cast<int32_t*>(take(sizeof(int32_t) * n_keys));
  W.order = reinterpret_cast<int32_t*>(take(sizeof(int32_t) * n_nodes));
  W.groups = reinterpret_cast<int64_t*>(take(sizeof(int64_t) * n_keys));
  W.n_groups = reinterpret_cast<int32_t*>(take(sizeof(int32_t) * 4));
  W.n_occ = reinterpret_cast<int32_t*>(take(sizeof(int32_t) * 4));
  W.slice_lo = reinterpret_cast<int32_t*>(take(sizeof(int32_t) * P.n_slices));
  W.slice_hi = reinterpret_cast<int32_t*>(take(sizeof(int32_t) * P.n_slices));
  W.slice_point = reinterpret_cast<int32_t*>(take(sizeof(int32_t) * P.n_slices * NB));
  W.slice_wide = reinterpret_cast<int32_t*>(take(sizeof(int32_t) * P.n_slices * NB));
  W.deposit = reinterpret_cast<double*>(take(sizeof(double) * n_keys * NB * 5 * P.nch));
  W.zero = reinterpret_cast<double*>(take(sizeof(double) * P.n_slices * NB * 5));
  W.centroid = reinterpret_cast<double*>(take(sizeof(double) * P.n_slices * NB * 2));
  W.bytes = off;
  return W;
}

static bool src_valid(const lh_source_problem* P) {
  if (!P) return false;
  if (P->n_el < 1 || !P->start || !P->direction || !P->length || !P->c0 || !P->c2 || !P->beta ||
      !P->t0 || !P->t1)
    return false;
  if (P->n_bands < 1 || P->n_bands > kSrcMaxBands) return false;
  if (P->degree < 0 || P->degree > 16 || P->max_m < 0 || P->max_m > 4 || P->max_m > P->degree ||
      P->nch < 1 || P->nch > kSrcMaxNch)
    return false;
  if (P->element_order < 1 || P->element_order > 2) return false;
  if (!(P->cell_m > 0) || !(P->stencil_m > 0) || !(P->time_step_ns > 0)) return false;
  if (P->n_slices < 4 || P->kmax < 2 || P->n_slices * P->kmax > (1ll << 30)) return false;
  if (P->n_omega < 1 || !P->omega) return false;
  return true;
}

}  // namespace lh

extern "C" size_t lh_source_workspace_bytes(const lh_source_problem* P) {
  if (!lh::src_valid(P)) return 0;
  return lh::src_layout(*P, nullptr).bytes;
}

extern "C" int lh_source_compile(const lh_source_problem* P, const lh_source_output* O,
                                 void* workspace, size_t workspace_bytes, int32_t* status,
                                 void* stream) {
  if (!lh::src_valid(P) || !O || !O->points || !O->channels || !O->n_points || !status)
    return LH_EINVAL;
  if (O->capacity < P->n_slices * 5) return LH_EINVAL;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  lh::SrcWorkspace W = lh::src_layout(*P, static_cast<unsigned char*>(workspace));
  if (!workspace || workspace_bytes < W.bytes) return LH_ENOMEM;
  const int64_t n_nodes = (int64_t)P->n_el * P->element_order;
  const int64_t n_keys = P->n_slices * P->kmax;
  const int NB = P->n_bands;
  cudaMemsetAsync(W.counts, 0, sizeof(int32_t) * n_keys, s);
  cudaMemsetAsync(W.slice_lo, 0x7f, sizeof(int32_t) * P->n_slices, s);
  cudaMemsetAsync(W.slice_hi, 0xff, sizeof(int32_t) * P->n_slices, s);
  cudaMemsetAsync(W.deposit, 0, sizeof(double) * n_keys * NB * 5 * P->nch, s);
  cudaMemsetAsync(W.zero, 0, sizeof(double) * P->n_slices * NB * 5, s);
  cudaMemsetAsync(O->channels, 0, sizeof(float) * 2 * NB * O->capacity * P->nch * P->n_omega, s);
  int blocks = (int)std::min<int64_t>((n_nodes + 255) / 256, 148 * 32);
  lh::src_nodes_kernel<<<std::max(blocks, 1), 256, 0, s>>>(*P, W.nodes, W.counts, W.slice_lo,
                                                          W.slice_hi, status);
  lh::src_scan_kernel<<<1, 1024, 0, s>>>(n_keys, W.counts, W.offsets, W.cursor, W.groups,
                                         W.n_groups);
  lh::src_scatter_kernel<<<std::max(blocks, 1), 256, 0, s>>>(*P, W.nodes, W.cursor, W.order);
  const size_t gsmem = sizeof(lh::SrcGroupShared) + sizeof(double) * (NB * 45 * P->nch + NB * 20);
  if (gsmem > 200 * 1024) return LH_EUNSUPPORTED;
  if (cudaFuncSetAttribute(lh::src_group_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)gsmem) != cudaSuccess)
    return LH_ECUDA;
  {
    lh::TimedLaunch timed_launch(LH_KT_SRC_GROUP, s);
    lh::src_group_kernel<<<148 * 4, lh::kSrcThreads, gsmem, s>>>(
        *P, W.nodes, W.offsets, W.counts, W.order, W.groups, W.n_groups, W.deposit, W.zero);
  }
  lh::src_layout_kernel<<<1, 32, 0, s>>>(*P, W.slice_lo, W.slice_hi, W.zero, W.slice_point,
                                         W.slice_wide, W.centroid, W.n_occ, *O);
  const int w_block = std::max(1, std::min(lh::kSrcOmegaBlock, 1024 / P->nch));
  dim3 grid((unsigned)P->n_slices, (unsigned)NB, (unsigned)((P->n_omega + w_block - 1) / w_block));
  const int threads = ((P->nch * w_block + 31) / 32) * 32;
  {
    lh::TimedLaunch timed_launch(LH_KT_SRC_TRANSFORM, s);
    lh::src_transform_kernel<<<grid, threads, lh::kSrcStageBytes, s>>>(
        *P, W.slice_lo, W.slice_hi, W.deposit, W.slice_point, W.slice_wide, W.n_occ, *O, w_block);
  }
  return cudaGetLastError() == cudaSuccess ? LH_OK : LH_ECUDA;
}

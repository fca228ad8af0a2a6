// Order >=2 near field: element portions closer to an OM than the radial
// minimum of the order >=2 tables (reference near_field.py:39-171 with the
// clamped evaluator _cone_many_looks, muon/track_ge2_primitive.py:612-660).
//
// For a portion [s0, s1] of element e within radius R of OM d, in the frame
// (ex, ey, axis) of the element with the OM at impact rho and axial offset
// u = z - s from the emission point s, the reference sums over Gauss points
//
//   N_d(w) += (c0 / len) w_u e^{i w (t_emit(s) - origin_d)}
//             sum_lam S_lam e^{i w r / v_lam} sum_l h_lam,l sum_p F_l,p C_lam,l,p(t, w),
//
// r = hypot(rho, u), S_lam = weight_lam area_d e^{-mu_lam r_a} / (4 pi r_a^2),
// r_a = max(r, r_min) (the clamp: the amplitude of the first radial interval
// at r_min, the flight phase of the actual distance), F_l,p the m = 0 Wigner
// column times the acceptance-weighted detector harmonics of the look, h the
// spectral cone harmonics of the element per unit coefficient0.
//
// Grid (OM, element slice), 256 threads. A CTA tests its slice of the elements
// 256 at a time (one thread per element, near_portions :39-69), compacts the
// portions in element order, sets up groups of 64 portions (frame, look, cone
// harmonics, panel count: one thread each), and runs the group's Gauss points
// in batches of 64: one thread per point forms F, the clamped scales and the
// phase arguments in float64; one thread per (wavelength, frequency) contracts
// F with the interval-0 splines in float32 and accumulates the phased values in
// float64. near_reduce_kernel sums each OM's slices in order.
#include <algorithm>

#include "lh_common.cuh"
#include "lh_harmonics.cuh"

namespace lh {

constexpr int kNearLam = 8;        // wavelength nodes bound
constexpr int kNearDeg = 16;       // kernel degree bound
constexpr int kNearOut = 4;        // detector degree bound
constexpr int kNearPairs = 8;      // detector pairs bound
constexpr int kNearGauss = 16;     // Gauss order bound
constexpr int kNearOmega = 128;    // frequencies bound
constexpr int kNearThreads = 256;
constexpr int kNearGroup = 64;     // portions set up together
constexpr int kNearBatch = 64;     // points per geometry batch
constexpr int kNearMaxSlices = 32;
constexpr int kNearElementsPerSlice = 4096;

struct NearPortion {
  double u_lo, u_hi, step;         // axial offsets z - s1, z - s0 and the panel step
  double rho;                      // impact (1e-9 on the line)
  double look[3];                  // OM look in (ex, ey, axis)
  double density, clock, closest;  // c0 / len, ns per m, start_ns + z clock - origin
  int count;                       // panels (0 when every cone harmonic is zero)
  int first_point;                 // first Gauss point of the portion in the group
  float h[kNearLam][kNearDeg + 1]; // cone harmonics per unit coefficient0
};

struct NearPoint {
  double radius, wd, trel;         // distance, w x density, emission time - origin
  double scale[kNearLam];          // band scales at the clamped radius
  float t;                         // log(r_a) - log_r0
  int portion;
};

// Dynamic shared memory of near_field_kernel.
size_t near_smem(const lh_near_table& T) {
  const size_t items = (size_t)T.n_lambda * T.n_omega;
  return sizeof(NearPortion) * kNearGroup + sizeof(NearPoint) * kNearBatch +
         sizeof(float) * kNearBatch * (T.degree + 1) * T.n_pairs + sizeof(double2) * items;
}

LH_DEVICE double dmul(double a, double b) { return __dmul_rn(a, b); }
LH_DEVICE double dadd(double a, double b) { return __dadd_rn(a, b); }

// Element e against OM position d (near_portions, near_field.py:55-68):
// the portion [s0, s1] of the element within radius R, if any.
LH_DEVICE bool near_portion(const lh_near_problem& P, int e, const double* d, double R2,
                            double& s0, double& s1) {
  const double* a = P.start_m + 3 * e;
  const double* n = P.direction + 3 * e;
  const double dx = d[0] - a[0], dy = d[1] - a[1], dz = d[2] - a[2];
  const double z = dadd(dadd(dmul(dx, n[0]), dmul(dy, n[1])), dmul(dz, n[2]));
  const double dd = dadd(dadd(dmul(dx, dx), dmul(dy, dy)), dmul(dz, dz));
  double rho2 = dd - dmul(z, z);
  rho2 = rho2 > 0.0 ? rho2 : 0.0;
  if (!(rho2 < R2)) return false;
  const double half = sqrt(R2 - rho2);
  s0 = fmax(z - half, 0.0);
  s1 = fmin(z + half, P.length_m[e]);
  return s1 > s0;
}

// One portion's frame, look, cone harmonics and panels (near_field.py:122-155,
// _harmonics :72-88).
LH_DEVICE void near_setup(const lh_near_table& T, const lh_near_problem& P, int e, const double* d,
                          const double* look, double origin, double s0, double s1, NearPortion& q,
                          int* n_eval) {
  const double* a = P.start_m + 3 * e;
  const double* n = P.direction + 3 * e;
  const double dx = d[0] - a[0], dy = d[1] - a[1], dz = d[2] - a[2];
  const double z = dadd(dadd(dmul(dx, n[0]), dmul(dy, n[1])), dmul(dz, n[2]));
  double rx = dx - dmul(z, n[0]), ry = dy - dmul(z, n[1]), rz = dz - dmul(z, n[2]);
  double rho = sqrt(rx * rx + ry * ry + rz * rz);
  if (rho < 1e-9) {  // the line goes through the OM centre: any transverse axis
    const double tx = fabs(n[0]) < 0.9 ? 1.0 : 0.0, ty = 1.0 - tx;
    const double c = tx * n[0] + ty * n[1];
    rx = tx - c * n[0];
    ry = ty - c * n[1];
    rz = -c * n[2];
    rho = 1e-9;
  }
  const double rn = sqrt(rx * rx + ry * ry + rz * rz);
  const double ex[3] = {rx / rn, ry / rn, rz / rn};
  const double ey[3] = {n[1] * ex[2] - n[2] * ex[1], n[2] * ex[0] - n[0] * ex[2],
                        n[0] * ex[1] - n[1] * ex[0]};
  q.rho = rho;
  q.look[0] = look[0] * ex[0] + look[1] * ex[1] + look[2] * ex[2];
  q.look[1] = look[0] * ey[0] + look[1] * ey[1] + look[2] * ey[2];
  q.look[2] = look[0] * n[0] + look[1] * n[1] + look[2] * n[2];
  const double len = P.length_m[e];
  q.clock = (P.end_ns[e] - P.start_ns[e]) / len;
  q.density = P.coefficient0[e] / len;
  q.closest = P.start_ns[e] + z * q.clock - origin;
  // spectral cone harmonics per unit coefficient0
  const double c0 = P.coefficient0[e];
  const double ratio = c0 > 0.0 ? P.coefficient2[e] / c0 : 0.0;
  const double beta = P.beta[e];
  bool any = false;
  for (int lam = 0; lam < T.n_lambda; ++lam) {
    const double phase = T.phase_index[lam], wl = T.wavelength_nm[lam];
    const double yield = (1.0 + ratio / (phase * phase)) / (wl * wl);
    const bool on = beta * phase > 1.0 && yield > 0.0;
    const double x = on ? 1.0 / (beta * phase) : 0.0;
    double p_prev = 1.0, p_cur = x;
    for (int l = 0; l <= T.degree; ++l) {
      double legendre;
      if (l == 0) legendre = 1.0;
      else if (l == 1) legendre = x;
      else {
        const double next = ((2 * l - 1) * x * p_cur - (l - 1) * p_prev) / l;
        p_prev = p_cur;
        p_cur = next;
        legendre = next;
      }
      const double v = on ? sqrt((2 * l + 1) / (4 * kPi)) * legendre * yield : 0.0;
      q.h[lam][l] = (float)v;
      any |= v != 0.0;
    }
  }
  // points as u = z - s on the panels of linspace(z - s1, z - s0, count + 1)
  const int count = max(1, (int)ceil((s1 - s0) / T.panel_m));
  q.u_lo = z - s1;
  q.u_hi = z - s0;
  q.step = (q.u_hi - q.u_lo) / count;
  q.count = any ? count : 0;
  if (any) atomicAdd(n_eval, 1);
}

// One Gauss point: F, clamped scales, phase terms (_cone_many_looks :628-659).
LH_DEVICE void near_point(const lh_near_table& T, const NearPortion& q, int local, double area,
                          double r_low, NearPoint& pt, float* F) {
  const int G = T.gauss_order, L = T.degree, A = T.acc_degree, NP = T.n_pairs;
  const int panel = local / G, node = local - panel * G;
  const double lo = dadd(dmul((double)panel, q.step), q.u_lo);
  const double hi = panel + 1 < q.count ? dadd(dmul((double)(panel + 1), q.step), q.u_lo) : q.u_hi;
  const double half = (hi - lo) / 2;
  const double u = lo + half * (T.gauss_x[node] + 1.0);
  const double w = half * T.gauss_w[node];
  const double radius = hypot(q.rho, u);
  if (radius > T.radial_high || radius == 0.0) {
    pt.wd = 0.0;
    pt.radius = 1.0;
    pt.trel = 0.0;
    pt.t = 0.f;
    for (int lam = 0; lam < kNearLam; ++lam) pt.scale[lam] = 0.0;
    for (int i = 0; i < (L + 1) * NP; ++i) F[i] = 0.f;
    return;
  }
  const double cosine = u / radius, sine = q.rho / radius;
  // Wigner d^l_(0 nu)-column for nu = 0..A (source m = 0), by recurrence in l
  double wig[kNearDeg + 1][kNearOut + 1];
  const double hc = sqrt((1.0 + cosine) / 2.0), hs = sqrt(fmax((1.0 - cosine) / 2.0, 0.0));
  for (int nu = 0; nu <= A; ++nu) {
    for (int l = 0; l < nu && l <= L; ++l) wig[l][nu] = 0.0;
    if (nu > L) continue;
    double prev = 0.0, cur = wigner_start(nu, 0, nu, hc, hs, T.start_norm, A);
    wig[nu][nu] = cur;
    for (int l = nu; l < L; ++l) {
      double value;
      if (l == 0) value = cosine * cur;
      else {
        double lower = (double)(l * l) * (double)(l * l - nu * nu);
        lower = lower > 0.0 ? sqrt(lower) : 0.0;
        const double upper = sqrt((double)((l + 1) * (l + 1)) * (double)((l + 1) * (l + 1) - nu * nu));
        value = ((2 * l + 1) * (l * (l + 1) * cosine) * cur - (l + 1) * lower * prev) / (l * upper);
      }
      prev = cur;
      cur = value;
      wig[l + 1][nu] = cur;
    }
  }
  double det[(kNearOut + 1) * (kNearOut + 1)];
  real_harmonics(cosine * q.look[0] - sine * q.look[2], q.look[1],
                 sine * q.look[0] + cosine * q.look[2], A, det);
  const double root2 = sqrt(2.0);
  for (int l = 0; l <= L; ++l)
    for (int p = 0; p < NP; ++p) {
      const int lam = T.pair_lambda[p], mu = T.pair_mu[p];
      double f = 0.0;
      if (mu <= l && mu <= A) {
        const double rot = mu == 0 ? wig[l][0] : root2 * par(mu) * wig[l][mu];
        f = rot * T.alpha[lam] * det[lam * lam + lam + mu];
      }
      F[l * NP + p] = (float)f;
    }
  const double amp = fmax(radius, r_low);
  pt.radius = radius;
  pt.t = (float)(log(amp) - T.log_r0);
  pt.wd = w * q.density;
  pt.trel = q.closest - u * q.clock;
  for (int lam = 0; lam < kNearLam; ++lam)
    pt.scale[lam] = lam < T.n_lambda ? T.spectral_weight[lam] * area *
                                           exp(-T.absorption[lam] * amp) / (4 * kPi * amp * amp)
                                     : 0.0;
}

__global__ void __launch_bounds__(kNearThreads)
near_field_kernel(lh_near_table T, lh_near_problem P, int slices, int per_slice,
                  double2* partial, int* counts) {
  extern __shared__ __align__(16) unsigned char near_smem_raw[];
  NearPortion* s_q = reinterpret_cast<NearPortion*>(near_smem_raw);
  NearPoint* s_pt = reinterpret_cast<NearPoint*>(s_q + kNearGroup);
  const int NP = T.n_pairs, fsz = (T.degree + 1) * NP;
  float* s_F = reinterpret_cast<float*>(s_pt + kNearBatch);
  double2* s_acc = reinterpret_cast<double2*>(
      near_smem_raw + ((sizeof(NearPortion) * kNearGroup + sizeof(NearPoint) * kNearBatch +
                        sizeof(float) * kNearBatch * fsz + 15) & ~size_t(15)));
  __shared__ int s_warp[kNearThreads / 32];
  __shared__ int s_total, s_points, s_portions, s_eval;
  __shared__ double s_d[3], s_look[3];

  const int om = blockIdx.x, slice = blockIdx.y, tid = threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5;
  const int items = T.n_lambda * T.n_omega;
  for (int i = tid; i < items; i += blockDim.x) s_acc[i] = make_double2(0.0, 0.0);
  if (tid < 3) {
    s_d[tid] = P.om_pos[3 * om + tid];
    s_look[tid] = P.om_look[3 * om + tid];
  }
  if (tid == 0) {
    s_portions = 0;
    s_eval = 0;
  }
  __syncthreads();
  const double area = P.om_area[om], origin = P.time_origin_ns[om];
  const double R2 = P.radius_m * P.radius_m, r_low = exp(T.log_r0);
  const int e_begin = slice * per_slice;
  const int e_end = min(P.n_elements, e_begin + per_slice);

  for (int base = e_begin; base < e_end; base += blockDim.x) {
    const int e = base + tid;
    double s0 = 0.0, s1 = 0.0;
    const bool hit = e < e_end && near_portion(P, e, s_d, R2, s0, s1);
    // ordered compaction: rank of this element among the block's portions
    const unsigned mask = __ballot_sync(0xffffffffu, hit);
    if (lane == 0) s_warp[warp] = __popc(mask);
    __syncthreads();
    if (tid == 0) {
      int run = 0;
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
        const int c = s_warp[w];
        s_warp[w] = run;
        run += c;
      }
      s_total = run;
      s_portions += run;
    }
    __syncthreads();
    const int rank = s_warp[warp] + __popc(mask & ((1u << lane) - 1u));
    const int total = s_total;
    for (int g = 0; g < total; g += kNearGroup) {
      if (hit && rank >= g && rank < g + kNearGroup)
        near_setup(T, P, e, s_d, s_look, origin, s0, s1, s_q[rank - g], &s_eval);
      __syncthreads();
      const int in_group = min(kNearGroup, total - g);
      if (tid == 0) {
        int run = 0;
        for (int k = 0; k < in_group; ++k) {
          s_q[k].first_point = run;
          run += s_q[k].count * T.gauss_order;
        }
        s_points = run;
      }
      __syncthreads();
      const int n_points = s_points;
      for (int pb = 0; pb < n_points; pb += kNearBatch) {
        const int nb = min(kNearBatch, n_points - pb);
        if (tid < nb) {
          const int k = pb + tid;
          int lo = 0, hi = in_group - 1;  // last portion with first_point <= k
          while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (s_q[mid].first_point <= k) lo = mid;
            else hi = mid - 1;
          }
          s_pt[tid].portion = lo;
          near_point(T, s_q[lo], k - s_q[lo].first_point, area, r_low, s_pt[tid],
                     s_F + tid * fsz);
        }
        __syncthreads();
        for (int item = tid; item < items; item += blockDim.x) {
          const int lam = item / T.n_omega, f = item - lam * T.n_omega;
          const double w_f = T.omega[f];
          const double inv_v = T.flight ? 1.0 / T.speed[lam] : 0.0;
          const float2* cf = reinterpret_cast<const float2*>(T.coef) +
                             (int64_t)lam * (T.degree + 1) * NP * 4 * T.n_omega + f;
          double ar = 0.0, ai = 0.0;
          for (int i = 0; i < nb; ++i) {
            const NearPoint& pt = s_pt[i];
            if (pt.wd == 0.0) continue;
            const float* h = s_q[pt.portion].h[lam];
            const float* F = s_F + i * fsz;
            const float t = pt.t;
            float vr = 0.f, vi = 0.f;
            for (int l = 0; l <= T.degree; ++l) {
              const float hl = h[l];
              if (hl == 0.f) continue;
              float gr = 0.f, gi = 0.f;
              for (int p = 0; p < NP; ++p) {
                const float2* k = cf + ((int64_t)(l * NP + p) * 4) * T.n_omega;
                const float2 k0 = __ldg(k), k1 = __ldg(k + T.n_omega);
                const float2 k2 = __ldg(k + 2 * T.n_omega), k3 = __ldg(k + 3 * T.n_omega);
                const float rr = fmaf(fmaf(fmaf(k0.x, t, k1.x), t, k2.x), t, k3.x);
                const float ri = fmaf(fmaf(fmaf(k0.y, t, k1.y), t, k2.y), t, k3.y);
                gr = fmaf(F[l * NP + p], rr, gr);
                gi = fmaf(F[l * NP + p], ri, gi);
              }
              vr = fmaf(hl, gr, vr);
              vi = fmaf(hl, gi, vi);
            }
            double sn, cs;
            sincos(w_f * (pt.radius * inv_v + pt.trel), &sn, &cs);
            const double amp = pt.scale[lam] * pt.wd;
            ar += amp * ((double)vr * cs - (double)vi * sn);
            ai += amp * ((double)vr * sn + (double)vi * cs);
          }
          s_acc[item].x += ar;
          s_acc[item].y += ai;
        }
        __syncthreads();
      }
    }
    __syncthreads();  // every thread has read s_warp and s_total before they change
  }
  const int64_t at = (int64_t)om * slices + slice;
  for (int f = tid; f < T.n_omega; f += blockDim.x) {
    double re = 0.0, im = 0.0;
    for (int lam = 0; lam < T.n_lambda; ++lam) {
      re += s_acc[lam * T.n_omega + f].x;
      im += s_acc[lam * T.n_omega + f].y;
    }
    partial[at * T.n_omega + f] = make_double2(re, im);
  }
  if (tid == 0) {
    counts[2 * at] = s_portions;
    counts[2 * at + 1] = s_eval;
  }
}

// One thread per (OM, frequency): the OM's slices in order.
__global__ void near_reduce_kernel(lh_near_table T, lh_near_problem P, int slices,
                                   const double2* partial, const int* counts) {
  const int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (idx >= (int64_t)P.n_om * T.n_omega) return;
  const int om = (int)(idx / T.n_omega), f = (int)(idx % T.n_omega);
  double re = 0.0, im = 0.0;
  for (int s = 0; s < slices; ++s) {
    const double2 v = partial[((int64_t)om * slices + s) * T.n_omega + f];
    re += v.x;
    im += v.y;
  }
  P.spectrum[2 * idx] = re;
  P.spectrum[2 * idx + 1] = im;
  if (f == 0) {
    P.charge[om] = re;
    int portions = 0, evaluated = 0;
    for (int s = 0; s < slices; ++s) {
      portions += counts[2 * ((int64_t)om * slices + s)];
      evaluated += counts[2 * ((int64_t)om * slices + s) + 1];
    }
    P.portions[2 * om] = portions;
    P.portions[2 * om + 1] = evaluated;
  }
}

int near_slices(const lh_near_problem& P) {
  const int s = (P.n_elements + kNearElementsPerSlice - 1) / kNearElementsPerSlice;
  return std::max(1, std::min(kNearMaxSlices, s));
}

size_t near_workspace(const lh_near_table& T, const lh_near_problem& P) {
  const size_t cells = (size_t)P.n_om * near_slices(P);
  return ((cells * T.n_omega * sizeof(double2) + 255) & ~size_t(255)) + cells * 2 * sizeof(int);
}

bool near_valid(const lh_near_table& T, const lh_near_problem& P) {
  if (T.n_lambda < 1 || T.n_lambda > kNearLam || T.degree < 0 || T.degree > kNearDeg ||
      T.acc_degree < 0 || T.acc_degree > kNearOut || T.n_pairs < 1 || T.n_pairs > kNearPairs ||
      T.n_omega < 1 || T.n_omega > kNearOmega || T.gauss_order < 1 || T.gauss_order > kNearGauss)
    return false;
  if (!T.coef || !T.absorption || !T.speed || !T.omega || !T.pair_lambda || !T.pair_mu ||
      !T.alpha || !T.start_norm || !T.wavelength_nm || !T.phase_index || !T.spectral_weight ||
      !T.gauss_x || !T.gauss_w)
    return false;
  if (!(T.panel_m > 0.0) || !(T.log_r1 > T.log_r0) || !(T.radial_high > 0.0)) return false;
  if (P.n_om < 0 || P.n_om > 65535 || P.n_elements < 0) return false;
  if (!(P.radius_m > 0.0) || P.radius_m > exp(T.log_r0) * (1.0 + 1e-9)) return false;
  if (P.n_om > 0 && (!P.om_pos || !P.om_look || !P.om_area || !P.time_origin_ns ||
                     !P.spectrum || !P.charge || !P.portions))
    return false;
  if (P.n_elements > 0 && (!P.start_m || !P.direction || !P.length_m || !P.coefficient0 ||
                           !P.coefficient2 || !P.beta || !P.start_ns || !P.end_ns))
    return false;
  return true;
}

int near_launch(const lh_near_table& T, const lh_near_problem& P, void* ws, size_t ws_bytes,
                cudaStream_t s) {
  if (!near_valid(T, P)) return LH_EINVAL;
  if (P.n_om == 0) return LH_OK;
  if (!ws || ws_bytes < near_workspace(T, P)) return LH_ENOMEM;
  const int slices = near_slices(P);
  const int per_slice = std::max(1, (P.n_elements + slices - 1) / slices);
  const size_t cells = (size_t)P.n_om * slices;
  double2* partial = static_cast<double2*>(ws);
  int* counts = reinterpret_cast<int*>(static_cast<uint8_t*>(ws) +
                                       ((cells * T.n_omega * sizeof(double2) + 255) & ~size_t(255)));
  const size_t smem = near_smem(T) + 16;
  if (smem > 48 * 1024 &&
      cudaFuncSetAttribute(near_field_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)smem) != cudaSuccess)
    return LH_ECUDA;
  near_field_kernel<<<dim3(P.n_om, slices), kNearThreads, smem, s>>>(T, P, slices, per_slice,
                                                                     partial, counts);
  const int64_t outs = (int64_t)P.n_om * T.n_omega;
  near_reduce_kernel<<<(unsigned)((outs + 255) / 256), 256, 0, s>>>(T, P, slices, partial, counts);
  return cudaGetLastError() == cudaSuccess ? LH_OK : LH_ECUDA;
}

}  // namespace lh

extern "C" size_t lh_near_workspace_bytes(const lh_near_table* t, const lh_near_problem* p) {
  if (!t || !p || !lh::near_valid(*t, *p)) return 0;
  return lh::near_workspace(*t, *p);
}

extern "C" int lh_near_field(const lh_near_table* t, const lh_near_problem* p, void* workspace,
                             size_t workspace_bytes, void* stream) {
  if (!t || !p) return LH_EINVAL;
  return lh::near_launch(*t, *p, workspace, workspace_bytes, static_cast<cudaStream_t>(stream));
}

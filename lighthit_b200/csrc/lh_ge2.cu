// Order >=2: contraction of axial-basis source moments with band-folded RTE
// kernels (reference _shower_basis.py:894-1050, apply_multi_spectral
// :1126-1198, shower/ge2.py:99-119).
//
// For an OM d and a basis point c at distance r (interval j of the log-r
// grid, offset t) the reference sums, per band lambda and frequency w,
//
//   N_d(w) += s_lambda(r) e^{i w r / v_lambda}
//             sum_l sum_a rot_l[a](w) * sum_p D_p[a] cubic_{lambda j l p}(t, w),
//   rot_l[a](w) = sum_b erow_l[a][b] ch_lambda[c][l, b](w).
//
// Exchanging the sums over a and b gives
//
//   N_d(w) += s e^{i w r/v} sum_l sum_b ch[c][l,b](w) sum_p F_l[b][p] cubic_{j l p}(t, w),
//   F_l[b][p] = sum_a erow_l[a][b] D_p[a],
//
// where F (nch x pairs real numbers per (d, c)) carries all the geometry:
// Wigner small-d rotation, azimuthal rotation, detector harmonics and the
// acceptance coefficients. ge2_geometry_kernel forms F in float64 once per
// (d, c); ge2_apply_kernel runs the float32 contraction with one thread per
// (band, frequency); ge2_reduce_kernel sums the point chunks in a fixed order
// (identical results alone or in a batch) and applies the emission-time phase.
#include <algorithm>

#include "lh_common.cuh"
#include "lh_timing.cuh"
#include "lh_harmonics.cuh"

namespace lh {

constexpr int kGe2Degree = 16;   // source/kernel degree bound
constexpr int kGe2Out = 4;       // acceptance (detector) degree bound
constexpr int kGe2M = 4;         // azimuthal degree bound
constexpr int kGe2Chunk = 32;    // points per partial sum

// One thread per (OM, point): radius, interval, band scales and F.
LH_DEVICE void ge2_geometry_body(const lh_ge2_table& T, const lh_ge2_problem& P, int64_t idx,
                                 int* g_j, float* g_t, double* g_r, float* g_scale, float* g_F) {
  const int64_t total = (int64_t)P.n_om * P.n_points;
  if (idx >= total) return;
  const int d = (int)(idx / P.n_points), c = (int)(idx % P.n_points);
  const double dx = P.receivers[3 * d] - P.points[3 * c];
  const double dy = P.receivers[3 * d + 1] - P.points[3 * c + 1];
  const double dz = P.receivers[3 * d + 2] - P.points[3 * c + 2];
  const double radius = sqrt(dx * dx + dy * dy + dz * dz);
  g_r[idx] = radius;
  if (!(radius >= P.radial_low && radius <= P.radial_high)) {
    g_j[idx] = -1;
    return;
  }
  const int L = T.degree, A = T.acc_degree, M = T.max_m, W = 2 * A + 1, NP = T.n_pairs;
  double cosine = dz / radius;
  cosine = cosine > 1.0 ? 1.0 : (cosine < -1.0 ? -1.0 : cosine);
  const double phi = atan2(dy, dx);
  const double tr = sqrt(dx * dx + dy * dy);
  const double sine = tr / radius;
  const double cp = tr == 0.0 ? 1.0 : dx / tr;
  const double sp = tr == 0.0 ? 0.0 : dy / tr;
  double cosn[kGe2M + 1], sinn[kGe2M + 1];
  for (int n = 0; n <= M; ++n) {
    cosn[n] = cos(n * phi);
    sinn[n] = sin(n * phi);
  }
  const double lx = P.looks[3 * d], ly = P.looks[3 * d + 1], lz = P.looks[3 * d + 2];
  const double a1 = cosine * cp * lx + cosine * sp * ly - sine * lz;
  const double a2 = -sp * lx + cp * ly;
  const double a3 = sine * cp * lx + sine * sp * ly + cosine * lz;
  double det[(kGe2Out + 1) * (kGe2Out + 1)];
  real_harmonics(a1, a2, a3, A, det);
  // pair weights D_p[a]: alpha_lam Y[lam, +mu] at a = A + mu, alpha Y[lam, -mu] at A - mu
  // Wigner d^l_(mu nu): wig[l][nu + A][mu], mu = 0..M, by recurrence in l (:51-87)
  double wig[kGe2Degree + 1][2 * kGe2Out + 1][kGe2M + 1];
  for (int l = 0; l <= L; ++l)
    for (int a = 0; a < W; ++a)
      for (int m = 0; m <= M; ++m) wig[l][a][m] = 0.0;
  const double hc = sqrt((1.0 + cosine) / 2.0), hs = sqrt((1.0 - cosine) / 2.0);
  for (int nu = -A; nu <= A; ++nu) {
    for (int mu = 0; mu <= M; ++mu) {
      const int start = abs(nu) > mu ? abs(nu) : mu;
      if (start > L) continue;
      double prev = 0.0, cur = wigner_start(start, mu, nu, hc, hs, T.start_norm, T.jmax);
      wig[start][nu + A][mu] = cur;
      for (int l = start; l < L; ++l) {
        double value;
        if (l == 0) value = cosine * cur;
        else {
          double lower = (double)(l * l - mu * mu) * (double)(l * l - nu * nu);
          lower = lower > 0.0 ? sqrt(lower) : 0.0;
          const double upper = sqrt((double)((l + 1) * (l + 1) - mu * mu) *
                                    (double)((l + 1) * (l + 1) - nu * nu));
          value = ((2 * l + 1) * (l * (l + 1) * cosine - mu * nu) * cur - (l + 1) * lower * prev) /
                  (l * upper);
        }
        prev = cur;
        cur = value;
        wig[l + 1][nu + A][mu] = cur;
      }
    }
  }
  // F_l[b][p] for every kept source channel (row = starts[l] + (b - M + keep))
  float* F = g_F + idx * (int64_t)T.nch * NP;
  const double root2 = sqrt(2.0);
  for (int l = 0; l <= L; ++l) {
    double erow[2 * kGe2Out + 1][2 * kGe2M + 1];
    for (int a = 0; a < W; ++a)
      for (int b = 0; b <= 2 * M; ++b) erow[a][b] = 0.0;
    erow[A][M] = wig[l][A][0];
    const int top_n = l < M ? l : M, top_p = l < A ? l : A;
    for (int n = 1; n <= top_n; ++n) {
      const double base = root2 * par(n) * wig[l][A][n];
      erow[A][M + n] = base * cosn[n];
      erow[A][M - n] = base * sinn[n];
    }
    for (int pp = 1; pp <= top_p; ++pp) {
      erow[A + pp][M] = root2 * par(pp) * wig[l][A + pp][0];
      for (int n = 1; n <= top_n; ++n) {
        const double cross = par(pp) * wig[l][A + pp][n];
        const double straight = wig[l][A - pp][n];
        const double cc = par(n) * (cross + straight), ss = par(n) * (cross - straight);
        erow[A + pp][M + n] = cc * cosn[n];
        erow[A + pp][M - n] = cc * sinn[n];
        erow[A - pp][M + n] = -ss * sinn[n];
        erow[A - pp][M - n] = ss * cosn[n];
      }
    }
    const int keep = top_n;
    for (int b = M - keep; b <= M + keep; ++b) {
      const int row = T.starts[l] + keep + (b - M);
      for (int p = 0; p < NP; ++p) {
        const int lam = T.pair_lambda[p], mup = T.pair_mu[p];
        double f = 0.0;
        if (mup <= top_p) {
          const int cidx = lam * lam + lam;
          const double pos = T.alpha[lam] * det[cidx + mup];
          const double neg = mup ? T.alpha[lam] * det[cidx - mup] : 0.0;
          if (neg != 0.0) f += erow[A - mup][b] * neg;
          if (pos != 0.0) f += erow[A + mup][b] * pos;
        }
        F[row * NP + p] = (float)f;
      }
    }
  }
  const double logr = log(radius);
  int j = bin_right(T.log_r, T.n_intervals + 1, logr);
  j = j < 0 ? 0 : (j > T.n_intervals - 1 ? T.n_intervals - 1 : j);
  g_j[idx] = j;
  g_t[idx] = (float)(logr - T.log_r[j]);
  for (int lam = 0; lam < T.n_bands; ++lam)
    g_scale[(int64_t)lam * total + idx] =
        (float)(P.out_scale[(int64_t)lam * P.n_om + d] * exp(-T.absorption[lam] * radius) /
                (4 * kPi * radius * radius));
}

// Grid (OM, point chunk); thread = (band, frequency). Partial sums per chunk.
LH_DEVICE void ge2_apply_body(const lh_ge2_table& T, const lh_ge2_problem& P, int d, int chunk,
                              int chunks, const int* g_j, const float* g_t, const double* g_r,
                              const float* g_scale, const float* g_F, double2* partial) {
  extern __shared__ float s_F[];  // [kGe2Chunk][nch*NP] for the chunk's points
  const int c0 = chunk * kGe2Chunk;
  const int c1 = min(P.n_points, c0 + kGe2Chunk);
  const int NP = T.n_pairs, nch = T.nch, Wn = P.n_omega;
  const int64_t total = (int64_t)P.n_om * P.n_points;
  const int64_t base = (int64_t)d * P.n_points;
  const int fsz = nch * NP;
  for (int i = threadIdx.x; i < (c1 - c0) * fsz; i += blockDim.x)
    s_F[i] = g_F[(base + c0) * fsz + i];
  __syncthreads();
  const int items = T.n_bands * Wn;
  if (2 * items <= (int)blockDim.x) {
    // few (band, frequency) items (zero-frequency applies): one thread per
    // (point, item), the chunk's point values summed in point order
    float2* s_val = reinterpret_cast<float2*>(s_F + kGe2Chunk * fsz);  // [point][item]
    const int n = c1 - c0;
    for (int k = threadIdx.x; k < n * items; k += blockDim.x) {
      const int u = k / items, item = k - u * items;
      const int lam = item / Wn, w = item % Wn;
      const int64_t idx = base + c0 + u;
      const int j = g_j[idx];
      float2 value = make_float2(0.f, 0.f);
      if (j >= 0) {
        const float t = g_t[idx];
        const float* F = s_F + u * fsz;
        const float2* ch = reinterpret_cast<const float2*>(P.channels) +
                           (((int64_t)lam * P.n_points + c0 + u) * nch) * P.n_omega_channels;
        float pr = 0.f, pi = 0.f;
        for (int l = 0; l <= T.degree; ++l) {
          float rr[8], ri[8];
          const float2* cf = reinterpret_cast<const float2*>(T.coef) +
                             ((((int64_t)lam * T.n_intervals + j) * (T.degree + 1) + l) * NP * 4) *
                                 T.n_omega + w;
          for (int p = 0; p < NP; ++p) {
            const float2 k0 = cf[(p * 4 + 0) * T.n_omega], k1 = cf[(p * 4 + 1) * T.n_omega];
            const float2 k2 = cf[(p * 4 + 2) * T.n_omega], k3 = cf[(p * 4 + 3) * T.n_omega];
            rr[p] = fmaf(fmaf(fmaf(k0.x, t, k1.x), t, k2.x), t, k3.x);
            ri[p] = fmaf(fmaf(fmaf(k0.y, t, k1.y), t, k2.y), t, k3.y);
          }
          const int keep = l < T.max_m ? l : T.max_m;
          for (int row = T.starts[l]; row < T.starts[l] + 2 * keep + 1; ++row) {
            float gr = 0.f, gi = 0.f;
            for (int p = 0; p < NP; ++p) {
              const float f = F[row * NP + p];
              gr = fmaf(f, rr[p], gr);
              gi = fmaf(f, ri[p], gi);
            }
            const float2 x = ch[row * P.n_omega_channels + w];
            pr += x.x * gr - x.y * gi;
            pi += x.x * gi + x.y * gr;
          }
        }
        const float sc = g_scale[(int64_t)lam * total + idx];
        float sv = 0.f, cv = 1.f;
        if (T.flight) {
          const double turns = T.omega[w] * g_r[idx] / T.speed[lam] * (1.0 / (2 * kPi));
          sincospif(2.f * (float)(turns - rint(turns)), &sv, &cv);
        }
        value = make_float2(sc * (pr * cv - pi * sv), sc * (pr * sv + pi * cv));
      }
      s_val[u * items + item] = value;
    }
    __syncthreads();
    for (int item = threadIdx.x; item < items; item += blockDim.x) {
      const int lam = item / Wn, w = item % Wn;
      float acc_re = 0.f, acc_im = 0.f;
      for (int u = 0; u < n; ++u) {
        acc_re += s_val[u * items + item].x;
        acc_im += s_val[u * items + item].y;
      }
      partial[(((int64_t)d * chunks + chunk) * T.n_bands + lam) * Wn + w] =
          make_double2(acc_re, acc_im);
    }
    return;
  }
  for (int item = threadIdx.x; item < items; item += blockDim.x) {
    const int lam = item / Wn, w = item % Wn;
    const double om = T.omega[w];
    float acc_re = 0.f, acc_im = 0.f;
    for (int c = c0; c < c1; ++c) {
      const int64_t idx = base + c;
      const int j = g_j[idx];
      if (j < 0) continue;
      const float t = g_t[idx];
      const float* F = s_F + (c - c0) * fsz;
      const float2* ch = reinterpret_cast<const float2*>(P.channels) +
                         (((int64_t)lam * P.n_points + c) * nch) * P.n_omega_channels;
      float pr = 0.f, pi = 0.f;
      for (int l = 0; l <= T.degree; ++l) {
        // radial cubic of every pair at (lam, j, l, w)
        float rr[8], ri[8];
        const float2* cf = reinterpret_cast<const float2*>(T.coef) +
                           ((((int64_t)lam * T.n_intervals + j) * (T.degree + 1) + l) * NP * 4) *
                               T.n_omega + w;
        for (int p = 0; p < NP; ++p) {
          const float2 k0 = cf[(p * 4 + 0) * T.n_omega], k1 = cf[(p * 4 + 1) * T.n_omega];
          const float2 k2 = cf[(p * 4 + 2) * T.n_omega], k3 = cf[(p * 4 + 3) * T.n_omega];
          rr[p] = fmaf(fmaf(fmaf(k0.x, t, k1.x), t, k2.x), t, k3.x);
          ri[p] = fmaf(fmaf(fmaf(k0.y, t, k1.y), t, k2.y), t, k3.y);
        }
        const int keep = l < T.max_m ? l : T.max_m;
        for (int row = T.starts[l]; row < T.starts[l] + 2 * keep + 1; ++row) {
          float gr = 0.f, gi = 0.f;
          for (int p = 0; p < NP; ++p) {
            const float f = F[row * NP + p];
            gr = fmaf(f, rr[p], gr);
            gi = fmaf(f, ri[p], gi);
          }
          const float2 x = ch[row * P.n_omega_channels + w];
          pr += x.x * gr - x.y * gi;
          pi += x.x * gi + x.y * gr;
        }
      }
      // band scale and flight phase e^{i w r / v}
      const float sc = g_scale[(int64_t)lam * total + idx];
      float sv = 0.f, cv = 1.f;
      if (T.flight) {
        const double turns = om * g_r[idx] / T.speed[lam] * (1.0 / (2 * kPi));
        sincospif(2.f * (float)(turns - rint(turns)), &sv, &cv);
      }
      acc_re += sc * (pr * cv - pi * sv);
      acc_im += sc * (pr * sv + pi * cv);
    }
    partial[(((int64_t)d * chunks + chunk) * T.n_bands + lam) * Wn + w] =
        make_double2(acc_re, acc_im);
  }
}

// result[d][w] = e^{i w ref} * sum over chunks and bands, fixed order.
LH_DEVICE void ge2_reduce_body(const lh_ge2_table& T, const lh_ge2_problem& P, int64_t idx,
                               int chunks, const double2* partial) {
  const int Wn = P.n_omega;
  if (idx >= (int64_t)P.n_om * Wn) return;
  const int d = (int)(idx / Wn), w = (int)(idx % Wn);
  double re = 0.0, im = 0.0;
  for (int ch = 0; ch < chunks; ++ch)
    for (int lam = 0; lam < T.n_bands; ++lam) {
      const double2 v = partial[(((int64_t)d * chunks + ch) * T.n_bands + lam) * Wn + w];
      re += v.x;
      im += v.y;
    }
  const double ang = T.omega[w] * P.reference_ns;
  const double c = cos(ang), s = sin(ang);
  P.result[2 * idx] = re * c - im * s;
  P.result[2 * idx + 1] = re * s + im * c;
}

// One problem: grids over its own sizes.
__global__ void ge2_geometry_kernel(lh_ge2_table T, lh_ge2_problem P, int* g_j, float* g_t,
                                    double* g_r, float* g_scale, float* g_F) {
  ge2_geometry_body(T, P, blockIdx.x * (int64_t)blockDim.x + threadIdx.x, g_j, g_t, g_r, g_scale,
                    g_F);
}

__global__ void __launch_bounds__(256, 4)
ge2_apply_kernel(lh_ge2_table T, lh_ge2_problem P, const int* g_j,
                                 const float* g_t, const double* g_r, const float* g_scale,
                                 const float* g_F, double2* partial) {
  ge2_apply_body(T, P, blockIdx.x, blockIdx.y, gridDim.y, g_j, g_t, g_r, g_scale, g_F, partial);
}

__global__ void ge2_reduce_kernel(lh_ge2_table T, lh_ge2_problem P, int chunks,
                                  const double2* partial) {
  ge2_reduce_body(T, P, blockIdx.x * (int64_t)blockDim.x + threadIdx.x, chunks, partial);
}

// Many problems (events) in one launch: blockIdx.z (or .y) selects the problem,
// whose workspace regions start at its pair / partial offsets.
struct Ge2Slot {
  lh_ge2_problem P;
  int64_t pair_offset;     // sum of n_om * n_points of the earlier problems
  int64_t partial_offset;  // sum of n_om * chunks * n_bands * n_omega of the earlier problems
  int32_t chunks;
};

struct Ge2Arrays {
  int* g_j;
  float* g_t;
  double* g_r;
  float* g_scale;  // [problem][band][pairs]
  float* g_F;
  double2* partial;
};

__global__ void ge2_geometry_batch_kernel(lh_ge2_table T, const Ge2Slot* slots, Ge2Arrays A) {
  const Ge2Slot& S = slots[blockIdx.y];
  const int64_t o = S.pair_offset;
  ge2_geometry_body(T, S.P, blockIdx.x * (int64_t)blockDim.x + threadIdx.x, A.g_j + o, A.g_t + o,
                    A.g_r + o, A.g_scale + o * T.n_bands, A.g_F + o * T.nch * T.n_pairs);
}

__global__ void __launch_bounds__(256, 4)
ge2_apply_batch_kernel(lh_ge2_table T, const Ge2Slot* slots, Ge2Arrays A) {
  const Ge2Slot& S = slots[blockIdx.z];
  if ((int)blockIdx.x >= S.P.n_om || (int)blockIdx.y >= S.chunks) return;
  const int64_t o = S.pair_offset;
  ge2_apply_body(T, S.P, blockIdx.x, blockIdx.y, S.chunks, A.g_j + o, A.g_t + o, A.g_r + o,
                 A.g_scale + o * T.n_bands, A.g_F + o * T.nch * T.n_pairs,
                 A.partial + S.partial_offset);
}

__global__ void ge2_reduce_batch_kernel(lh_ge2_table T, const Ge2Slot* slots, Ge2Arrays A) {
  const Ge2Slot& S = slots[blockIdx.y];
  ge2_reduce_body(T, S.P, blockIdx.x * (int64_t)blockDim.x + threadIdx.x, S.chunks,
                  A.partial + S.partial_offset);
}

int ge2_chunks(const lh_ge2_problem& P) { return (P.n_points + kGe2Chunk - 1) / kGe2Chunk; }

// Shared memory of the apply kernels (256 threads): the chunk's F rows, then
// the point values of the few-item path when a problem takes it (at most 128
// (band, frequency) items).
size_t ge2_apply_smem(const lh_ge2_table& T, int items) {
  return (size_t)kGe2Chunk * T.nch * T.n_pairs * sizeof(float) +
         (2 * items <= 256 ? (size_t)kGe2Chunk * items * sizeof(float2) : 0);
}

size_t ge2_workspace(const lh_ge2_table& T, const lh_ge2_problem& P) {
  const size_t pairs = (size_t)P.n_om * P.n_points;
  const size_t chunks = (size_t)ge2_chunks(P);
  auto up = [](size_t x) { return (x + 255) & ~size_t(255); };
  return up(pairs * 4) + up(pairs * 4) + up(pairs * 8) + up(pairs * T.n_bands * 4) +
         up(pairs * T.nch * T.n_pairs * 4) +
         up((size_t)P.n_om * chunks * T.n_bands * P.n_omega * sizeof(double2));
}

int ge2_launch(const lh_ge2_table& T, const lh_ge2_problem& P, void* ws, cudaStream_t s) {
  const size_t pairs = (size_t)P.n_om * P.n_points;
  auto up = [](size_t x) { return (x + 255) & ~size_t(255); };
  uint8_t* p = static_cast<uint8_t*>(ws);
  int* g_j = reinterpret_cast<int*>(p); p += up(pairs * 4);
  float* g_t = reinterpret_cast<float*>(p); p += up(pairs * 4);
  double* g_r = reinterpret_cast<double*>(p); p += up(pairs * 8);
  float* g_scale = reinterpret_cast<float*>(p); p += up(pairs * T.n_bands * 4);
  float* g_F = reinterpret_cast<float*>(p); p += up(pairs * T.nch * T.n_pairs * 4);
  double2* partial = reinterpret_cast<double2*>(p);
  ge2_geometry_kernel<<<(unsigned)((pairs + 127) / 128), 128, 0, s>>>(T, P, g_j, g_t, g_r, g_scale, g_F);
  const int chunks = ge2_chunks(P);
  const size_t smem = ge2_apply_smem(T, T.n_bands * P.n_omega);
  if (smem > 48 * 1024)
    cudaFuncSetAttribute(ge2_apply_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  ge2_apply_kernel<<<dim3(P.n_om, chunks), 256, smem, s>>>(T, P, g_j, g_t, g_r, g_scale, g_F,
                                                            partial);
  const int64_t outs = (int64_t)P.n_om * P.n_omega;
  ge2_reduce_kernel<<<(unsigned)((outs + 255) / 256), 256, 0, s>>>(T, P, chunks, partial);
  return cudaGetLastError() == cudaSuccess ? LH_OK : LH_ECUDA;
}

size_t ge2_slot_size() { return sizeof(Ge2Slot); }

size_t ge2_batch_workspace(const lh_ge2_table& T, const lh_ge2_problem* P, int32_t n) {
  size_t pairs = 0, partial = 0;
  for (int i = 0; i < n; ++i) {
    pairs += (size_t)P[i].n_om * P[i].n_points;
    partial += (size_t)P[i].n_om * ge2_chunks(P[i]) * T.n_bands * P[i].n_omega;
  }
  auto up = [](size_t x) { return (x + 255) & ~size_t(255); };
  return up(sizeof(Ge2Slot) * (size_t)n) + up(pairs * 4) + up(pairs * 4) + up(pairs * 8) +
         up(pairs * T.n_bands * 4) + up(pairs * T.nch * T.n_pairs * 4) +
         up(partial * sizeof(double2));
}

// The slot table is staged in `host_slots` (caller memory, pinned when the call
// should not wait) and copied to the workspace on the stream.
int ge2_batch_launch(const lh_ge2_table& T, const lh_ge2_problem* P, int32_t n, void* ws,
                     void* host_slots, cudaStream_t s) {
  auto up = [](size_t x) { return (x + 255) & ~size_t(255); };
  Ge2Slot* hs = static_cast<Ge2Slot*>(host_slots);
  size_t pairs = 0, partial = 0;
  int max_om = 0, max_chunks = 0;
  int64_t max_pairs = 0, max_outs = 0;
  for (int i = 0; i < n; ++i) {
    hs[i].P = P[i];
    hs[i].pair_offset = (int64_t)pairs;
    hs[i].partial_offset = (int64_t)partial;
    hs[i].chunks = ge2_chunks(P[i]);
    const int64_t pp = (int64_t)P[i].n_om * P[i].n_points;
    pairs += pp;
    partial += (size_t)P[i].n_om * hs[i].chunks * T.n_bands * P[i].n_omega;
    max_om = std::max(max_om, P[i].n_om);
    max_chunks = std::max(max_chunks, hs[i].chunks);
    max_pairs = std::max(max_pairs, pp);
    max_outs = std::max(max_outs, (int64_t)P[i].n_om * P[i].n_omega);
  }
  uint8_t* p = static_cast<uint8_t*>(ws);
  Ge2Slot* slots = reinterpret_cast<Ge2Slot*>(p); p += up(sizeof(Ge2Slot) * (size_t)n);
  Ge2Arrays A;
  A.g_j = reinterpret_cast<int*>(p); p += up(pairs * 4);
  A.g_t = reinterpret_cast<float*>(p); p += up(pairs * 4);
  A.g_r = reinterpret_cast<double*>(p); p += up(pairs * 8);
  A.g_scale = reinterpret_cast<float*>(p); p += up(pairs * T.n_bands * 4);
  A.g_F = reinterpret_cast<float*>(p); p += up(pairs * T.nch * T.n_pairs * 4);
  A.partial = reinterpret_cast<double2*>(p);
  if (cudaMemcpyAsync(slots, hs, sizeof(Ge2Slot) * (size_t)n, cudaMemcpyHostToDevice, s) !=
      cudaSuccess)
    return LH_ECUDA;
  if (max_outs == 0) return LH_OK;
  if (max_pairs > 0) {  // problems without points reduce nothing: their results are zero
    ge2_geometry_batch_kernel<<<dim3((unsigned)((max_pairs + 127) / 128), n), 128, 0, s>>>(
        T, slots, A);
    size_t smem = 0;
    for (int i = 0; i < n; ++i) smem = std::max(smem, ge2_apply_smem(T, T.n_bands * P[i].n_omega));
    if (smem > 48 * 1024)
      cudaFuncSetAttribute(ge2_apply_batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)smem);
    {
      lh::TimedLaunch timed_launch(LH_KT_GE2_APPLY, s);
      ge2_apply_batch_kernel<<<dim3(max_om, max_chunks, n), 256, smem, s>>>(T, slots, A);
    }
  }
  ge2_reduce_batch_kernel<<<dim3((unsigned)((max_outs + 255) / 256), n), 256, 0, s>>>(T, slots, A);
  return cudaGetLastError() == cudaSuccess ? LH_OK : LH_ECUDA;
}


// ------------------------------------------------------------------ tensor cores
// The contraction on tcgen05 (BF16 operands, FP32 accumulation in TMEM). In
// the split mode every operand is the sum of three BF16 parts (hi + mid + lo,
// 24 significant bits, as float32) and six products are accumulated: hi hi,
// hi mid, mid hi, hi lo, lo hi, mid mid (the rest lie below float32's
// rounding); the single mode multiplies the hi parts.
//
// For interval j and kernel degree l the band-folded coefficients form a real
// matrix A_jl[(band, w, part)][(pair p, power q)] (part: real or imaginary
// coefficient; K = 4 x pairs <= 32), and a (OM, point) pair of interval j
// forms B[(channel row r of degree l)][(p, q)] = F[r][p] t^(3 - q). The
// product X = A_jl B^T holds, for every source channel row of the pair and
// every (band, w), the row's F contracted with the cubic radial kernels. The
// epilogue multiplies each X entry by the row's source channel (complex, per
// band and frequency) and sums rows and degrees in registers; then the pair's
// band scale and flight phase give its spectrum, written per pair and summed
// over points by ge2_tc_reduce_kernel in a fixed order.
//
// Layout: M = (band, w) rows in H <= 2 halves of 128 TMEM lanes, each half as
// a real and an imaginary accumulator; N = channel row x pair columns
// (column r * kTcSub + i for pair i of a sub-tile). Pairs are bucketed by
// interval (counting sort); a CTA takes up to kTcPairs pairs of one interval,
// streams A_jl with one bulk copy per degree (double-buffered) and keeps the
// pairs' accumulators in registers across degrees.
constexpr int kTcSub = 8;                   // pairs per MMA sub-tile
constexpr int kTcSubs = 4;                  // sub-tiles per CTA tile
constexpr int kTcPairs = kTcSub * kTcSubs;  // pairs per CTA tile
constexpr int kTcThreads = 256;
constexpr int kTcK = 32;                                  // K columns (pairs x 4 <= 32)
constexpr uint32_t kTcTileBytes = 128u * kTcK * 2u;       // one 128 x 32 BF16 operand tile
constexpr int kTcParts = 3;                               // BF16 parts of a split operand

struct Ge2TcArgs {
  const Ge2Slot* slots;
  Ge2Arrays A;
  const uint8_t* packed;        // [interval][degree] blocks: [hi, lo][half][re, im] tiles
  const int32_t* sorted;        // global pair ids bucketed by interval
  const int32_t* sorted_slot;   // their problems
  const int32_t* bucket_start;  // [n_intervals + 1]
  const int32_t* tile_start;    // [n_intervals + 1]
  float2* partial;              // [global pair][band * n_omega + w]
  int32_t* status;
  int passes;                   // 6 split-BF16, 1 BF16
  int halves;                   // H: ceil(bands x omega / 128)
  int n_pad_max;                // widest sub-tile (16-column multiple)
  int tmem_cols;                // 256 (two CTAs per SM) or 512
  int a_buffers;                // 1 with two CTAs per SM, 2 (prefetch) with one
};

// (A part, B part) of each product of the split mode, largest first.
__constant__ int kTcPassA[6] = {0, 0, 1, 0, 2, 1};
__constant__ int kTcPassB[6] = {0, 1, 0, 2, 0, 1};

struct Ge2TcPair {
  const float2* channels;  // the point's channel block, band 0, channel row 0, w 0
  int64_t band_stride;     // float2 elements between bands
  int64_t scale_at;        // g_scale index of band 0
  int64_t scale_stride;    // between bands
  int32_t pair;            // global pair id, -1 for an empty place
  int32_t omega_stride;    // float2 elements between channel rows
  float t;
  float pad;
};

// Whether a table takes the tensor-core path, and its widest sub-tile.
bool ge2_tc_supported(const lh_ge2_table& T, int& halves, int& n_pad_max) {
  const int M = T.n_bands * T.n_omega;
  const int rows_max = 2 * std::min(T.degree, T.max_m) + 1;
  halves = (M + 127) / 128;
  n_pad_max = (rows_max * kTcSub + 15) & ~15;
  return M <= 256 && 4 * T.n_pairs <= kTcK && 2 * halves * n_pad_max <= 512;
}

size_t ge2_tc_block_bytes(const lh_ge2_table& T, int halves) {
  (void)T;
  return (size_t)kTcParts * halves * 2 * kTcTileBytes;
}

// x = hi + mid + lo, each BF16 (24 significant bits together).
LH_DEVICE void split3_bf16(float x, __nv_bfloat16& hi, __nv_bfloat16& mid, __nv_bfloat16& lo) {
  hi = __float2bfloat16_rn(x);
  const float r = x - __bfloat162float(hi);
  mid = __float2bfloat16_rn(r);
  lo = __float2bfloat16_rn(r - __bfloat162float(mid));
}

// Packs the folded coefficients into the operand tiles (no swizzle, K-major
// 8 x 16-byte core matrices), hi, mid and lo parts.
__global__ void ge2_tc_pack_kernel(const lh_ge2_table T, int halves, __nv_bfloat16* out) {
  const int L1 = T.degree + 1, W = T.n_omega, M = T.n_bands * W;
  const int64_t per_block = (int64_t)halves * 2 * 128 * kTcK;
  const int64_t total = (int64_t)T.n_intervals * L1 * per_block;
  const int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (idx >= total) return;
  const int k = (int)(idx % kTcK);
  const int m = (int)((idx / kTcK) % 128);
  const int part = (int)((idx / (kTcK * 128)) % 2);
  const int h = (int)((idx / (kTcK * 256)) % halves);
  const int64_t jl = idx / per_block;
  const int l = (int)(jl % L1), j = (int)(jl / L1);
  const int flat = h * 128 + m;
  float v = 0.f;
  if (flat < M && k < 4 * T.n_pairs) {
    const int lam = flat / W, w = flat % W, pp = k >> 2, q = k & 3;
    const float2 c = reinterpret_cast<const float2*>(T.coef)
        [((((int64_t)lam * T.n_intervals + j) * L1 + l) * T.n_pairs * 4 + pp * 4 + q) * W + w];
    v = part ? c.y : c.x;
  }
  __nv_bfloat16 hi, mid, lo;
  split3_bf16(v, hi, mid, lo);
  const int64_t tile = (int64_t)(h * 2 + part) * 128 * kTcK;
  const int64_t at = jl * kTcParts * per_block + tile + tile_offset(m, k);
  out[at] = hi;
  out[at + per_block] = mid;
  out[at + 2 * per_block] = lo;
}

// Bucket pass 1 and 3 over every pair of every problem, points outermost so
// that a bucket lists the OMs of one point together: count per interval, then
// place (warp-aggregated atomics).
__global__ void ge2_tc_bucket_kernel(const Ge2Slot* slots, Ge2Arrays A, int32_t* counts,
                                     int32_t* sorted, int32_t* sorted_slot, int fill) {
  const Ge2Slot& S = slots[blockIdx.y];
  const int64_t total = (int64_t)S.P.n_om * S.P.n_points;
  const int64_t rounded = (total + 31) & ~(int64_t)31;
  const int lane = threadIdx.x & 31;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < rounded;
       t += (int64_t)gridDim.x * blockDim.x) {
    int j = -1;
    int64_t idx = 0;
    if (t < total) {
      const int64_t c = t / S.P.n_om, d = t % S.P.n_om;
      idx = d * S.P.n_points + c;
      j = A.g_j[S.pair_offset + idx];
    }
    const unsigned peers = __match_any_sync(0xffffffffu, j);
    const int leader = __ffs(peers) - 1;
    int base = 0;
    if (lane == leader && j >= 0) base = atomicAdd(counts + j, __popc(peers));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (fill && j >= 0) {
      const int pos = base + __popc(peers & ((1u << lane) - 1u));
      sorted[pos] = (int32_t)(S.pair_offset + idx);
      sorted_slot[pos] = (int32_t)blockIdx.y;
    }
  }
}

// Bucket starts, tile starts (kTcPairs pairs per tile) and the fill cursors.
__global__ void ge2_tc_scan_kernel(int n_intervals, int32_t* counts, int32_t* bucket_start,
                                   int32_t* tile_start, unsigned long long* units) {
  if (threadIdx.x != 0) return;
  int32_t at = 0, tiles = 0;
  for (int j = 0; j < n_intervals; ++j) {
    const int32_t c = counts[j];
    bucket_start[j] = at;
    tile_start[j] = tiles;
    counts[j] = at;  // the fill pass counts from the bucket's start
    at += c;
    tiles += (c + kTcPairs - 1) / kTcPairs;
  }
  bucket_start[n_intervals] = at;
  tile_start[n_intervals] = tiles;
  if (units) atomicAdd(units, (unsigned long long)at);  // (OM, point) pairs in range
}

__global__ void __launch_bounds__(kTcThreads, 2)
ge2_tc_kernel(const lh_ge2_table T, const Ge2TcArgs G) {
  extern __shared__ __align__(1024) uint8_t smem[];
  const int H = G.halves;
  const int parts = G.passes > 1 ? kTcParts : 1;
  const uint32_t block_bytes = (uint32_t)kTcParts * H * 2u * kTcTileBytes;
  const uint32_t load_bytes = (uint32_t)parts * H * 2u * kTcTileBytes;
  uint8_t* s_a0 = smem;
  uint8_t* s_a1 = smem + (G.a_buffers > 1 ? load_bytes : 0);
  __nv_bfloat16* s_b = reinterpret_cast<__nv_bfloat16*>(smem + G.a_buffers * load_bytes);
  const int b_elems = G.n_pad_max * kTcK;
  Ge2TcPair* s_pair = reinterpret_cast<Ge2TcPair*>(smem + G.a_buffers * load_bytes +
                                                   (size_t)parts * b_elems * 2);
  uint64_t* bars = reinterpret_cast<uint64_t*>(s_pair + kTcPairs);  // load[2], mma
  uint32_t* s_tmem = reinterpret_cast<uint32_t*>(bars + 3);

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (tid == 0) {
    mbar_init(bars + 0, 1);
    mbar_init(bars + 1, 1);
    mbar_init(bars + 2, 1);
    fence_barrier_init();
  }
  if (warp == 0) {
    tmem_alloc(s_tmem, (uint32_t)G.tmem_cols);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *s_tmem;
  const int L1 = T.degree + 1, W = T.n_omega, M = T.n_bands * W;
  const int h = warp >> 2, quarter = warp & 3;
  const int m = h * 128 + quarter * 32 + lane;
  const bool m_ok = m < M;
  const int lam = m_ok ? m / W : 0, wq = m_ok ? m % W : 0;
  const bool reads = h < H;  // warps of a missing half read no TMEM
  const uint32_t lane_base = tmem + ((uint32_t)(quarter * 32) << 16);
  const int k_used = 4 * T.n_pairs;
  const double omega = T.omega[wq];
  const double inv_speed = 1.0 / T.speed[lam];
  uint32_t ph_load[2] = {0u, 0u}, ph_mma = 0u;
  bool failed = false, mma_pending = false;
  const int n_tiles = G.tile_start[T.n_intervals];

  for (int tile = blockIdx.x; tile < n_tiles && !failed; tile += gridDim.x) {
    int lo = 0, hi = T.n_intervals;  // the bucket: last j with tile_start[j] <= tile
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (G.tile_start[mid] <= tile) lo = mid; else hi = mid;
    }
    const int j = lo;
    const int first = G.bucket_start[j] + (tile - G.tile_start[j]) * kTcPairs;
    const int count = min(kTcPairs, G.bucket_start[j + 1] - first);
    if (tid < kTcPairs) {
      Ge2TcPair e{};
      e.pair = -1;
      if (tid < count) {
        const int g = G.sorted[first + tid];
        const Ge2Slot& S = G.slots[G.sorted_slot[first + tid]];
        const int64_t idx = g - S.pair_offset;
        const int c = (int)(idx % S.P.n_points);
        const int64_t pairs = (int64_t)S.P.n_om * S.P.n_points;
        e.pair = g;
        e.t = G.A.g_t[g];
        e.omega_stride = S.P.n_omega_channels;
        e.band_stride = (int64_t)S.P.n_points * T.nch * S.P.n_omega_channels;
        e.channels = reinterpret_cast<const float2*>(S.P.channels) +
                     (int64_t)c * T.nch * S.P.n_omega_channels;
        e.scale_at = S.pair_offset * T.n_bands + idx;
        e.scale_stride = pairs;
      }
      s_pair[tid] = e;
    }
    if (tid == 0) {  // degree 0 of this interval
      mbar_expect_tx(bars + 0, load_bytes);
      bulk_g2s(s_a0, G.packed + (size_t)j * L1 * block_bytes, load_bytes, bars + 0);
    }
    __syncthreads();
    float acc_re[kTcSubs][kTcSub], acc_im[kTcSubs][kTcSub];
#pragma unroll
    for (int s = 0; s < kTcSubs; ++s)
#pragma unroll
      for (int i = 0; i < kTcSub; ++i) acc_re[s][i] = acc_im[s][i] = 0.f;

    for (int l = 0; l < L1 && !failed; ++l) {
      const int buf = G.a_buffers > 1 ? (l & 1) : 0;
      uint8_t* s_a = buf ? s_a1 : s_a0;
      const int keep = min(l, T.max_m), nr = 2 * keep + 1, row0 = T.starts[l];
      const int n_cols = nr * kTcSub, n_pad = (n_cols + 15) & ~15;
      if (G.a_buffers > 1 && tid == 0 && l + 1 < L1) {
        // the next degree into the other buffer (its MMAs are done)
        mbar_expect_tx(bars + (buf ^ 1), load_bytes);
        bulk_g2s(buf ? s_a0 : s_a1, G.packed + ((size_t)j * L1 + l + 1) * block_bytes,
                 load_bytes, bars + (buf ^ 1));
      }
      bool ok = mbar_wait(bars + buf, ph_load[buf]);
      ph_load[buf] ^= 1u;
      if (__syncthreads_or(!ok)) { failed = true; break; }
#pragma unroll
      for (int s = 0; s < kTcSubs; ++s) {
        if (failed) continue;
        if (s * kTcSub >= count) continue;  // the same for the whole CTA
        // B of sub-tile s: column n = r * kTcSub + i, K index k = 4 p + q
        for (int e = tid; e < n_pad * kTcK; e += kTcThreads) {
          const int n = e / kTcK, k = e % kTcK;
          float v = 0.f;
          if (n < n_cols && k < k_used) {
            const Ge2TcPair& P = s_pair[s * kTcSub + n % kTcSub];
            if (P.pair >= 0) {
              const int r = n / kTcSub, pp = k >> 2, q = k & 3;
              float power = 1.f;
              for (int u = q; u < 3; ++u) power *= P.t;
              v = G.A.g_F[((int64_t)P.pair * T.nch + row0 + r) * T.n_pairs + pp] * power;
            }
          }
          __nv_bfloat16 bh, bm, bl;
          split3_bf16(v, bh, bm, bl);
          const int off = ((k >> 3) * n_pad + n) * 8 + (k & 7);
          s_b[off] = bh;
          if (parts > 1) {
            s_b[b_elems + off] = bm;
            s_b[2 * b_elems + off] = bl;
          }
        }
        fence_proxy_async();  // generic-proxy smem writes -> visible to the tensor core
        __syncthreads();
        tc_fence_after();
        if (tid == 0) {
          const uint32_t idesc = instr_desc_bf16_f32(128, n_pad);
          const uint32_t lbo_a = 128u * 16u, lbo_b = (uint32_t)n_pad * 16u;
          for (int hh = 0; hh < H; ++hh)
            for (int part = 0; part < 2; ++part) {
              const uint32_t d = tmem + (uint32_t)((hh * 2 + part) * n_pad);
              int first_mma = 1;
              for (int pass = 0; pass < G.passes; ++pass) {
                const uint8_t* pa =
                    s_a + (size_t)((kTcPassA[pass] * H + hh) * 2 + part) * kTcTileBytes;
                const uint8_t* pb =
                    reinterpret_cast<const uint8_t*>(s_b + kTcPassB[pass] * b_elems);
                for (int kk = 0; kk < kTcK / 16; ++kk) {
                  const uint64_t da = smem_desc_kmajor(pa + kk * 2 * lbo_a, lbo_a, 128);
                  const uint64_t db = smem_desc_kmajor(pb + kk * 2 * lbo_b, lbo_b, 128);
                  tc_mma_bf16(d, da, db, idesc, first_mma ? 0u : 1u);
                  first_mma = 0;
                }
              }
            }
          tc_commit(bars + 2);
        }
        mma_pending = true;
        ok = mbar_wait(bars + 2, ph_mma);
        ph_mma ^= 1u;
        if (__syncthreads_or(!ok)) { failed = true; continue; }
        mma_pending = false;
        tc_fence_after();
        if (reads) {
          for (int r = 0; r < nr; ++r) {
            float xr[kTcSub], xi[kTcSub];
            tmem_ld8(lane_base + (uint32_t)((h * 2) * n_pad + r * kTcSub), xr);
            tmem_ld8(lane_base + (uint32_t)((h * 2 + 1) * n_pad + r * kTcSub), xi);
            if (m_ok) {
#pragma unroll
              for (int i = 0; i < kTcSub; ++i) {
                const Ge2TcPair& P = s_pair[s * kTcSub + i];
                if (P.pair < 0) continue;
                const float2 ch =
                    P.channels[lam * P.band_stride + (int64_t)(row0 + r) * P.omega_stride + wq];
                acc_re[s][i] += ch.x * xr[i] - ch.y * xi[i];
                acc_im[s][i] += ch.x * xi[i] + ch.y * xr[i];
              }
            }
          }
        }
        tc_fence_before();
        __syncthreads();  // TMEM and the B tile are free for the next sub-tile
      }
      if (G.a_buffers == 1 && tid == 0 && l + 1 < L1 && !failed) {
        // one buffer: the next degree once this degree's MMAs are done
        mbar_expect_tx(bars + 0, load_bytes);
        bulk_g2s(s_a0, G.packed + ((size_t)j * L1 + l + 1) * block_bytes, load_bytes, bars + 0);
      }
    }
    // the pairs' spectra: band scale and flight phase e^{i w r / v}
    if (!failed && m_ok) {
#pragma unroll
      for (int s = 0; s < kTcSubs; ++s)
#pragma unroll
        for (int i = 0; i < kTcSub; ++i) {
          const Ge2TcPair& P = s_pair[s * kTcSub + i];
          if (P.pair < 0) continue;
          const float sc = G.A.g_scale[P.scale_at + lam * P.scale_stride];
          float sv = 0.f, cv = 1.f;
          if (T.flight) {
            const double turns = omega * G.A.g_r[P.pair] * inv_speed * (1.0 / (2 * kPi));
            sincospif(2.f * (float)(turns - rint(turns)), &sv, &cv);
          }
          G.partial[(int64_t)P.pair * M + m] =
              make_float2(sc * (acc_re[s][i] * cv - acc_im[s][i] * sv),
                          sc * (acc_re[s][i] * sv + acc_im[s][i] * cv));
        }
    }
    __syncthreads();  // the pair table is rewritten by the next tile
  }
  if (failed && tid == 0) atomicOr(reinterpret_cast<unsigned*>(G.status), LH_STATUS_TIMEOUT);
  // nothing in flight may outlive the TMEM allocation (bounded waits)
  if (mma_pending) mbar_wait(bars + 2, ph_mma);
  for (int b = 0; b < G.a_buffers; ++b)  // a prefetched degree that was never waited for
    if (failed) mbar_wait(bars + b, ph_load[b]);
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, (uint32_t)G.tmem_cols);
}

// result[d][w] = e^{i w ref} * sum over points (in order) and bands of the pairs' spectra.
__global__ void ge2_tc_reduce_kernel(const lh_ge2_table T, const Ge2Slot* slots, Ge2Arrays A,
                                     const float2* partial) {
  const Ge2Slot& S = slots[blockIdx.y];
  const int W = S.P.n_omega, M = T.n_bands * T.n_omega;
  const int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (idx >= (int64_t)S.P.n_om * W) return;
  const int d = (int)(idx / W), w = (int)(idx % W);
  double re = 0.0, im = 0.0;
  for (int c = 0; c < S.P.n_points; ++c) {
    const int64_t g = S.pair_offset + (int64_t)d * S.P.n_points + c;
    if (A.g_j[g] < 0) continue;
    for (int lam = 0; lam < T.n_bands; ++lam) {
      const float2 v = partial[g * M + lam * T.n_omega + w];
      re += v.x;
      im += v.y;
    }
  }
  const double ang = T.omega[w] * S.P.reference_ns;
  const double c = cos(ang), s = sin(ang);
  S.P.result[2 * idx] = re * c - im * s;
  S.P.result[2 * idx + 1] = re * s + im * c;
}

size_t ge2_tc_smem_bytes(int halves, int n_pad_max, int parts, int a_buffers) {
  return (size_t)a_buffers * parts * halves * 2 * kTcTileBytes +
         (size_t)parts * n_pad_max * kTcK * 2 + sizeof(Ge2TcPair) * kTcPairs +
         3 * sizeof(uint64_t) + 16;
}

size_t ge2_tc_pack_bytes(const lh_ge2_table& T) {
  int halves, n_pad_max;
  if (!ge2_tc_supported(T, halves, n_pad_max)) return 0;
  return (size_t)T.n_intervals * (T.degree + 1) * ge2_tc_block_bytes(T, halves);
}

int ge2_tc_pack(const lh_ge2_table& T, void* packed, cudaStream_t s) {
  int halves, n_pad_max;
  if (!ge2_tc_supported(T, halves, n_pad_max)) return LH_EUNSUPPORTED;
  const int64_t total = (int64_t)T.n_intervals * (T.degree + 1) * halves * 2 * 128 * kTcK;
  ge2_tc_pack_kernel<<<(unsigned)((total + 255) / 256), 256, 0, s>>>(
      T, halves, static_cast<__nv_bfloat16*>(packed));
  return cudaGetLastError() == cudaSuccess ? LH_OK : LH_ECUDA;
}

// Workspace of the tensor-core batch: the batch layout of ge2_batch_workspace,
// then the bucket arrays, the sorted pairs and the per-pair spectra.
size_t ge2_tc_workspace(const lh_ge2_table& T, const lh_ge2_problem* P, int32_t n) {
  size_t pairs = 0;
  for (int i = 0; i < n; ++i) pairs += (size_t)P[i].n_om * P[i].n_points;
  auto up = [](size_t x) { return (x + 255) & ~size_t(255); };
  return ge2_batch_workspace(T, P, n) + 3 * up(sizeof(int32_t) * (T.n_intervals + 1)) +
         2 * up(sizeof(int32_t) * pairs) + up(sizeof(float2) * pairs * T.n_bands * T.n_omega);
}

int ge2_tc_batch_launch(const lh_ge2_table& T, const lh_ge2_problem* P, int32_t n, int passes,
                        const void* packed, void* ws, void* host_slots, int32_t* status,
                        cudaStream_t s) {
  int halves, n_pad_max;
  if (!ge2_tc_supported(T, halves, n_pad_max)) return LH_EUNSUPPORTED;
  auto up = [](size_t x) { return (x + 255) & ~size_t(255); };
  Ge2Slot* hs = static_cast<Ge2Slot*>(host_slots);
  size_t pairs = 0;
  int64_t max_pairs = 0, max_outs = 0;
  for (int i = 0; i < n; ++i) {
    if (P[i].n_omega != T.n_omega) return LH_EINVAL;  // full spectra only
    hs[i].P = P[i];
    hs[i].pair_offset = (int64_t)pairs;
    hs[i].partial_offset = 0;
    hs[i].chunks = 0;
    const int64_t pp = (int64_t)P[i].n_om * P[i].n_points;
    pairs += pp;
    max_pairs = std::max(max_pairs, pp);
    max_outs = std::max(max_outs, (int64_t)P[i].n_om * P[i].n_omega);
  }
  uint8_t* p = static_cast<uint8_t*>(ws);
  Ge2Slot* slots = reinterpret_cast<Ge2Slot*>(p); p += up(sizeof(Ge2Slot) * (size_t)n);
  Ge2Arrays A;
  A.g_j = reinterpret_cast<int*>(p); p += up(pairs * 4);
  A.g_t = reinterpret_cast<float*>(p); p += up(pairs * 4);
  A.g_r = reinterpret_cast<double*>(p); p += up(pairs * 8);
  A.g_scale = reinterpret_cast<float*>(p); p += up(pairs * T.n_bands * 4);
  A.g_F = reinterpret_cast<float*>(p); p += up(pairs * T.nch * T.n_pairs * 4);
  A.partial = nullptr;
  // the CUDA-core path's chunk partials are not used here
  p = static_cast<uint8_t*>(ws) + ge2_batch_workspace(T, P, n);
  int32_t* counts = reinterpret_cast<int32_t*>(p); p += up(sizeof(int32_t) * (T.n_intervals + 1));
  int32_t* bucket_start = reinterpret_cast<int32_t*>(p); p += up(sizeof(int32_t) * (T.n_intervals + 1));
  int32_t* tile_start = reinterpret_cast<int32_t*>(p); p += up(sizeof(int32_t) * (T.n_intervals + 1));
  int32_t* sorted = reinterpret_cast<int32_t*>(p); p += up(sizeof(int32_t) * pairs);
  int32_t* sorted_slot = reinterpret_cast<int32_t*>(p); p += up(sizeof(int32_t) * pairs);
  float2* partial = reinterpret_cast<float2*>(p);
  if (cudaMemcpyAsync(slots, hs, sizeof(Ge2Slot) * (size_t)n, cudaMemcpyHostToDevice, s) !=
      cudaSuccess)
    return LH_ECUDA;
  if (max_outs == 0) return LH_OK;
  if (max_pairs == 0) {  // no points anywhere: every result is zero
    for (int i = 0; i < n; ++i)
      cudaMemsetAsync(P[i].result, 0, sizeof(double) * 2 * (size_t)P[i].n_om * P[i].n_omega, s);
    return cudaGetLastError() == cudaSuccess ? LH_OK : LH_ECUDA;
  }
  ge2_geometry_batch_kernel<<<dim3((unsigned)((max_pairs + 127) / 128), n), 128, 0, s>>>(T, slots,
                                                                                      A);
  cudaMemsetAsync(counts, 0, sizeof(int32_t) * (T.n_intervals + 1), s);
  const unsigned bucket_blocks = (unsigned)std::min<int64_t>((max_pairs + 255) / 256, 148 * 4);
  ge2_tc_bucket_kernel<<<dim3(bucket_blocks, n), 256, 0, s>>>(slots, A, counts, sorted,
                                                              sorted_slot, 0);
  ge2_tc_scan_kernel<<<1, 32, 0, s>>>(T.n_intervals, counts, bucket_start, tile_start,
                                      kernel_units() ? kernel_units() + LH_KT_GE2_TC : nullptr);
  ge2_tc_bucket_kernel<<<dim3(bucket_blocks, n), 256, 0, s>>>(slots, A, counts, sorted,
                                                              sorted_slot, 1);
  Ge2TcArgs G;
  G.slots = slots;
  G.A = A;
  G.packed = static_cast<const uint8_t*>(packed);
  G.sorted = sorted;
  G.sorted_slot = sorted_slot;
  G.bucket_start = bucket_start;
  G.tile_start = tile_start;
  G.partial = partial;
  G.status = status;
  G.passes = passes;
  G.halves = halves;
  G.n_pad_max = n_pad_max;
  // Two CTAs per SM (one overlapping the other's waits) when the accumulators
  // fit 256 TMEM columns and one coefficient buffer each fits half the shared
  // memory; otherwise one CTA per SM with 512 columns and a prefetch buffer.
  const int parts = passes > 1 ? kTcParts : 1;
  const bool two = 2 * halves * n_pad_max <= 256 &&
                   ge2_tc_smem_bytes(halves, n_pad_max, parts, 1) <= 110 * 1024;
  G.tmem_cols = two ? 256 : 512;
  G.a_buffers = two ? 1 : 2;
  const size_t smem = ge2_tc_smem_bytes(halves, n_pad_max, parts, G.a_buffers);
  if (smem > 227 * 1024) return LH_EUNSUPPORTED;
  if (cudaFuncSetAttribute(ge2_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)smem) != cudaSuccess)
    return LH_ECUDA;
  // persistent CTAs (one or two per SM); tiles beyond the grid are taken in turn
  const int64_t tile_bound = (int64_t)(pairs + kTcPairs - 1) / kTcPairs + T.n_intervals;
  const unsigned grid =
      (unsigned)std::max<int64_t>(1, std::min<int64_t>(tile_bound, two ? 2 * 148 : 148));
  {
    lh::TimedLaunch timed_launch(LH_KT_GE2_TC, s);
    ge2_tc_kernel<<<grid, kTcThreads, smem, s>>>(T, G);
  }
  ge2_tc_reduce_kernel<<<dim3((unsigned)((max_outs + 255) / 256), n), 256, 0, s>>>(T, slots, A,
                                                                                   partial);
  return cudaGetLastError() == cudaSuccess ? LH_OK : LH_ECUDA;
}

}  // namespace lh

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

}  // namespace lh

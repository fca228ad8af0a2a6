/*
 * Oracle (test infrastructure only): the order >=2 contraction of axial-basis
 * sources with band-folded kernels, in float64 C.
 *
 * Restates _apply_multi_spectral (_shower_basis.py:894-1050) without its
 * tolerance screen (the route passes none), with the Wigner small-d
 * recurrence _wigner_into and its start values (_directional_numba.py:37-87,
 * 389-397) and the real harmonics _harmonics_into (:90-128). Loops run in the
 * reference's order (receiver, point, degree, band, frequency). The NumPy
 * restatement in oracle/ge2.py checks this file; only tests/,
 * __graft_entry__.smoke() and bench.py's CPU baseline load it.
 */
#include <complex.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define G2_PI 3.14159265358979323846

static double parity(int n) { return (n % 2 == 0) ? 1.0 : -1.0; }

static double ipow_real(double x, int n) {
  double r = 1.0;
  for (int k = 0; k < n; ++k) r *= x;
  return r;
}

/* d^j_(mu nu) at j = max(|mu|, |nu|) */
static double start_value(int j, int mu, int nu, double half_cos, double half_sin,
                          const double* start_norm, int jmax) {
  double sign = 1.0;
  if (abs(nu) == j && abs(mu) != j) {
    int t = mu;
    mu = nu;
    nu = t;
    sign *= parity(mu - nu);
  }
  if (mu == -j) {
    mu = j;
    nu = -nu;
    sign *= parity(j + nu);
  }
  return sign * start_norm[j * (2 * jmax + 1) + nu + jmax] * ipow_real(half_cos, j + nu) *
         ipow_real(-half_sin, j - nu);
}

/* out[l][nu + max_out][mu] = d^l_(mu nu), mu in 0..max_in */
static void wigner(int degree, int max_out, int max_in, double cosine, const double* start_norm,
                   int jmax, double* out) {
  const int width = 2 * max_out + 1;
  memset(out, 0, sizeof(double) * (degree + 1) * width * (max_in + 1));
  double half_cos = sqrt((1.0 + cosine) / 2.0), half_sin = sqrt((1.0 - cosine) / 2.0);
  for (int nu = -max_out; nu <= max_out; ++nu)
    for (int mu = 0; mu <= max_in; ++mu) {
      int start = abs(nu) > mu ? abs(nu) : mu;
      if (start > degree) continue;
      double previous = 0.0;
      double current = start_value(start, mu, nu, half_cos, half_sin, start_norm, jmax);
      out[(start * width + nu + max_out) * (max_in + 1) + mu] = current;
      for (int ell = start; ell < degree; ++ell) {
        double value;
        if (ell == 0) {
          value = cosine * current;
        } else {
          double lower = (double)(ell * ell - mu * mu) * (double)(ell * ell - nu * nu);
          lower = lower > 0.0 ? sqrt(lower) : 0.0;
          double upper = sqrt((double)((ell + 1) * (ell + 1) - mu * mu) *
                              (double)((ell + 1) * (ell + 1) - nu * nu));
          value = (((2 * ell + 1) * (ell * (ell + 1) * cosine - mu * nu) * current -
                    (ell + 1) * lower * previous) /
                   (ell * upper));
        }
        previous = current;
        current = value;
        out[((ell + 1) * width + nu + max_out) * (max_in + 1) + mu] = current;
      }
    }
}

static void harmonics(double x, double y, double z, int degree, double* out) {
  double radius = sqrt(x * x + y * y + z * z);
  double mu = z / radius;
  double transverse = sqrt(x * x + y * y);
  double sine = transverse / radius;
  double cp = transverse == 0.0 ? 1.0 : x / transverse;
  double sp = transverse == 0.0 ? 0.0 : y / transverse;
  double cm = 1.0, sm = 0.0;
  double diagonal = 1.0 / sqrt(4 * G2_PI);
  double v0 = 0.0, v1 = 0.0;
  for (int m = 0; m <= degree; ++m) {
    if (m) {
      diagonal *= sqrt((2.0 * m + 1) / (2.0 * m)) * sine;
      double ncm = cm * cp - sm * sp;
      sm = sm * cp + cm * sp;
      cm = ncm;
    }
    v0 = diagonal;
    for (int ell = m; ell <= degree; ++ell) {
      double value;
      if (ell == m) {
        value = v0;
      } else if (ell == m + 1) {
        value = sqrt(2 * m + 3) * mu * v0;
        v1 = value;
      } else {
        double aa = sqrt((4.0 * ell * ell - 1) / (double)(ell * ell - m * m));
        double bb = sqrt(((2.0 * ell + 1) * ((double)(ell - 1) * (ell - 1) - m * m)) /
                         ((2.0 * ell - 3) * (double)(ell * ell - m * m)));
        value = aa * mu * v1 - bb * v0;
        v0 = v1;
        v1 = value;
      }
      int centre = ell * ell + ell;
      if (m == 0) {
        out[centre] = value;
      } else {
        out[centre - m] = sqrt(2) * value * sm;
        out[centre + m] = sqrt(2) * value * cm;
      }
    }
  }
}

/* channels: complex128 [nlam][n_points][nch][nfreq]; coefficients: complex128
 * [nlam][n_int][degree+1][npair][4][nfreq]; out_scale [nlam][nrec]. Points,
 * receivers and looks are in the source frame. result: complex128 [nrec][nfreq]. */
int o2c_apply(int64_t n_points, const double* points, int64_t nrec, const double* receivers,
              const double* looks, int nlam, int nch, const double _Complex* channels,
              const double* out_scale, const int64_t* starts, int degree, int max_m, int max_out,
              const double* alpha, int npair, const int64_t* pair_lambda, const int64_t* pair_mu,
              int n_log_r, const double* log_r, const double _Complex* coefficients,
              const double* absorption, const double* velocity, int nfreq, const double* omega,
              int flight, double radial_low, double radial_high, double _Complex* result) {
  const int width = 2 * max_out + 1;
  const int jmax = max_m > max_out ? max_m : max_out;
  const double root2 = sqrt(2.0);
  double* start_norm = (double*)calloc((size_t)(jmax + 1) * (2 * jmax + 1), sizeof(double));
  double* wig = (double*)malloc(sizeof(double) * (degree + 1) * width * (max_m + 1));
  double* detector = (double*)malloc(sizeof(double) * (max_out + 1) * (max_out + 1));
  double* erow = (double*)malloc(sizeof(double) * width * (2 * max_m + 1));
  double _Complex* rotated = (double _Complex*)malloc(sizeof(double _Complex) * nlam * width * nfreq);
  double _Complex* channel_sum = (double _Complex*)malloc(sizeof(double _Complex) * width * nfreq);
  double _Complex* scale_phase = (double _Complex*)malloc(sizeof(double _Complex) * nlam * nfreq);
  double _Complex* response = (double _Complex*)malloc(sizeof(double _Complex) * nlam * nfreq);
  double* cosines = (double*)malloc(sizeof(double) * (max_m + 1));
  double* sines = (double*)malloc(sizeof(double) * (max_m + 1));
  if (!start_norm || !wig || !detector || !erow || !rotated || !channel_sum || !scale_phase ||
      !response || !cosines || !sines)
    return -1;
  for (int j = 0; j <= jmax; ++j)
    for (int nu = -j; nu <= j; ++nu)
      start_norm[j * (2 * jmax + 1) + nu + jmax] =
          exp(0.5 * (lgamma(2 * j + 1) - lgamma(j + nu + 1) - lgamma(j - nu + 1)));
  const int64_t per_int = (int64_t)(degree + 1) * npair * 4 * nfreq;
  const int64_t per_lam = (int64_t)(n_log_r - 1) * per_int;
  memset(result, 0, sizeof(double _Complex) * nrec * nfreq);
  for (int64_t index = 0; index < nrec; ++index) {
    for (int64_t cell = 0; cell < n_points; ++cell) {
      double dx = receivers[3 * index] - points[3 * cell];
      double dy = receivers[3 * index + 1] - points[3 * cell + 1];
      double dz = receivers[3 * index + 2] - points[3 * cell + 2];
      double radius = sqrt(dx * dx + dy * dy + dz * dz);
      if (radius < radial_low || radius > radial_high) continue;
      double cosine = dz / radius;
      if (cosine > 1.0) cosine = 1.0;
      else if (cosine < -1.0) cosine = -1.0;
      double phi = atan2(dy, dx);
      double transverse = sqrt(dx * dx + dy * dy);
      double sine = transverse / radius;
      double cp = transverse == 0.0 ? 1.0 : dx / transverse;
      double sp = transverse == 0.0 ? 0.0 : dy / transverse;
      for (int n = 0; n <= max_m; ++n) {
        cosines[n] = cos(n * phi);
        sines[n] = sin(n * phi);
      }
      double lx = looks[3 * index], ly = looks[3 * index + 1], lz = looks[3 * index + 2];
      double a1 = cosine * cp * lx + cosine * sp * ly - sine * lz;
      double a2 = -sp * lx + cp * ly;
      double a3 = sine * cp * lx + sine * sp * ly + cosine * lz;
      harmonics(a1, a2, a3, max_out, detector);
      wigner(degree, max_out, max_m, cosine, start_norm, jmax, wig);
      double logr = log(radius);
      int j = 0; /* searchsorted(log_r, logr, side='right') - 1 */
      {
        int lo = 0, hi = n_log_r;
        while (lo < hi) {
          int mid = (lo + hi) / 2;
          if (log_r[mid] <= logr) lo = mid + 1; else hi = mid;
        }
        j = lo - 1;
      }
      if (j < 0) j = 0;
      if (j > n_log_r - 2) j = n_log_r - 2;
      double t = logr - log_r[j];
      for (int lam = 0; lam < nlam; ++lam) {
        double scale = (out_scale[lam * nrec + index] * exp(-absorption[lam] * radius) /
                        (4 * G2_PI * radius * radius));
        for (int w = 0; w < nfreq; ++w) {
          response[lam * nfreq + w] = 0.0;
          if (flight) {
            double angle = omega[w] * radius / velocity[lam];
            scale_phase[lam * nfreq + w] = scale * (cos(angle) + I * sin(angle));
          } else {
            scale_phase[lam * nfreq + w] = scale;
          }
        }
      }
      for (int ell = 0; ell <= degree; ++ell) {
#define WG(l, a, m) wig[((l) * width + (a)) * (max_m + 1) + (m)]
#define ER(a, b) erow[(a) * (2 * max_m + 1) + (b)]
        memset(erow, 0, sizeof(double) * width * (2 * max_m + 1));
        ER(max_out, max_m) = WG(ell, max_out, 0);
        int top_n = ell < max_m ? ell : max_m;
        int top_p = ell < max_out ? ell : max_out;
        for (int n = 1; n <= top_n; ++n) {
          double base = root2 * parity(n) * WG(ell, max_out, n);
          ER(max_out, max_m + n) = base * cosines[n];
          ER(max_out, max_m - n) = base * sines[n];
        }
        for (int p = 1; p <= top_p; ++p) {
          ER(max_out + p, max_m) = (root2 * parity(p) * WG(ell, max_out + p, 0));
          for (int n = 1; n <= top_n; ++n) {
            double cross = parity(p) * WG(ell, max_out + p, n);
            double straight = WG(ell, max_out - p, n);
            double cc = parity(n) * (cross + straight);
            double ss = parity(n) * (cross - straight);
            ER(max_out + p, max_m + n) = cc * cosines[n];
            ER(max_out + p, max_m - n) = cc * sines[n];
            ER(max_out - p, max_m + n) = -ss * sines[n];
            ER(max_out - p, max_m - n) = ss * cosines[n];
          }
        }
        int keep = top_n;
        int centre = (int)starts[ell] + keep;
        memset(rotated, 0, sizeof(double _Complex) * nlam * width * nfreq);
        for (int a = max_out - top_p; a <= max_out + top_p; ++a)
          for (int b = max_m - keep; b <= max_m + keep; ++b) {
            double factor = ER(a, b);
            if (factor == 0.0) continue;
            int column = centre + (b - max_m);
            for (int lam = 0; lam < nlam; ++lam) {
              const double _Complex* ch =
                  channels + (((int64_t)lam * n_points + cell) * nch + column) * nfreq;
              double _Complex* rot = rotated + ((int64_t)lam * width + a) * nfreq;
              for (int w = 0; w < nfreq; ++w) rot[w] += factor * ch[w];
            }
          }
        for (int lam = 0; lam < nlam; ++lam) {
          memset(channel_sum, 0, sizeof(double _Complex) * width * nfreq);
          for (int p = 0; p < npair; ++p) {
            int lam_d = (int)pair_lambda[p], mu_pair = (int)pair_mu[p];
            if (mu_pair > top_p) continue;
            int dc = lam_d * lam_d + lam_d;
            double positive = alpha[lam_d] * detector[dc + mu_pair];
            double negative = mu_pair ? alpha[lam_d] * detector[dc - mu_pair] : 0.0;
            if (positive == 0.0 && negative == 0.0) continue;
            const double _Complex* cf =
                coefficients + lam * per_lam + (int64_t)j * per_int + ((int64_t)ell * npair + p) * 4 * nfreq;
            for (int w = 0; w < nfreq; ++w) {
              double _Complex radial =
                  ((cf[w] * t + cf[nfreq + w]) * t + cf[2 * nfreq + w]) * t + cf[3 * nfreq + w];
              if (negative != 0.0) channel_sum[(max_out - mu_pair) * nfreq + w] += negative * radial;
              if (positive != 0.0) channel_sum[(max_out + mu_pair) * nfreq + w] += positive * radial;
            }
          }
          for (int a = max_out - top_p; a <= max_out + top_p; ++a)
            for (int w = 0; w < nfreq; ++w) {
              double _Complex value = rotated[((int64_t)lam * width + a) * nfreq + w];
              if (value == 0.0) continue;
              response[lam * nfreq + w] += value * channel_sum[a * nfreq + w];
            }
        }
#undef WG
#undef ER
      }
      for (int lam = 0; lam < nlam; ++lam)
        for (int w = 0; w < nfreq; ++w)
          result[index * nfreq + w] += response[lam * nfreq + w] * scale_phase[lam * nfreq + w];
    }
  }
  free(start_norm); free(wig); free(detector); free(erow); free(rotated);
  free(channel_sum); free(scale_phase); free(response); free(cosines); free(sines);
  return 0;
}

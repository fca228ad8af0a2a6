// Rotation helpers shared by the order >=2 kernels: Wigner small-d start
// values and real orthonormal spherical harmonics (reference
// _directional_numba.py:37-128).
#pragma once

#include "lh_common.cuh"

namespace lh {

LH_DEVICE double par(int n) { return (n & 1) ? -1.0 : 1.0; }

// d^j_(mu nu) at j = max(|mu|, |nu|)  (_directional_numba.py:37-48)
LH_DEVICE double wigner_start(int j, int mu, int nu, double hc, double hs, const double* norm,
                              int jmax) {
  double sign = 1.0;
  if (abs(nu) == j && abs(mu) != j) {
    int t = mu; mu = nu; nu = t;
    sign *= par(mu - nu);
  }
  if (mu == -j) {
    mu = j;
    nu = -nu;
    sign *= par(j + nu);
  }
  double v = sign * norm[j * (2 * jmax + 1) + nu + jmax];
  for (int k = 0; k < j + nu; ++k) v *= hc;
  for (int k = 0; k < j - nu; ++k) v *= -hs;
  return v;
}

// Real orthonormal harmonics up to degree A of (x, y, z), flat l*l+l+m (:90-128)
LH_DEVICE void real_harmonics(double x, double y, double z, int A, double* out) {
  const double radius = sqrt(x * x + y * y + z * z);
  const double mu = z / radius;
  const double tr = sqrt(x * x + y * y);
  const double sine = tr / radius;
  const double cp = tr == 0.0 ? 1.0 : x / tr;
  const double sp = tr == 0.0 ? 0.0 : y / tr;
  double cm = 1.0, sm = 0.0, diag = 1.0 / sqrt(4 * kPi), v0 = 0.0, v1 = 0.0;
  for (int m = 0; m <= A; ++m) {
    if (m) {
      diag *= sqrt((2.0 * m + 1) / (2.0 * m)) * sine;
      const double c2 = cm * cp - sm * sp, s2 = sm * cp + cm * sp;
      cm = c2;
      sm = s2;
    }
    v0 = diag;
    for (int l = m; l <= A; ++l) {
      double value;
      if (l == m) value = v0;
      else if (l == m + 1) {
        value = sqrt(2.0 * m + 3) * mu * v0;
        v1 = value;
      } else {
        const double aa = sqrt((4.0 * l * l - 1) / (double)(l * l - m * m));
        const double bb = sqrt(((2.0 * l + 1) * ((l - 1) * (l - 1) - m * m)) /
                               ((2.0 * l - 3) * (double)(l * l - m * m)));
        value = aa * mu * v1 - bb * v0;
        v0 = v1;
        v1 = value;
      }
      const int c = l * l + l;
      if (m == 0) out[c] = value;
      else {
        out[c - m] = sqrt(2.0) * value * sm;
        out[c + m] = sqrt(2.0) * value * cm;
      }
    }
  }
}

}  // namespace lh

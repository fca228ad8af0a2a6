// Host-side preparation of a shower's source frame (no device code).
//
// AxisFrame.of (axial_source.py:88-118) takes the element midpoints' weighted
// centre and covariance; the route must reproduce them bit for bit (one
// rounding apart can move a node across a slice edge or a slice across the
// stencil threshold). NumPy evaluates the reference's expressions as
// elementwise products rounded to float64 and sums along the element axis in
// element order; these loops do the same in one pass over the elements
// instead of a dozen temporary arrays. The library is built with
// -ffp-contract=off, so no product is fused into a sum.
#include <cstdint>

#include "../../include/lighthit_b200.h"

extern "C" int lh_axis_frame_sums(int64_t n, const double* start, const double* direction,
                                  const double* length, const double* share, double* centre,
                                  double* covariance) {
  if (n < 1 || !start || !direction || !length || !share || !centre || !covariance)
    return LH_EINVAL;
  double c[3] = {0.0, 0.0, 0.0};
  for (int64_t i = 0; i < n; ++i) {
    const double half = 0.5 * length[i];
    for (int j = 0; j < 3; ++j) {
      const double point = start[3 * i + j] + half * direction[3 * i + j];
      const double weighted = share[i] * point;
      c[j] = c[j] + weighted;
    }
  }
  double cov[3][3] = {{0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}};
  for (int64_t i = 0; i < n; ++i) {
    const double half = 0.5 * length[i];
    double offset[3], lead[3];
    for (int j = 0; j < 3; ++j) {
      offset[j] = (start[3 * i + j] + half * direction[3 * i + j]) - c[j];
      lead[j] = share[i] * offset[j];
    }
    for (int j = 0; j < 3; ++j)
      for (int k = 0; k <= j; ++k) {
        const double term = lead[j] * offset[k];
        cov[j][k] = cov[j][k] + term;
      }
  }
  for (int j = 0; j < 3; ++j) {
    centre[j] = c[j];
    for (int k = 0; k < 3; ++k) covariance[3 * j + k] = k <= j ? cov[j][k] : 0.0;
  }
  return LH_OK;
}

// Per-coordinate minima and maxima over the element starts and ends
// start + length * direction (the cell grid of compress, prompt.py:1317-1402,
// and the route's radial and clock decisions). A NaN coordinate makes that
// coordinate's bounds NaN, as NumPy's min and max do.
extern "C" int lh_element_box(int64_t n, const double* start, const double* direction,
                              const double* length, double* low, double* high) {
  if (n < 1 || !start || !direction || !length || !low || !high) return LH_EINVAL;
  for (int j = 0; j < 3; ++j) {
    double lo = start[j], hi = start[j];
    bool nan = false;
    for (int64_t i = 0; i < n; ++i) {
      const double a = start[3 * i + j];
      const double product = length[i] * direction[3 * i + j];
      const double b = a + product;
      nan = nan || a != a || b != b;
      lo = a < lo ? a : lo;
      hi = a > hi ? a : hi;
      lo = b < lo ? b : lo;
      hi = b > hi ? b : hi;
    }
    low[j] = nan ? __builtin_nan("") : lo;
    high[j] = nan ? __builtin_nan("") : hi;
  }
  return LH_OK;
}

// delay_groups (shower/ge2.py:122-147): each step's delay behind the light
// front of step `first`, (t_i - t_first) - |x_i - x_first| / c, with the
// distance summed x, y, z in that order and every operation rounded to
// float64 as NumPy evaluates the expression; `distance` (optional) receives
// |x_i - x_first|.
extern "C" int lh_element_delays(int64_t n, const double* start, const double* start_ns,
                                 int64_t first, double c_m_per_ns, double* delay,
                                 double* distance) {
  if (n < 1 || first < 0 || first >= n || !start || !start_ns || !delay || !(c_m_per_ns > 0.0))
    return LH_EINVAL;
  const double x0 = start[3 * first], y0 = start[3 * first + 1], z0 = start[3 * first + 2];
  const double t0 = start_ns[first];
  for (int64_t i = 0; i < n; ++i) {
    const double dx = start[3 * i] - x0, dy = start[3 * i + 1] - y0, dz = start[3 * i + 2] - z0;
    const double xx = dx * dx, yy = dy * dy, zz = dz * dz;
    const double d = __builtin_sqrt((xx + yy) + zz);
    delay[i] = (start_ns[i] - t0) - d / c_m_per_ns;
    if (distance) distance[i] = d;
  }
  return LH_OK;
}

// compress's sub-segment layout (prompt.py:1317-1402): element i is cut into
// n_a = max(1, ceil(length_i / a_step)) sub-segments; offsets[i] is the first
// sub-segment of element i (offsets[n] = *n_sub). Lengths must be finite and
// non-negative.
extern "C" int lh_subsegment_offsets(int64_t n, const double* length, double a_step,
                                     int64_t* offsets, int64_t* n_sub) {
  if (n < 0 || (n && !length) || !offsets || !n_sub || !(a_step > 0.0)) return LH_EINVAL;
  int64_t total = 0;
  offsets[0] = 0;
  for (int64_t i = 0; i < n; ++i) {
    const double x = length[i];
    if (!(x >= 0.0) || x > 1e300) return LH_EINVAL;
    const double pieces = __builtin_ceil(x / a_step);
    total += pieces < 1.0 ? 1 : (int64_t)pieces;
    offsets[i + 1] = total;
  }
  *n_sub = total;
  return LH_OK;
}

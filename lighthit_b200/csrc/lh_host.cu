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

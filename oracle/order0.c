/*
 * Oracle (test infrastructure only): order-0 direct light to the first glass
 * entry of each OM sphere, in float64 C.
 *
 * Restates, loop for loop, the reference's
 *   interval_candidates         _ballistic_interval_numba.py:449-519
 *     _cone_can_reach_sphere    _ballistic_interval_numba.py:226-251
 *     _support                  _ballistic_interval_numba.py:151-185
 *   _surface_ballistic_rays.evaluate   _surface_ballistic_rays.py:36-156
 *     _quadratic_cuts           _surface_ballistic_rays.py:14-30
 *     _entry                    _surface_ballistic_rays.py:33-35
 *     _acceptance               _ballistic_interval_numba.py:21-37
 *     _insert_cuts/_sort_small  _ballistic_interval_numba.py:50-58, 294-306
 * Built by oracle/build.py with gcc; only tests/, __graft_entry__.smoke() and
 * bench.py's CPU baseline load it.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define O0_C 0.299792458
#define O0_PI 3.14159265358979323846

enum { O0_OK = 0, O0_ON_TRACK = -1, O0_INSIDE_GLASS = -2, O0_NEGATIVE = -3, O0_CAPACITY = -4 };

static double acceptance(const double* alpha, int n_alpha, double x, int* err) {
  double result = alpha[0] / (4 * O0_PI);
  double previous = 1.0, current = x;
  if (n_alpha > 1) result += 3 * alpha[1] * current / (4 * O0_PI);
  for (int ell = 2; ell < n_alpha; ++ell) {
    double value = ((2 * ell - 1) * x * current - (ell - 1) * previous) / ell;
    result += (2 * ell + 1) * alpha[ell] * value / (4 * O0_PI);
    previous = current;
    current = value;
  }
  if (result < 0.) {
    double s = 0.;
    for (int k = 0; k < n_alpha; ++k) s += fabs(alpha[k]);
    if (result < -1e-12 * (s > 1. ? s : 1.)) *err = O0_NEGATIVE;
  }
  return result > 0. ? result : 0.;
}

static int support(double z, double rho, double length, double beta, double radius, double* nmin,
                   double* nmax, double* cut0, double* cut1) {
  if (radius == 0.) {
    if (z <= 0.) return 0;
    *nmin = hypot(z, rho) / (beta * z);
    *nmax = INFINITY;
    if (z > length) {
      double rz = z - length;
      *nmax = hypot(rz, rho) / (beta * rz);
    }
    *cut0 = *cut1 = INFINITY;
    return 1;
  }
  const double quarter = .5 * O0_PI;
  double psi0 = atan2(rho, z), psi1 = atan2(rho, z - length);
  double r0 = radius / hypot(z, rho), r1 = radius / hypot(z - length, rho);
  double a0 = asin(r0 < 1. ? r0 : 1.), a1 = asin(r1 < 1. ? r1 : 1.);
  double low = psi0 - a0, high = psi1 + a1;
  if (low >= quarter) return 0;
  double floor_n = (1. + 1e-9) / beta;
  if (low <= 0.) *nmin = floor_n;
  else {
    double v = 1. / (beta * cos(low));
    *nmin = floor_n > v ? floor_n : v;
  }
  *nmax = high >= quarter ? INFINITY : 1. / (beta * cos(high));
  double inner0 = psi0 + a0, inner1 = psi1 - a1;
  *cut0 = inner0 >= quarter ? INFINITY : 1. / (beta * cos(inner0));
  *cut1 = (inner1 <= 0. || inner1 >= quarter) ? INFINITY : 1. / (beta * cos(inner1));
  return 1;
}

static int cone_can_reach_sphere(double z, double rho, double length, double beta, double radius,
                                 double phase_min, double phase_max) {
  if (z <= -radius || beta * phase_max <= 1.) return 0;
  double c_hi = 1. / (beta * phase_max);
  double t = (1. - c_hi) * (1. + c_hi);
  double s_hi = sqrt(t > 0. ? t : 0.);
  double c_lo = 1. / (beta * phase_min);
  if (c_lo > 1.) c_lo = 1.;
  t = (1. - c_lo) * (1. + c_lo);
  double s_lo = sqrt(t > 0. ? t : 0.);
  double q_hi = rho * c_hi - z * s_hi;
  double other = rho * c_lo - z * s_lo;
  double minimum = z >= 0. ? q_hi : (q_hi < other ? q_hi : other);
  double rounding = 16 * 2.220446049250313e-16 * (fabs(z) + rho + length + radius);
  if (minimum > radius + rounding) return 0;
  double end_z = z - length;
  if (end_z >= 0. && rho * c_lo - end_z * s_lo < -radius - rounding) return 0;
  return 1;
}

/* Pairs passing the geometry precheck, receiver-major in element order.
 * Returns the count, or O0_ON_TRACK / O0_CAPACITY. */
int64_t o0_candidates(int32_t n_om, const double* pos, const double* radii, double reach,
                      int32_t n_el, const double* start, const double* dir, const double* len,
                      const double* c0, const double* beta, int32_t n_phase, const double* phase,
                      int32_t include_axis, int64_t* out_om, int64_t* out_el, int64_t capacity) {
  double gmin = phase[0], gmax = phase[0];
  for (int k = 1; k < n_phase; ++k) {
    if (phase[k] < gmin) gmin = phase[k];
    if (phase[k] > gmax) gmax = phase[k];
  }
  int64_t count = 0;
  for (int om = 0; om < n_om; ++om) {
    const int sphere = radii[om] > 0.;
    for (int i = 0; i < n_el; ++i) {
      if (c0[i] == 0. || beta[i] * gmax <= 1.) continue;
      double dx = pos[3 * om] - start[3 * i], dy = pos[3 * om + 1] - start[3 * i + 1];
      double dz = pos[3 * om + 2] - start[3 * i + 2];
      double ux = dir[3 * i], uy = dir[3 * i + 1], uz = dir[3 * i + 2];
      double z = dx * ux + dy * uy + dz * uz;
      if (z <= 0. && (!sphere || z <= -reach || z <= -radii[om])) continue;
      double cx = dy * uz - dz * uy, cy = dz * ux - dx * uz, cz = dx * uy - dy * ux;
      double rho = sqrt(cx * cx + cy * cy + cz * cz);
      double radius = 0.;
      if (sphere && rho < reach) {
        double along = z < 0. ? z : (z > len[i] ? z - len[i] : 0.);
        if (along * along + rho * rho < reach * reach) radius = radii[om];
      }
      if (z <= 0. && radius == 0.) continue;
      double nmin, nmax, cut0, cut1;
      int ok;
      if (rho == 0.) {
        if (radius == 0. || !include_axis) {
          if (0. < z && z < len[i]) return O0_ON_TRACK;
          continue;
        }
        if (count >= capacity) return O0_CAPACITY;
        out_om[count] = om;
        out_el[count] = i;
        ++count;
        continue;
      }
      if (radius == 0.) {
        nmin = hypot(z, rho) / (beta[i] * z);
        nmax = INFINITY;
        if (z > len[i]) {
          double rz = z - len[i];
          nmax = hypot(rz, rho) / (beta[i] * rz);
        }
        ok = 1;
      } else {
        if (!cone_can_reach_sphere(z, rho, len[i], beta[i], radius, gmin, gmax)) continue;
        ok = support(z, rho, len[i], beta[i], radius, &nmin, &nmax, &cut0, &cut1);
      }
      if (!ok || nmin > gmax || nmax <= gmin) continue;
      if (count >= capacity) return O0_CAPACITY;
      out_om[count] = om;
      out_el[count] = i;
      ++count;
    }
  }
  return count;
}

static void sort_small(double* v, int count) {
  for (int k = 1; k < count; ++k) {
    double value = v[k];
    int m = k - 1;
    while (m >= 0 && v[m] > value) {
      v[m + 1] = v[m];
      --m;
    }
    v[m + 1] = value;
  }
}

static int quadratic_cuts(double* cuts, int count, double a, double b, double c, double low,
                          double high) {
  if (a == 0.) {
    if (b != 0.) {
      double root = -c / b;
      if (low < root && root < high) cuts[count++] = root;
    }
    return count;
  }
  double disc = b * b - 4 * a * c;
  if (disc < 0.) return count;
  double q = -.5 * (b + copysign(sqrt(disc), b));
  if (q == 0.) {
    double root = -b / (2 * a);
    if (low < root && root < high) cuts[count++] = root;
  } else {
    double r1 = q / a, r2 = c / q;
    if (low < r1 && r1 < high) cuts[count++] = r1;
    if (low < r2 && r2 < high) cuts[count++] = r2;
  }
  return count;
}

static double entry(double B, double dot) {
  double t = dot * dot - B;
  return B / (dot + sqrt(t > 0. ? t : 0.));
}

/* searchsorted(edges, x, side) over n ascending values */
static int search_right(const double* e, int n, double x) {
  int lo = 0, hi = n;
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if (e[mid] > x) hi = mid; else lo = mid + 1;
  }
  return lo;
}
static int search_left(const double* e, int n, double x) {
  int lo = 0, hi = n;
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if (e[mid] >= x) hi = mid; else lo = mid + 1;
  }
  return lo;
}

/* _surface_ballistic_rays.evaluate: charge[om] and bins[om][slot] accumulate
 * (caller zeroes them). Returns O0_OK or an error code. */
int o0_rays(int64_t n_pairs, const int64_t* po, const int64_t* pe, const double* pos,
            const double* looks, const double* areas, const double* radii, const double* starts,
            const double* axes, const double* lengths, const double* c0, const double* c2,
            const double* beta, const double* t0, const double* t1, int32_t n_panel_edges,
            const double* panels, const double* phases, const double* groups,
            const double* extinction, const double* efficiency, int32_t eff_cols,
            int32_t n_alpha, const double* alpha, int32_t order, const double* gx,
            const double* gw, const double* origins, int32_t n_edges, const double* edges,
            double* charge, double* bins) {
  const int nb = n_edges - 1;
  double* phicuts = (double*)malloc(sizeof(double) * (n_edges + 2));
  double* scuts = (double*)malloc(sizeof(double) * (6 * n_edges + 2));
  double pmin = phases[0], pmax = phases[0];
  for (int k = 1; k < n_panel_edges; ++k) {
    if (phases[k] < pmin) pmin = phases[k];
    if (phases[k] > pmax) pmax = phases[k];
  }
  int err = O0_OK;
  for (int64_t pair = 0; pair < n_pairs && err == O0_OK; ++pair) {
    const int64_t om = po[pair], i = pe[pair];
    const double radius = radii[om];
    double w[3], u[3];
    for (int k = 0; k < 3; ++k) {
      w[k] = pos[3 * om + k] - starts[3 * i + k];
      u[k] = axes[3 * i + k];
    }
    double z = w[0] * u[0] + w[1] * u[1] + w[2] * u[2];
    double tr[3] = {w[0] - z * u[0], w[1] - z * u[1], w[2] - z * u[2]};
    double rho = sqrt(tr[0] * tr[0] + tr[1] * tr[1] + tr[2] * tr[2]);
    double nmin, nmax, cut0, cut1;
    const double L = lengths[i];
    if (!support(z, rho, L, beta[i], radius, &nmin, &nmax, &cut0, &cut1) || nmin > pmax ||
        nmax <= pmin)
      continue;
    double along_min = z < 0. ? z : (z > L ? z - L : 0.);
    if (rho * rho + along_min * along_min <= radius * radius) { err = O0_INSIDE_GLASS; break; }
    double e1[3], e2[3];
    if (rho > 0.) {
      for (int k = 0; k < 3; ++k) e1[k] = tr[k] / rho;
    } else {
      double aux[3] = {0., 0., 0.};
      if (fabs(u[0]) < .9) aux[0] = 1.; else aux[1] = 1.;
      e1[0] = u[1] * aux[2] - u[2] * aux[1];
      e1[1] = u[2] * aux[0] - u[0] * aux[2];
      e1[2] = u[0] * aux[1] - u[1] * aux[0];
      double nn = sqrt(e1[0] * e1[0] + e1[1] * e1[1] + e1[2] * e1[2]);
      for (int k = 0; k < 3; ++k) e1[k] /= nn;
    }
    e2[0] = u[1] * e1[2] - u[2] * e1[1];
    e2[1] = u[2] * e1[0] - u[0] * e1[2];
    e2[2] = u[0] * e1[1] - u[1] * e1[0];
    const double* lk = looks + 3 * om;
    double axial = u[0] * lk[0] + u[1] * lk[1] + u[2] * lk[2];
    double across = e1[0] * lk[0] + e1[1] * lk[1] + e1[2] * lk[2];
    double side = e2[0] * lk[0] + e2[1] * lk[1] + e2[2] * lk[2];
    double tau = (t1[i] - t0[i]) / L;
    for (int panel = 0; panel < n_panel_edges - 1 && err == O0_OK; ++panel) {
      double left = panels[panel], width = panels[panel + 1] - left;
      double n0 = phases[panel], dn = phases[panel + 1] - n0;
      double a = left, b = left + width;
      if (dn == 0.) {
        if (n0 < nmin || n0 >= nmax) continue;
      } else {
        double x0 = (nmin - n0) / dn, x1 = (nmax - n0) / dn;
        double lo = x0 < x1 ? x0 : x1, hi = x0 < x1 ? x1 : x0;
        a = left + width * (lo > 0. ? lo : 0.);
        b = left + width * (hi < 1. ? hi : 1.);
      }
      if (a >= b) continue;
      double cuts[7];
      cuts[0] = a;
      cuts[1] = b;
      int count = 2;
      if (dn != 0.) {
        double lo = cuts[0], hi = cuts[count - 1];
        double vals[2] = {cut0, cut1};
        for (int v = 0; v < 2; ++v) {
          if (isfinite(vals[v])) {
            double lam = left + width * (vals[v] - n0) / dn;
            if (lo < lam && lam < hi) cuts[count++] = lam;
          }
        }
        sort_small(cuts, count);
      }
      for (int piece = 0; piece < count - 1; ++piece) {
        double low = cuts[piece], high = cuts[piece + 1];
        for (int ilam = 0; ilam < order; ++ilam) {
          double lam = (low + high) / 2 + (high - low) / 2 * gx[ilam];
          double q = (lam - left) / width, n = n0 + dn * q, bn = beta[i] * n;
          if (bn <= 1.) continue;
          double cosine = 1 / bn, sine = sqrt(1 - cosine * cosine);
          double centre = z - rho * cosine / sine, spread = radius / sine;
          double slo = centre - spread > 0. ? centre - spread : 0.;
          double shi = centre + spread < L ? centre + spread : L;
          if (slo >= shi) continue;
          double absorption = extinction[panel] + q * (extinction[panel + 1] - extinction[panel]);
          double group = groups[panel] + q * (groups[panel + 1] - groups[panel]);
          double velocity = O0_C / group;
          const double* ef = efficiency + panel * eff_cols;
          double eta = ((ef[3] * q + ef[2]) * q + ef[1]) * q + ef[0];
          if (eff_cols > 4) eta *= exp(ef[4] + q * ef[5]);
          double spectral = (c0[i] + c2[i] / (n * n)) / L / (lam * lam) * eta;
          double scale = (high - low) / 2 * gw[ilam] * spectral * areas[om] / (O0_PI * radius * radius);
          scuts[0] = slo;
          scuts[1] = shi;
          int ns = 2;
          double d0 = (z - slo) * (z - slo), d1 = (z - shi) * (z - shi);
          double rmax = sqrt(rho * rho + (d0 > d1 ? d0 : d1));
          double rmin = sqrt(rho * rho + ((slo < z && z < shi) ? 0. : (d0 < d1 ? d0 : d1)));
          double e_lo = t0[i] + tau * slo, e_hi = t0[i] + tau * shi;
          double earliest = (e_lo < e_hi ? e_lo : e_hi) + (rmin - radius) / velocity - origins[om];
          double latest = (e_lo > e_hi ? e_lo : e_hi) + rmax / velocity - origins[om];
          int first_edge = search_right(edges, n_edges, earliest);
          int last_edge = search_left(edges, n_edges, latest);
          for (int edge = first_edge; edge < last_edge; ++edge) {
            double A = (origins[om] + edges[edge] - t0[i]) * velocity, B = tau * velocity;
            for (int sgn = -1; sgn <= 1; sgn += 2) {
              double D = cosine * z + sgn * sine * rho;
              ns = quadratic_cuts(scuts, ns, 1 + B * B - 2 * B * cosine,
                                  -2 * z - 2 * A * B + 2 * (A * cosine + B * D),
                                  z * z + rho * rho - radius * radius + A * A - 2 * A * D, slo, shi);
            }
            ns = quadratic_cuts(scuts, ns, B * B - 1., -2 * A * B + 2 * z,
                                A * A - z * z - rho * rho + radius * radius, slo, shi);
          }
          sort_small(scuts, ns);
          for (int sp = 0; sp < ns - 1; ++sp) {
            double sa = scuts[sp], sb = scuts[sp + 1];
            if (sa >= sb) continue;
            for (int j = 0; j < order; ++j) {
              double psi = O0_PI / 2 * gx[j];
              double s = (sa + sb) / 2 + (sb - sa) / 2 * sin(psi);
              double ds = (sb - sa) / 2 * cos(psi) * O0_PI / 2 * gw[j];
              double along = z - s, B = rho * rho + along * along - radius * radius;
              double half;
              if (rho > 0.) {
                double arg = (sqrt(B) - cosine * along) / (sine * rho);
                arg = arg < -1. ? -1. : (arg > 1. ? 1. : arg);
                half = acos(arg);
              } else {
                half = cosine * along >= sqrt(B) ? O0_PI : 0.;
              }
              if (half == 0.) continue;
              double emission = t0[i] + tau * s - origins[om];
              double tmin = emission + entry(B, cosine * along + sine * rho) / velocity;
              double tmax = emission + entry(B, cosine * along + sine * rho * cos(half)) / velocity;
              phicuts[0] = 0.;
              int nphi = 1;
              if (rho > 0.) {
                int first = search_right(edges, n_edges, tmin);
                int last = search_left(edges, n_edges, tmax);
                for (int edge = first; edge < last; ++edge) {
                  double distance = (edges[edge] - emission) * velocity;
                  double dot = (B + distance * distance) / (2 * distance);
                  double arg = (dot - cosine * along) / (sine * rho);
                  arg = arg < -1. ? -1. : (arg > 1. ? 1. : arg);
                  double phi = acos(arg);
                  double r = phi / half;
                  phicuts[nphi++] = asin(r < 1. ? r : 1.);
                }
              }
              phicuts[nphi++] = O0_PI / 2;
              for (int pp = 0; pp < nphi - 1; ++pp) {
                double pa = phicuts[pp], pb = phicuts[pp + 1];
                if (pa >= pb) continue;
                double integral = 0.;
                for (int jp = 0; jp < order; ++jp) {
                  double eta_phi = (pa + pb) / 2 + (pb - pa) / 2 * gx[jp];
                  double phi = half * sin(eta_phi);
                  double dphi = half * cos(eta_phi) * (pb - pa) / 2 * gw[jp];
                  double cp = cos(phi), ss = sin(phi);
                  double distance = entry(B, cosine * along + sine * rho * cp);
                  double accept =
                      acceptance(alpha, n_alpha, cosine * axial + sine * (cp * across + ss * side), &err) +
                      acceptance(alpha, n_alpha, cosine * axial + sine * (cp * across - ss * side), &err);
                  integral += dphi * accept * exp(-absorption * distance) / (2 * O0_PI);
                }
                double value = scale * ds * integral;
                charge[om] += value;
                double phi_mid = half * sin((pa + pb) / 2);
                double arrival =
                    emission + entry(B, cosine * along + sine * rho * cos(phi_mid)) / velocity;
                int slot = search_right(edges, n_edges, arrival) - 1;
                if (slot >= 0 && slot < nb) bins[om * nb + slot] += value;
              }
            }
          }
        }
      }
    }
  }
  free(phicuts);
  free(scuts);
  return err;
}

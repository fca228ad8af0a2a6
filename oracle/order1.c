/*
 * Oracle (test infrastructure only): order 1 (single scattering) of spectral
 * elements as grouped pencils, in float64 C.
 *
 * Restates the reference's grouped prompt order 1:
 *   stage A  compress                    prompt.py:1317-1402
 *            subsegment_cells            _prompt_numba.py:1083-1105
 *            compress_subsegments        _prompt_numba.py:1108-1232
 *            _pixel, _cell_key           _prompt_numba.py:1014-1043, 1078-1083
 *            finish_pencils              _prompt_numba.py:2246-2354
 *            parent_keys, pack_pencils   _prompt_screen.py:44-85 (coarse screen)
 *   stage B  grouped_pencils_order1      _prompt_numba.py:1750-2064
 *            _screen_block               _prompt_screen.py:172-440 (coarse screen:
 *                                        receiver-local angular refinement and
 *                                        the two-node radial rule)
 *            _prepare_pencil_shape       _prompt_numba.py:1324-1348
 *            _pencil_shape_factor_from_ray  _prompt_numba.py:1368-1416
 *            pencil_radial_rule, inverse_radius_rule  _prompt_screen.py:101-169
 *            gauss_inverse_mean_prepared _prompt_numba.py:115-129
 *            _fill_moments_averaged_pair _prompt_numba.py:1259-1276
 *            _batch_grid, _batch_sigma   _prompt_numba.py:255-296
 *            _cubic_moment_coefficients, _batch_add_moments  _prompt_numba.py:350-447
 *            _batch_deposit              _prompt_numba.py:450-551
 *            _deposit_panel, _find_bin, _quad_integral, _ifuncs  _prompt_numba.py:138-251
 *            _finalize                   _prompt_numba.py:609-632
 *            scalar_theta_index          _prompt_numba.py:1637-1641 (the reference's
 *                                        threshold tables reproduce this index)
 * Every loop runs in the reference's order (pencils in table order, groups in
 * key order, panels in node order), so each sum is formed as the reference
 * forms it. Built by oracle/build.py with gcc -ffp-contract=off; only tests/,
 * __graft_entry__.smoke() and bench.py's CPU baseline load it.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define O1_PI 3.14159265358979323846
#define O1_TWO_PI (2.0 * O1_PI)
#define O1_NM 23 /* moments of a stage-A bin */

static inline double dmin(double a, double b) { return a < b ? a : b; }
static inline double dmax(double a, double b) { return a > b ? a : b; }

/* ---------------------------------------------------------------- key -> row map */
typedef struct {
  int64_t* keys;  /* slot -> key (-1 free) */
  int64_t* rows;  /* slot -> row index */
  int64_t cap, used, width;
  double* values; /* used x width, insertion order */
  int64_t* row_keys;
  int64_t row_cap;
} o1_map;

static uint64_t o1_mix(uint64_t v) {
  v = (v ^ (v >> 30)) * 0xbf58476d1ce4e5b9ull;
  v = (v ^ (v >> 27)) * 0x94d049bb133111ebull;
  return v ^ (v >> 31);
}

static int map_init(o1_map* m, int64_t width, int64_t cap) {
  int64_t c = 1024;
  while (c < cap) c <<= 1;
  m->cap = c;
  m->used = 0;
  m->width = width;
  m->keys = (int64_t*)malloc(sizeof(int64_t) * c);
  m->rows = (int64_t*)malloc(sizeof(int64_t) * c);
  m->row_cap = c / 2;
  m->values = (double*)malloc(sizeof(double) * m->row_cap * width);
  m->row_keys = (int64_t*)malloc(sizeof(int64_t) * m->row_cap);
  if (!m->keys || !m->rows || !m->values || !m->row_keys) return -1;
  memset(m->keys, 0xff, sizeof(int64_t) * c);
  return 0;
}

static void map_free(o1_map* m) {
  free(m->keys);
  free(m->rows);
  free(m->values);
  free(m->row_keys);
  memset(m, 0, sizeof(*m));
}

static int map_grow(o1_map* m) {
  int64_t cap = m->cap * 2;
  int64_t* keys = (int64_t*)malloc(sizeof(int64_t) * cap);
  int64_t* rows = (int64_t*)malloc(sizeof(int64_t) * cap);
  double* values = (double*)realloc(m->values, sizeof(double) * (cap / 2) * m->width);
  int64_t* row_keys = (int64_t*)realloc(m->row_keys, sizeof(int64_t) * (cap / 2));
  if (!keys || !rows || !values || !row_keys) return -1;
  m->values = values;
  m->row_keys = row_keys;
  memset(keys, 0xff, sizeof(int64_t) * cap);
  for (int64_t r = 0; r < m->used; ++r) {
    uint64_t slot = o1_mix((uint64_t)m->row_keys[r]) & (uint64_t)(cap - 1);
    while (keys[slot] != -1) slot = (slot + 1) & (uint64_t)(cap - 1);
    keys[slot] = m->row_keys[r];
    rows[slot] = r;
  }
  free(m->keys);
  free(m->rows);
  m->keys = keys;
  m->rows = rows;
  m->cap = cap;
  m->row_cap = cap / 2;
  return 0;
}

/* The row of `key`, created (zeroed) when new. */
static double* map_row(o1_map* m, int64_t key) {
  if (2 * (m->used + 1) > m->cap && map_grow(m)) return NULL;
  uint64_t slot = o1_mix((uint64_t)key) & (uint64_t)(m->cap - 1);
  while (m->keys[slot] != -1 && m->keys[slot] != key) slot = (slot + 1) & (uint64_t)(m->cap - 1);
  if (m->keys[slot] == -1) {
    m->keys[slot] = key;
    m->rows[slot] = m->used;
    m->row_keys[m->used] = key;
    memset(m->values + m->used * m->width, 0, sizeof(double) * m->width);
    m->used++;
  }
  return m->values + m->rows[slot] * m->width;
}

static int cmp_i64(const void* a, const void* b) {
  int64_t x = *(const int64_t*)a, y = *(const int64_t*)b;
  return (x > y) - (x < y);
}

typedef struct { int64_t k1, k2, row; } o1_pair;
static int cmp_pair(const void* a, const void* b) {
  const o1_pair* x = (const o1_pair*)a;
  const o1_pair* y = (const o1_pair*)b;
  if (x->k1 != y->k1) return (x->k1 > y->k1) - (x->k1 < y->k1);
  return (x->k2 > y->k2) - (x->k2 < y->k2);
}

/* Row indices of the map in increasing key order. */
static int64_t* map_sorted_rows(const o1_map* m) {
  o1_pair* pairs = (o1_pair*)malloc(sizeof(o1_pair) * (m->used ? m->used : 1));
  int64_t* out = (int64_t*)malloc(sizeof(int64_t) * (m->used ? m->used : 1));
  for (int64_t r = 0; r < m->used; ++r) {
    pairs[r].k1 = m->row_keys[r];
    pairs[r].k2 = 0;
    pairs[r].row = r;
  }
  qsort(pairs, (size_t)m->used, sizeof(o1_pair), cmp_pair);
  for (int64_t r = 0; r < m->used; ++r) out[r] = pairs[r].row;
  free(pairs);
  return out;
}

/* ---------------------------------------------------------------- stage A */
static int o1_pixel(double sx, double sy, double sz, int n_face) {
  double ax = fabs(sx), ay = fabs(sy), az = fabs(sz), u, v;
  int face;
  if (ax >= ay && ax >= az) {
    face = sx > 0 ? 0 : 1;
    u = sy / ax;
    v = sz / ax;
  } else if (ay >= az) {
    face = sy > 0 ? 2 : 3;
    u = sx / ay;
    v = sz / ay;
  } else {
    face = sz > 0 ? 4 : 5;
    u = sx / az;
    v = sy / az;
  }
  double quarter = 0.25 * O1_PI;
  int i = (int)((atan(u) + quarter) / (2.0 * quarter) * n_face);
  int j = (int)((atan(v) + quarter) / (2.0 * quarter) * n_face);
  if (i >= n_face) i = n_face - 1;
  if (j >= n_face) j = n_face - 1;
  if (i < 0) i = 0;
  if (j < 0) j = 0;
  return (face * n_face + i) * n_face + j;
}

static int64_t clamp64(int64_t v, int64_t lo, int64_t hi) { return v < lo ? lo : (v > hi ? hi : v); }

static int64_t cell_key(double px, double py, double pz, double cell_m, const double* origin,
                        const int64_t* dims) {
  int64_t cx = clamp64((int64_t)floor((px - origin[0]) / cell_m), 0, dims[0] - 1);
  int64_t cy = clamp64((int64_t)floor((py - origin[1]) / cell_m), 0, dims[1] - 1);
  int64_t cz = clamp64((int64_t)floor((pz - origin[2]) / cell_m), 0, dims[2] - 1);
  return (cx * dims[1] + cy) * dims[2] + cz;
}

/* Pencil table: the fields of finish_pencils, one row per pencil. */
typedef struct {
  int64_t n;
  double *position, *direction, *w0, *w2, *time, *major, *var_major, *var_minor, *pos_cov;
  int64_t *parent, *next; /* coarse-screen hierarchy (preorder), else NULL */
} o1_table;

static int table_alloc(o1_table* t, int64_t n, int hierarchy) {
  int64_t m = n ? n : 1;
  t->n = n;
  t->position = (double*)malloc(sizeof(double) * 3 * m);
  t->direction = (double*)malloc(sizeof(double) * 3 * m);
  t->w0 = (double*)malloc(sizeof(double) * m);
  t->w2 = (double*)malloc(sizeof(double) * m);
  t->time = (double*)malloc(sizeof(double) * m);
  t->major = (double*)malloc(sizeof(double) * 3 * m);
  t->var_major = (double*)malloc(sizeof(double) * m);
  t->var_minor = (double*)malloc(sizeof(double) * m);
  t->pos_cov = (double*)malloc(sizeof(double) * 6 * m);
  t->parent = hierarchy ? (int64_t*)malloc(sizeof(int64_t) * m) : NULL;
  t->next = hierarchy ? (int64_t*)malloc(sizeof(int64_t) * m) : NULL;
  return (t->position && t->direction && t->w0 && t->w2 && t->time && t->major && t->var_major &&
          t->var_minor && t->pos_cov)
             ? 0
             : -1;
}

static void table_free(o1_table* t) {
  free(t->position); free(t->direction); free(t->w0); free(t->w2); free(t->time);
  free(t->major); free(t->var_major); free(t->var_minor); free(t->pos_cov);
  free(t->parent); free(t->next);
  memset(t, 0, sizeof(*t));
}

/* finish_pencils for one accumulated moment row `a` into row q of `t`. */
static void finish_one(const double* a, o1_table* t, int64_t q) {
  double w = a[0];
  double mx = a[2] / w, my = a[3] / w, mz = a[4] / w;
  t->position[3 * q] = mx;
  t->position[3 * q + 1] = my;
  t->position[3 * q + 2] = mz;
  t->time[q] = a[5] / w;
  t->w0[q] = w;
  t->w2[q] = a[1];
  double rx = a[6] / w, ry = a[7] / w, rz = a[8] / w;
  double norm = sqrt(rx * rx + ry * ry + rz * rz);
  double dx = rx / norm, dy = ry / norm, dz = rz / norm;
  t->direction[3 * q] = dx;
  t->direction[3 * q + 1] = dy;
  t->direction[3 * q + 2] = dz;
  double cxx = a[11] / w - rx * rx, cyy = a[12] / w - ry * ry, czz = a[13] / w - rz * rz;
  double cxy = a[14] / w - rx * ry, cxz = a[15] / w - rx * rz, cyz = a[16] / w - ry * rz;
  double hx, hy, hz;
  if (fabs(dz) < 0.9) { hx = 0.0; hy = 0.0; hz = 1.0; } else { hx = 1.0; hy = 0.0; hz = 0.0; }
  double e1x = dy * hz - dz * hy, e1y = dz * hx - dx * hz, e1z = dx * hy - dy * hx;
  double nn = sqrt(e1x * e1x + e1y * e1y + e1z * e1z);
  e1x /= nn; e1y /= nn; e1z /= nn;
  double e2x = dy * e1z - dz * e1y, e2y = dz * e1x - dx * e1z, e2z = dx * e1y - dy * e1x;
  double c11 = (e1x * (cxx * e1x + cxy * e1y + cxz * e1z) + e1y * (cxy * e1x + cyy * e1y + cyz * e1z)
                + e1z * (cxz * e1x + cyz * e1y + czz * e1z));
  double c22 = (e2x * (cxx * e2x + cxy * e2y + cxz * e2z) + e2y * (cxy * e2x + cyy * e2y + cyz * e2z)
                + e2z * (cxz * e2x + cyz * e2y + czz * e2z));
  double c12 = (e1x * (cxx * e2x + cxy * e2y + cxz * e2z) + e1y * (cxy * e2x + cyy * e2y + cyz * e2z)
                + e1z * (cxz * e2x + cyz * e2y + czz * e2z));
  double half = 0.5 * (c11 + c22);
  double disc = sqrt(dmax(0.25 * ((c11 - c22) * (c11 - c22)) + c12 * c12, 0.0));
  t->var_major[q] = dmax(half + disc, 0.0);
  t->var_minor[q] = dmax(half - disc, 0.0);
  double angle = 0.5 * atan2(2.0 * c12, c11 - c22);
  double ca = cos(angle), sa = sin(angle);
  t->major[3 * q] = ca * e1x + sa * e2x;
  t->major[3 * q + 1] = ca * e1y + sa * e2y;
  t->major[3 * q + 2] = ca * e1z + sa * e2z;
  t->pos_cov[6 * q] = dmax(a[17] / w - mx * mx, 0.0);
  t->pos_cov[6 * q + 1] = dmax(a[18] / w - my * my, 0.0);
  t->pos_cov[6 * q + 2] = dmax(a[19] / w - mz * mz, 0.0);
  t->pos_cov[6 * q + 3] = a[20] / w - mx * my;
  t->pos_cov[6 * q + 4] = a[21] / w - mx * mz;
  t->pos_cov[6 * q + 5] = a[22] / w - my * mz;
}

static int64_t parent_key(int64_t key, int face, int parent_face) {
  int64_t per_cell = 6ll * face * face;
  int64_t cell = key / per_cell, pixel = key % per_cell;
  int64_t cube = pixel / ((int64_t)face * face), ij = pixel % ((int64_t)face * face);
  int64_t i = ij / face, j = ij % face;
  int64_t factor = face / parent_face;
  return cell * (6ll * parent_face * parent_face) + (cube * parent_face + i / factor) * parent_face +
         j / factor;
}

typedef struct {
  o1_table fine;   /* finish_pencils of every occupied (cell, pixel) with w0 > 0 */
  o1_table screen; /* pack_pencils layout when a parent face was given */
  int64_t ring_nodes_deposited;
} o1_compressed;

/* compress (prompt.py:1317-1402) with frozen cone cosines `cone`. `origin`
 * and `dims` are the cell grid of the elements' start/end box. With
 * parent_face > 0 the coarse-screen pack is formed too (_prompt_screen.py:
 * compress_screen, pack_pencils). Returns a handle (NULL on failure). */
void* o1c_compress(int64_t n_el, const double* start, const double* direction,
                   const double* length, const double* c0, const double* c2, const double* cone,
                   const double* start_ns, const double* end_ns, double cell_m, int n_face,
                   int ring_nodes, const double* origin, const int64_t* dims, int parent_face) {
  o1_compressed* out = (o1_compressed*)calloc(1, sizeof(o1_compressed));
  if (!out) return NULL;
  o1_map map;
  if (map_init(&map, O1_NM, 4096)) return NULL;
  const double golden = 0.6180339887498949;
  const double a_step = 0.5 * cell_m;
  const int64_t n_pix = 6ll * n_face * n_face;
  const double step_c = cos(O1_TWO_PI / ring_nodes), step_s = sin(O1_TWO_PI / ring_nodes);
  int64_t deposited = 0;
  /* Pencils never span two cells and the reference's ranges hold whole cells,
   * so each bin sums its nodes in (element, sub-segment, ring node) order:
   * the order of this loop. */
  for (int64_t i = 0; i < n_el; ++i) {
    double ux = direction[3 * i], uy = direction[3 * i + 1], uz = direction[3 * i + 2];
    double hx, hy, hz;
    if (fabs(uz) < 0.9) { hx = 0.0; hy = 0.0; hz = 1.0; } else { hx = 1.0; hy = 0.0; hz = 0.0; }
    double e1x = uy * hz - uz * hy, e1y = uz * hx - ux * hz, e1z = ux * hy - uy * hx;
    double norm = sqrt(e1x * e1x + e1y * e1y + e1z * e1z);
    e1x /= norm; e1y /= norm; e1z /= norm;
    double e2x = uy * e1z - uz * e1y, e2y = uz * e1x - ux * e1z, e2z = ux * e1y - uy * e1x;
    double cc = cone[i];
    double cs = sqrt(dmax(1.0 - cc * cc, 0.0));
    int64_t n_a = (int64_t)ceil(length[i] / a_step);
    if (n_a < 1) n_a = 1;
    double share = 1.0 / (double)(n_a * ring_nodes);
    double arc = O1_TWO_PI * cs / ring_nodes;
    double arc2 = arc * arc / 12.0;
    double sl = length[i] / n_a;
    double sub2 = sl * sl / 12.0;
    double w0 = c0[i] * share, w2 = c2[i] * share;
    double offset = fmod((double)i * golden, 1.0) * O1_TWO_PI / ring_nodes;
    for (int64_t ia = 0; ia < n_a; ++ia) {
      double frac = (ia + 0.5) / n_a;
      double px = start[3 * i] + frac * length[i] * direction[3 * i];
      double py = start[3 * i + 1] + frac * length[i] * direction[3 * i + 1];
      double pz = start[3 * i + 2] + frac * length[i] * direction[3 * i + 2];
      double t = start_ns[i] + frac * (end_ns[i] - start_ns[i]);
      int64_t ck = cell_key(px, py, pz, cell_m, origin, dims);
      double cp = cos(offset), sp = sin(offset);
      for (int q = 0; q < ring_nodes; ++q) {
        if (q > 0) {
          double ncp = cp * step_c - sp * step_s;
          sp = sp * step_c + cp * step_s;
          cp = ncp;
        }
        double sx = cc * ux + cs * (cp * e1x + sp * e2x);
        double sy = cc * uy + cs * (cp * e1y + sp * e2y);
        double sz = cc * uz + cs * (cp * e1z + sp * e2z);
        int64_t key = ck * n_pix + o1_pixel(sx, sy, sz, n_face);
        double* row = map_row(&map, key);
        if (!row) return NULL;
        row[0] += w0;
        row[1] += w2;
        row[2] += w0 * px;
        row[3] += w0 * py;
        row[4] += w0 * pz;
        row[5] += w0 * t;
        row[6] += w0 * sx;
        row[7] += w0 * sy;
        row[8] += w0 * sz;
        row[9] += w0 * (px * px + py * py + pz * pz + sub2);
        row[10] += w0 * t * t;
        double tx = -sp * e1x + cp * e2x, ty = -sp * e1y + cp * e2y, tz = -sp * e1z + cp * e2z;
        row[11] += w0 * (sx * sx + arc2 * tx * tx);
        row[12] += w0 * (sy * sy + arc2 * ty * ty);
        row[13] += w0 * (sz * sz + arc2 * tz * tz);
        row[14] += w0 * (sx * sy + arc2 * tx * ty);
        row[15] += w0 * (sx * sz + arc2 * tx * tz);
        row[16] += w0 * (sy * sz + arc2 * ty * tz);
        row[17] += w0 * (px * px + sub2 * ux * ux);
        row[18] += w0 * (py * py + sub2 * uy * uy);
        row[19] += w0 * (pz * pz + sub2 * uz * uz);
        row[20] += w0 * (px * py + sub2 * ux * uy);
        row[21] += w0 * (px * pz + sub2 * ux * uz);
        row[22] += w0 * (py * pz + sub2 * uy * uz);
      }
    }
    deposited += n_a * ring_nodes;
  }
  out->ring_nodes_deposited = deposited;
  int64_t* order = map_sorted_rows(&map);
  int64_t keep = 0;
  for (int64_t r = 0; r < map.used; ++r)
    if (map.values[order[r] * O1_NM] > 0.0) keep++;
  if (table_alloc(&out->fine, keep, 0)) return NULL;
  int64_t* fine_keys = (int64_t*)malloc(sizeof(int64_t) * (keep ? keep : 1));
  int64_t q = 0;
  for (int64_t r = 0; r < map.used; ++r) {
    const double* a = map.values + order[r] * O1_NM;
    if (a[0] > 0.0) {
      fine_keys[q] = map.row_keys[order[r]];
      finish_one(a, &out->fine, q++);
    }
  }
  if (parent_face > 0) {
    /* coarse pencils: the fine rows summed per parent key in (parent, key)
     * order (lexsort((keys, coarse_keys))), then the preorder pack */
    o1_pair* pairs = (o1_pair*)malloc(sizeof(o1_pair) * (map.used ? map.used : 1));
    for (int64_t r = 0; r < map.used; ++r) {
      pairs[r].k1 = parent_key(map.row_keys[r], n_face, parent_face);
      pairs[r].k2 = map.row_keys[r];
      pairs[r].row = r;
    }
    qsort(pairs, (size_t)map.used, sizeof(o1_pair), cmp_pair);
    int64_t n_par = 0;
    for (int64_t r = 0; r < map.used; ++r)
      if (r == 0 || pairs[r].k1 != pairs[r - 1].k1) n_par++;
    double* acc = (double*)calloc((size_t)(n_par ? n_par : 1) * O1_NM, sizeof(double));
    int64_t* par_keys = (int64_t*)malloc(sizeof(int64_t) * (n_par ? n_par : 1));
    int64_t k = -1;
    for (int64_t r = 0; r < map.used; ++r) {
      if (r == 0 || pairs[r].k1 != pairs[r - 1].k1) par_keys[++k] = pairs[r].k1;
      const double* row = map.values + pairs[r].row * O1_NM;
      for (int c = 0; c < O1_NM; ++c) acc[k * O1_NM + c] += row[c];
    }
    int64_t n_coarse = 0;
    for (int64_t p = 0; p < n_par; ++p)
      if (acc[p * O1_NM] > 0.0) n_coarse++;
    o1_table coarse;
    table_alloc(&coarse, n_coarse, 0);
    int64_t* coarse_keys = (int64_t*)malloc(sizeof(int64_t) * (n_coarse ? n_coarse : 1));
    int64_t c = 0;
    for (int64_t p = 0; p < n_par; ++p)
      if (acc[p * O1_NM] > 0.0) {
        coarse_keys[c] = par_keys[p];
        finish_one(acc + p * O1_NM, &coarse, c++);
      }
    /* parent of every fine pencil (searchsorted of its parent key) */
    int64_t n_all = n_coarse + keep;
    if (table_alloc(&out->screen, n_all, 1)) return NULL;
    int64_t* parent_of = (int64_t*)malloc(sizeof(int64_t) * (keep ? keep : 1));
    int64_t* child_start = (int64_t*)calloc((size_t)n_coarse + 1, sizeof(int64_t));
    int64_t* children = (int64_t*)malloc(sizeof(int64_t) * (keep ? keep : 1));
    for (int64_t f = 0; f < keep; ++f) {
      int64_t pk = parent_key(fine_keys[f], n_face, parent_face);
      int64_t lo = 0, hi = n_coarse;
      while (lo < hi) {
        int64_t mid = (lo + hi) / 2;
        if (coarse_keys[mid] < pk) lo = mid + 1; else hi = mid;
      }
      if (lo >= n_coarse || coarse_keys[lo] != pk) return NULL; /* inconsistent hierarchy */
      parent_of[f] = lo;
      child_start[lo + 1]++;
    }
    /* children of each parent in fine-key order (the stable argsort of pack_pencils) */
    for (int64_t p = 0; p < n_coarse; ++p) child_start[p + 1] += child_start[p];
    {
      int64_t* fill = (int64_t*)malloc(sizeof(int64_t) * (n_coarse ? n_coarse : 1));
      for (int64_t p = 0; p < n_coarse; ++p) fill[p] = child_start[p];
      for (int64_t f = 0; f < keep; ++f) children[fill[parent_of[f]]++] = f;
      free(fill);
    }
    /* preorder: each coarse pencil followed by its children in key order */
    int64_t pos = 0;
    o1_table* s = &out->screen;
#define COPY_ROW(src, i, dst_row)                                                  \
  do {                                                                             \
    for (int d = 0; d < 3; ++d) {                                                  \
      s->position[3 * (dst_row) + d] = (src)->position[3 * (i) + d];              \
      s->direction[3 * (dst_row) + d] = (src)->direction[3 * (i) + d];            \
      s->major[3 * (dst_row) + d] = (src)->major[3 * (i) + d];                    \
    }                                                                              \
    for (int d = 0; d < 6; ++d) s->pos_cov[6 * (dst_row) + d] = (src)->pos_cov[6 * (i) + d]; \
    s->w0[dst_row] = (src)->w0[i];                                                 \
    s->w2[dst_row] = (src)->w2[i];                                                 \
    s->time[dst_row] = (src)->time[i];                                             \
    s->var_major[dst_row] = (src)->var_major[i];                                   \
    s->var_minor[dst_row] = (src)->var_minor[i];                                   \
  } while (0)
    for (int64_t p = 0; p < n_coarse; ++p) {
      int64_t root = pos;
      COPY_ROW(&coarse, p, pos);
      s->parent[pos] = -2;
      pos++;
      for (int64_t c = child_start[p]; c < child_start[p + 1]; ++c) {
        COPY_ROW(&out->fine, children[c], pos);
        s->parent[pos] = root;
        s->next[pos] = pos + 1;
        pos++;
      }
      s->next[root] = pos; /* the next root (or the end) */
    }
#undef COPY_ROW
    free(children);
    free(child_start);
    free(parent_of);
    free(coarse_keys);
    table_free(&coarse);
    free(par_keys);
    free(acc);
    free(pairs);
  }
  free(fine_keys);
  free(order);
  map_free(&map);
  return out;
}

int64_t o1c_count(void* handle, int which) {
  o1_compressed* h = (o1_compressed*)handle;
  return which ? h->screen.n : h->fine.n;
}

int64_t o1c_ring_nodes(void* handle) { return ((o1_compressed*)handle)->ring_nodes_deposited; }

void o1c_fetch(void* handle, int which, double* position, double* direction, double* w0,
               double* w2, double* time, double* major, double* var_major, double* var_minor,
               double* pos_cov, int64_t* parent, int64_t* next) {
  o1_compressed* h = (o1_compressed*)handle;
  const o1_table* t = which ? &h->screen : &h->fine;
  int64_t n = t->n;
  memcpy(position, t->position, sizeof(double) * 3 * n);
  memcpy(direction, t->direction, sizeof(double) * 3 * n);
  memcpy(w0, t->w0, sizeof(double) * n);
  memcpy(w2, t->w2, sizeof(double) * n);
  memcpy(time, t->time, sizeof(double) * n);
  memcpy(major, t->major, sizeof(double) * 3 * n);
  memcpy(var_major, t->var_major, sizeof(double) * n);
  memcpy(var_minor, t->var_minor, sizeof(double) * n);
  memcpy(pos_cov, t->pos_cov, sizeof(double) * 6 * n);
  if (which && parent && next) {
    memcpy(parent, t->parent, sizeof(int64_t) * n);
    memcpy(next, t->next, sizeof(int64_t) * n);
  }
}

void o1c_free(void* handle) {
  o1_compressed* h = (o1_compressed*)handle;
  if (!h) return;
  table_free(&h->fine);
  table_free(&h->screen);
  free(h);
}

/* ---------------------------------------------------------------- stage B helpers */
typedef struct {
  int n_gauss;
  const double *tangent, *wsec2;      /* _prepare_gauss_inverse */
  const double* taylor;               /* _IFUNC_TAYLOR [3][24] */
  int n_mono, max_power;
  const double* coef;
  const int64_t *ipow, *jpow;
  double g, y_g, h, h_tail, tail_exp;
  int n_lambda;
  const double *mus, *mut, *speed, *s0w, *s2w;
  int n_edges;
  const double *edges, *eedge, *itab; /* eedge [L][n_edges], itab [L][nb][3] */
  int direct_bins, max_nodes;
  double smoothing, theta_lo, theta_ratio, tau_step, log_r_step, speed_ref;
  int compute_bins;
} o1_params;

static double gauss_inverse_mean(double u, double v, double var_u, double var_v, const o1_params* P) {
  double scale = 2.0 * (var_u + var_v) + u * u + v * v;
  if (scale <= 0.0) return 1e300;
  double s0 = 1.0 / sqrt(scale), total = 0.0;
  for (int k = 0; k < P->n_gauss; ++k) {
    double s = s0 * P->tangent[k], s2 = s * s;
    double a = 1.0 + 2.0 * s2 * var_u, b = 1.0 + 2.0 * s2 * var_v;
    total += P->wsec2[k] * exp(-s2 * (u * u / a + v * v / b)) / sqrt(a * b);
  }
  return 2.0 / sqrt(O1_PI) * s0 * total;
}

static void ifuncs(double z, double ez, const double* taylor, double* i0, double* i1, double* i2) {
  if (fabs(z) < 1.0) {
    double a = taylor[23], b = taylor[24 + 23], c = taylor[48 + 23];
    for (int n = 22; n >= 0; --n) {
      a = a * z + taylor[n];
      b = b * z + taylor[24 + n];
      c = c * z + taylor[48 + n];
    }
    *i0 = a; *i1 = b; *i2 = c;
    return;
  }
  *i0 = (ez - 1.0) / z;
  *i1 = (ez * (z - 1.0) + 1.0) / (z * z);
  *i2 = (ez * (z * z - 2.0 * z + 2.0) - 2.0) / (z * z * z);
}

static double quad_integral(double e_start, double alpha, double beta, double gamma, double width,
                            double kappa, double e_end, const double* taylor) {
  double z = kappa * width;
  double ez = e_start > 0.0 ? e_end / e_start : exp(z);
  double i0, i1, i2;
  ifuncs(z, ez, taylor, &i0, &i1, &i2);
  return e_start * width * (alpha * i0 + width * (beta * i1 + width * gamma * i2));
}

static int find_bin(const double* edges, int nb, double t) {
  if (t < edges[0]) return -1;
  if (t >= edges[nb]) return nb;
  int low = 0, high = nb;
  while (high - low > 1) {
    int middle = (low + high) / 2;
    if (t < edges[middle]) high = middle; else low = middle;
  }
  return low;
}

static void deposit_panel(const o1_params* P, int lam, double t_a, double t_b, double e_a,
                          double e_b, double alpha, double beta, double gamma, double kappa,
                          double* pre, double* acc) {
  const int nb = P->n_edges - 1;
  const double* edges = P->edges;
  const double* eedge = P->eedge + (int64_t)lam * P->n_edges;
  double* A = acc + (int64_t)lam * nb * 4;
  double lo = t_a > edges[0] ? t_a : edges[0];
  double hi = t_b < edges[nb] ? t_b : edges[nb];
  if (hi <= lo) return;
  int k_lo = find_bin(edges, nb, lo), k_hi = find_bin(edges, nb, hi);
  if (k_hi >= nb || (k_hi > k_lo && hi <= edges[k_hi])) k_hi -= 1;
  if (k_hi - k_lo + 1 <= P->direct_bins) {
    for (int k = k_lo; k <= k_hi; ++k) {
      double s_lo = lo > edges[k] ? lo : edges[k];
      double s_hi = hi < edges[k + 1] ? hi : edges[k + 1];
      if (s_hi <= s_lo) continue;
      double e_lo = s_lo == t_a ? e_a : eedge[k];
      if (s_lo != t_a && s_lo != edges[k]) e_lo = exp(kappa * s_lo);
      double e_hi = s_hi == t_b ? e_b : eedge[k + 1];
      if (s_hi != t_b && s_hi != edges[k + 1]) e_hi = exp(kappa * s_hi);
      double shift = s_lo - t_a;
      double a_loc = alpha + shift * (beta + shift * gamma);
      double b_loc = beta + 2.0 * gamma * shift;
      A[k * 4 + 3] += quad_integral(e_lo, a_loc, b_loc, gamma, s_hi - s_lo, kappa, e_hi, P->taylor);
    }
    return;
  }
  double big_a = alpha - t_a * (beta - gamma * t_a);
  double big_b = beta - 2.0 * gamma * t_a;
  double big_c = gamma;
  if (t_a < edges[0]) {
    pre[lam * 3] += big_a;
    pre[lam * 3 + 1] += big_b;
    pre[lam * 3 + 2] += big_c;
  } else {
    int k = k_lo;
    A[k * 4] += big_a;
    A[k * 4 + 1] += big_b;
    A[k * 4 + 2] += big_c;
    A[k * 4 + 3] += quad_integral(e_a, alpha, beta, gamma, edges[k + 1] - t_a, kappa, eedge[k + 1],
                                  P->taylor);
  }
  if (t_b < edges[nb]) {
    int k = find_bin(edges, nb, t_b);
    A[k * 4] -= big_a;
    A[k * 4 + 1] -= big_b;
    A[k * 4 + 2] -= big_c;
    double shift = t_b - t_a;
    double a_loc = alpha + shift * (beta + shift * gamma);
    double b_loc = beta + 2.0 * gamma * shift;
    A[k * 4 + 3] -= quad_integral(e_b, a_loc, b_loc, gamma, edges[k + 1] - t_b, kappa, eedge[k + 1],
                                  P->taylor);
  }
}

static int batch_grid(double r, double sigma, double t_emit_rel, double h, double h_tail,
                      double tail_exp, double mut_min, double speed_max, double edge_end,
                      double* s_buf, int capacity) {
  double ext_end = tail_exp / mut_min;
  double ext_win = speed_max * (edge_end - t_emit_rel) - r;
  if (ext_win < 0.0) ext_win = 0.0;
  if (ext_win > ext_end) ext_win = ext_end;
  double u_end = asinh(ext_end / sigma), u_win = asinh(ext_win / sigma);
  int64_t n_in = u_win > 0.0 ? (int64_t)ceil(u_win / h) : 0;
  int64_t n_out = u_end > u_win ? (int64_t)ceil((u_end - u_win) / h_tail) : 0;
  if (n_in + n_out + 1 > capacity) {
    double scale = (capacity - 1.0) / (double)(n_in + n_out);
    n_in = (int64_t)(n_in * scale);
    n_out = capacity - 1 - n_in;
  }
  s_buf[0] = r;
  int n = 1;
  for (int64_t i = 1; i <= n_in; ++i) s_buf[n++] = r + sigma * sinh(u_win * i / n_in);
  for (int64_t i = 1; i <= n_out; ++i)
    s_buf[n++] = r + sigma * sinh(u_win + (u_end - u_win) * i / n_out);
  return n;
}

static double batch_sigma(double r, double sin_min, double tan_half_min, double y_g) {
  return dmax(0.5 * r * sin_min * dmax(y_g, 0.5 * tan_half_min), 1e-9 * r);
}

static void cubic_coefficients(const double* mom, const o1_params* P, double* a, double* b) {
  a[0] = a[1] = a[2] = a[3] = b[0] = b[1] = b[2] = 0.0;
  for (int m = 0; m < P->n_mono; ++m) {
    double value = P->coef[m] * mom[m];
    int64_t i = P->ipow[m], j = P->jpow[m];
    if (j == 0) {
      if (i == 0) a[0] += value; else if (i == 1) a[1] += value; else if (i == 2) a[2] += value;
      else a[3] += value;
    } else if (j == 1) {
      if (i == 0) b[0] += value; else if (i == 1) b[1] += value; else b[2] += value;
    } else if (j == 2) {
      if (i == 0) { a[0] += value; a[2] -= value; } else { a[1] += value; a[3] -= value; }
    } else {
      b[0] += value;
      b[2] -= value;
    }
  }
}

static void batch_add_moments(int n, const double* s_buf, double r, double sin_t, double cos_t,
                              double jac_sin, const double* mom0, const double* mom2,
                              const o1_params* P, double* g0, double* g2, int backward) {
  double rs = r * sin_t;
  double y_theta = backward ? 0.0 : sin_t / (1.0 + cos_t);
  double jac = backward ? 0.0 : 2.0 / (r * jac_sin);
  double g = P->g, g1 = 1.0 + g * g, gg = 2.0 * g, norm = (1.0 - g * g) / (4.0 * O1_PI);
  int cubic = P->max_power <= 3;
  double A0[4], B0[3], A2[4], B2[3];
  double cpow[8], spow[8];
  if (cubic) {
    cubic_coefficients(mom0, P, A0, B0);
    cubic_coefficients(mom2, P, A2, B2);
  }
  for (int k = 0; k < n; ++k) {
    double c, s, path_jacobian;
    if (backward) {
      double shift = s_buf[k] - r * cos_t;
      double denominator = rs * rs + shift * shift;
      c = (rs * rs - shift * shift) / denominator;
      s = 2.0 * rs * shift / denominator;
      path_jacobian = 2.0 * r / denominator;
    } else {
      double y = (s_buf[k] - r) / rs + y_theta;
      double inv = 1.0 / (1.0 + y * y);
      c = (1.0 - y * y) * inv;
      s = 2.0 * y * inv;
      path_jacobian = jac * inv;
    }
    double a0, a2;
    if (cubic) {
      a0 = A0[0] + c * (A0[1] + c * (A0[2] + c * A0[3]));
      a0 += s * (B0[0] + c * (B0[1] + c * B0[2]));
      a2 = A2[0] + c * (A2[1] + c * (A2[2] + c * A2[3]));
      a2 += s * (B2[0] + c * (B2[1] + c * B2[2]));
    } else {
      cpow[0] = 1.0;
      spow[0] = 1.0;
      for (int p = 1; p <= P->max_power; ++p) {
        cpow[p] = cpow[p - 1] * c;
        spow[p] = spow[p - 1] * s;
      }
      a0 = 0.0;
      a2 = 0.0;
      for (int m = 0; m < P->n_mono; ++m) {
        double basis = P->coef[m] * cpow[P->ipow[m]] * spow[P->jpow[m]];
        a0 += basis * mom0[m];
        a2 += basis * mom2[m];
      }
    }
    double den = g1 - gg * c;
    double value = path_jacobian * norm / (den * sqrt(den));
    g0[k] += a0 * value;
    g2[k] += a2 * value;
  }
}

static void batch_deposit(int n, const double* s_buf, const double* g0, const double* g2, double r,
                          double t_emit_rel, const o1_params* P, double* pre, double* acc,
                          double* charge, double* t_buf, double* h_buf, double front_extra) {
  const int nb = P->n_edges - 1;
  const double* edges = P->edges;
  for (int lam = 0; lam < P->n_lambda; ++lam) {
    if (P->mus[lam] == 0.0) continue;
    double v = P->speed[lam], mut = P->mut[lam];
    double kappa = -mut * v;
    int last = n - 1;
    double limit = r + P->tail_exp / mut;
    while (last > 2 && s_buf[last - 1] > limit) last--;
    if (last < 2) continue;
    double spread = dmin(front_extra + fabs(0.0 - 0.0 / v) * 0.0, (s_buf[last] - r) / v);
    double front_time = t_emit_rel + r / v;
    double end_time = t_emit_rel + s_buf[last] / v;
    int outside = (front_time - 0.5 * spread >= edges[nb] || end_time + 0.5 * spread <= edges[0]);
    double t_base = outside ? 0.0 : t_emit_rel;
    double e_emit = exp(kappa * t_base);
    double h_scale = P->mus[lam] * v / e_emit;
    double w0 = P->s0w[lam] * h_scale, w2 = P->s2w[lam] * h_scale;
    for (int j = 0; j <= last; ++j) {
      t_buf[j] = t_base + s_buf[j] / v;
      h_buf[j] = w0 * g0[j] + w2 * g2[j];
    }
    double h_front = h_buf[0];
    for (int j = 0; j <= last; ++j) h_buf[j] -= h_front;
    double total = 0.0;
    double e_first = e_emit * exp(-mut * s_buf[0]);
    double e_a = e_first, e_last = e_first;
    int j = 0;
    while (j < last) {
      double t_a, t_b, alpha, beta, gamma, e_b;
      int step;
      if (j + 2 <= last) {
        t_a = t_buf[j];
        double t_m = t_buf[j + 1];
        t_b = t_buf[j + 2];
        double u_m = t_m - t_a, u_b = t_b - t_a;
        double d1 = (h_buf[j + 1] - h_buf[j]) / u_m;
        double d2 = ((h_buf[j + 2] - h_buf[j + 1]) / (t_b - t_m) - d1) / u_b;
        alpha = h_buf[j];
        beta = d1 - d2 * u_m;
        gamma = d2;
        e_b = e_emit * exp(-mut * s_buf[j + 2]);
        step = 2;
      } else {
        double t_p = t_buf[j - 1];
        t_a = t_buf[j];
        t_b = t_buf[j + 1];
        double u_m = t_a - t_p, u_b = t_b - t_p;
        double d1 = (h_buf[j] - h_buf[j - 1]) / u_m;
        double d2 = ((h_buf[j + 1] - h_buf[j]) / (t_b - t_a) - d1) / u_b;
        alpha = h_buf[j];
        beta = d1 - d2 * u_m + 2.0 * d2 * u_m;
        gamma = d2;
        e_b = e_emit * exp(-mut * s_buf[j + 1]);
        step = 1;
      }
      double width = t_b - t_a;
      total += quad_integral(e_a, alpha, beta, gamma, width, kappa, e_b, P->taylor);
      if (P->compute_bins && !outside)
        deposit_panel(P, lam, t_a, t_b, e_a, e_b, alpha, beta, gamma, kappa, pre, acc);
      e_a = e_b;
      e_last = e_b;
      j += step;
    }
    double t_f = t_buf[0], t_end = t_buf[last];
    double exact = quad_integral(e_first, h_front, 0.0, 0.0, t_end - t_f, kappa, e_last, P->taylor);
    total += exact;
    if (P->compute_bins && spread > 0.0 && !outside) {
      double t_1 = t_f - 0.5 * spread, t_2 = t_f + 0.5 * spread;
      double e_1 = exp(kappa * t_1), e_2 = exp(kappa * t_2);
      double ramp = quad_integral(e_1, 0.0, 1.0 / spread, 0.0, spread, kappa, e_2, P->taylor);
      double flat = t_end > t_2 ? quad_integral(e_2, 1.0, 0.0, 0.0, t_end - t_2, kappa, e_last, P->taylor)
                                : 0.0;
      double height = ramp + flat != 0.0 ? exact / (ramp + flat) : 0.0;
      deposit_panel(P, lam, t_1, t_2, e_1, e_2, 0.0, height / spread, 0.0, kappa, pre, acc);
      if (t_end > t_2) deposit_panel(P, lam, t_2, t_end, e_2, e_last, height, 0.0, 0.0, kappa, pre, acc);
    } else if (P->compute_bins && t_end > t_f && !outside) {
      deposit_panel(P, lam, t_f, t_end, e_first, e_last, h_front, 0.0, 0.0, kappa, pre, acc);
    }
    charge[lam] += total;
  }
}

static double finalize(const o1_params* P, const double* pre, const double* acc, const double* charge,
                       double area, double* bins_out) {
  const int nb = P->n_edges - 1;
  double total = 0.0;
  for (int lam = 0; lam < P->n_lambda; ++lam) {
    double a = pre[lam * 3], b = pre[lam * 3 + 1], c = pre[lam * 3 + 2];
    const double* eedge = P->eedge + (int64_t)lam * P->n_edges;
    const double* itab = P->itab + (int64_t)lam * nb * 3;
    const double* A = acc + (int64_t)lam * nb * 4;
    for (int k = 0; k < nb; ++k) {
      double e_k = P->edges[k], width = P->edges[k + 1] - e_k;
      double a_loc = a + e_k * (b + c * e_k), b_loc = b + 2.0 * c * e_k;
      double value = eedge[k] * width *
                     (a_loc * itab[k * 3] + width * (b_loc * itab[k * 3 + 1] + width * c * itab[k * 3 + 2]));
      bins_out[k] += area * (value + A[k * 4 + 3]);
      a += A[k * 4];
      b += A[k * 4 + 1];
      c += A[k * 4 + 2];
    }
    total += charge[lam];
  }
  return area * total;
}

/* _pencil_shape_factor_from_ray: (factor, theta_eff, averaged, ok). */
static int shape_factor(int64_t p, double r, double theta, double sine, double hx, double hy,
                        double hz, const double* major, const double* var_major,
                        const double* var_minor, const double* prep, const o1_params* P,
                        double* factor, double* theta_eff, int* averaged) {
  double ax = major[3 * p], ay = major[3 * p + 1], az = major[3 * p + 2];
  const double* pr = prep + 7 * p;
  double bx = pr[0], by = pr[1], bz = pr[2];
  double inv_r2 = 1.0 / (r * r);
  double m11 = var_major[p] + pr[3] * inv_r2;
  double m22 = var_minor[p] + pr[4] * inv_r2;
  double m12 = pr[5] * inv_r2;
  double upper = dmax(m11, m22) + fabs(m12);
  double sf = P->smoothing;
  int far = (dmax(dmax(fabs(m11), fabs(m22)), fabs(m12)) < 1e150 &&
             theta * theta > (sf * sf * dmax(upper, 0.0) * (1.0 + 1e-12)));
  double mu1 = 0.0, mu2 = 0.0, extent = 0.0;
  if (!far) {
    double half_tr = 0.5 * (m11 + m22);
    double disc = sqrt(dmax(0.25 * ((m11 - m22) * (m11 - m22)) + m12 * m12, 0.0));
    mu1 = half_tr + disc;
    mu2 = dmax(half_tr - disc, 1e-16 * mu1 + 1e-300);
    extent = sqrt(dmax(mu1, 0.0));
  }
  double u = hx * ax + hy * ay + hz * az;
  double v = hx * bx + hy * by + hz * bz;
  if (!far && extent > 0.0 && theta < sf * extent) {
    double angle = 0.5 * atan2(2.0 * m12, m11 - m22);
    double ca = cos(angle), sa = sin(angle);
    double mean = gauss_inverse_mean(ca * u + sa * v, -sa * u + ca * v, mu1, mu2, P);
    double f = mean * (sine > 1e-300 ? theta / sine : 1.0);
    *factor = f;
    *theta_eff = f > 1.0 ? asin(dmin(1.0, 1.0 / f)) : theta;
    *averaged = theta < extent;
    return 1;
  }
  if (sine <= 1e-300) {
    *factor = 0.0;
    *theta_eff = theta;
    *averaged = 0;
    return 0;
  }
  double d2 = u * u + v * v;
  double f = 1.0 / sine;
  if (d2 > 0.0) {
    double quad_form = m11 * u * u + 2.0 * m12 * u * v + m22 * v * v;
    f *= 1.0 + 0.5 * (3.0 * quad_form / d2 - (m11 + m22)) / d2;
  }
  *factor = f;
  *theta_eff = theta;
  *averaged = 0;
  return 1;
}

/* inverse_radius_rule (_prompt_screen.py:101-140). */
static void inverse_radius_rule(double u, double v, double var_u, double var_v, const o1_params* P,
                                double* w0, double* t0, double* w1, double* t1) {
  double scale = 2.0 * (var_u + var_v) + u * u + v * v;
  if (scale <= 0.0) { *w0 = *t0 = *w1 = *t1 = 0.0; return; }
  double s0 = 1.0 / sqrt(scale), inverse = 0.0, radial = 0.0;
  for (int k = 0; k < P->n_gauss; ++k) {
    double t = s0 * P->tangent[k];
    double a = 1.0 + 2.0 * t * t * var_u, b = 1.0 + 2.0 * t * t * var_v;
    double mass = P->wsec2[k] * exp(-t * t * (u * u / a + v * v / b)) / sqrt(a * b);
    inverse += mass;
    radial += mass * (var_u / a + var_v / b + u * u / (a * a) + v * v / (b * b));
  }
  double multiplier = 2.0 / sqrt(O1_PI) * s0;
  inverse *= multiplier;
  radial *= multiplier;
  if (inverse <= 0.0) { *w0 = *t0 = *w1 = *t1 = 0.0; return; }
  double mean = 1.0 / inverse, second = radial / inverse;
  double variance = second - mean * mean;
  if (variance <= 0.0) { *w0 = inverse; *t0 = mean; *w1 = 0.0; *t1 = mean; return; }
  double third = (u * u + v * v + var_u + var_v) / inverse;
  double other = (third - 2.0 * mean * second + mean * mean * mean) / variance;
  double disc = sqrt((mean - other) * (mean - other) + 4.0 * variance);
  double low = 0.5 * (mean + other - disc), high = 0.5 * (mean + other + disc);
  double low_weight = inverse * (high - mean) / (high - low);
  *w0 = low_weight; *t0 = low; *w1 = inverse - low_weight; *t1 = high;
}

/* pencil_radial_rule (_prompt_screen.py:143-169). */
static int radial_rule(int64_t p, double r, double theta, double sine, double hx, double hy, double hz,
                       const double* major, const double* var_major, const double* var_minor,
                       const double* prep, const o1_params* P, double* f0, double* th0, double* f1,
                       double* th1, int* averaged) {
  const double* pr = prep + 7 * p;
  double m11 = var_major[p] + pr[3] / (r * r);
  double m22 = var_minor[p] + pr[4] / (r * r);
  double m12 = pr[5] / (r * r);
  double half = 0.5 * (m11 + m22);
  double disc = sqrt(dmax(0.25 * ((m11 - m22) * (m11 - m22)) + m12 * m12, 0.0));
  double mu1 = half + disc, mu2 = dmax(half - disc, 1e-16 * mu1 + 1e-300);
  double extent = sqrt(dmax(mu1, 0.0));
  if (extent > 0.0 && theta < P->smoothing * extent) {
    double u = hx * major[3 * p] + hy * major[3 * p + 1] + hz * major[3 * p + 2];
    double v = hx * pr[0] + hy * pr[1] + hz * pr[2];
    if (sine > 0.0) {
      u *= theta / sine;
      v *= theta / sine;
    }
    double angle = 0.5 * atan2(2 * m12, m11 - m22);
    double ca = cos(angle), sa = sin(angle);
    double w0, t0, w1, t1;
    inverse_radius_rule(ca * u + sa * v, -sa * u + ca * v, mu1, mu2, P, &w0, &t0, &w1, &t1);
    if (t0 > 0.0 && t1 < 0.5 * O1_PI && w0 > 0.0 && w1 >= 0.0) {
      *f0 = w0 * t0 / sin(t0);
      *th0 = t0;
      *f1 = w1 * t1 / sin(t1);
      *th1 = t1;
      *averaged = theta < extent;
      return 1;
    }
  }
  double factor, angle;
  int ok = shape_factor(p, r, theta, sine, hx, hy, hz, major, var_major, var_minor, prep, P, &factor,
                        &angle, averaged);
  *f0 = factor;
  *th0 = angle;
  *f1 = 0.0;
  *th1 = angle;
  return ok;
}

static int64_t theta_index(double theta, double theta_lo, double log_ratio) {
  if (theta < theta_lo) return 0;
  return 1 + (int64_t)(log(theta / theta_lo) / log_ratio);
}

/* grouped_pencils_order1 (parent == NULL) or the coarse screen's
 * screen_order1 (parent/next: the pack_pencils hierarchy) for the OMs in
 * `work`. Writes charge_out[d], bins_out[d][nb] (fine only), groups_out[d],
 * batches_out[d]. Returns 0, or -1 when scratch could not be allocated. */
int o1c_grouped(int64_t n_om, const double* receivers, const double* looks, const double* areas,
                const double* origins, int64_t n_work, const int64_t* work, int64_t n_pen,
                const double* pos, const double* dir, const double* w0p, const double* w2p,
                const double* tp, const double* major, const double* var_major,
                const double* var_minor, const double* pos_cov, const int64_t* parent,
                const int64_t* next, int n_gauss, const double* tangent, const double* wsec2,
                const double* taylor, int n_mono, const double* coef, const int64_t* ipow,
                const int64_t* jpow, int max_power, double g, double y_g, double h, double h_tail,
                double tail_exp, int n_lambda, const double* mus, const double* mut,
                const double* speed, const double* s0w, const double* s2w, int n_edges,
                const double* edges, const double* eedge, const double* itab, int direct_bins,
                int max_nodes, double smoothing, double theta_lo, double theta_ratio,
                double tau_step, double log_r_step, double speed_ref, int compute_bins,
                double* charge_out, double* bins_out, int64_t* groups_out, int64_t* batches_out) {
  (void)n_om;
  o1_params P = {n_gauss, tangent, wsec2, taylor, n_mono, max_power, coef, ipow, jpow,
                 g, y_g, h, h_tail, tail_exp, n_lambda, mus, mut, speed, s0w, s2w,
                 n_edges, edges, eedge, itab, direct_bins, max_nodes, smoothing, theta_lo,
                 theta_ratio, tau_step, log_r_step, speed_ref, compute_bins};
  const int screen = parent != NULL;
  const int nb = n_edges - 1;
  const int nv = 2 * n_mono + 6;
  double mut_min = mut[0], speed_max = speed[0];
  for (int l = 1; l < n_lambda; ++l) {
    mut_min = dmin(mut_min, mut[l]);
    speed_max = dmax(speed_max, speed[l]);
  }
  const double log_ratio = log(1.0 + theta_ratio);
  const int64_t theta_bins = 2 + (int64_t)(log(O1_PI / theta_lo) / log_ratio);
  /* _prepare_pencil_shape */
  double* prep = (double*)malloc(sizeof(double) * 7 * (n_pen ? n_pen : 1));
  for (int64_t p = 0; p < n_pen; ++p) {
    double ax = major[3 * p], ay = major[3 * p + 1], az = major[3 * p + 2];
    double sx = dir[3 * p], sy = dir[3 * p + 1], sz = dir[3 * p + 2];
    double bx = sy * az - sz * ay, by = sz * ax - sx * az, bz = sx * ay - sy * ax;
    const double* cov = pos_cov + 6 * p;
    double* pr = prep + 7 * p;
    pr[0] = bx; pr[1] = by; pr[2] = bz;
    pr[3] = (ax * (cov[0] * ax + cov[3] * ay + cov[4] * az) + ay * (cov[3] * ax + cov[1] * ay + cov[5] * az)
             + az * (cov[4] * ax + cov[5] * ay + cov[2] * az));
    pr[4] = (bx * (cov[0] * bx + cov[3] * by + cov[4] * bz) + by * (cov[3] * bx + cov[1] * by + cov[5] * bz)
             + bz * (cov[4] * bx + cov[5] * by + cov[2] * bz));
    pr[5] = (ax * (cov[0] * bx + cov[3] * by + cov[4] * bz) + ay * (cov[3] * bx + cov[1] * by + cov[5] * bz)
             + az * (cov[4] * bx + cov[5] * by + cov[2] * bz));
    pr[6] = cov[0] + cov[1] + cov[2];
  }
  double* pre = (double*)malloc(sizeof(double) * n_lambda * 3);
  double* acc = (double*)malloc(sizeof(double) * n_lambda * (nb > 0 ? nb : 1) * 4);
  double* charge = (double*)malloc(sizeof(double) * n_lambda);
  double* s_buf = (double*)malloc(sizeof(double) * max_nodes);
  double* t_buf = (double*)malloc(sizeof(double) * max_nodes);
  double* h_buf = (double*)malloc(sizeof(double) * max_nodes);
  double* g0 = (double*)malloc(sizeof(double) * max_nodes);
  double* g2 = (double*)malloc(sizeof(double) * max_nodes);
  double mom0[32], mom2[32], cp[8], sp[8];
  if (!prep || !pre || !acc || !charge || !s_buf || !t_buf || !h_buf || !g0 || !g2 || n_mono > 32 ||
      max_power > 7)
    return -1;
  for (int64_t index = 0; index < n_work; ++index) {
    const int64_t d = work[index];
    memset(pre, 0, sizeof(double) * n_lambda * 3);
    memset(acc, 0, sizeof(double) * n_lambda * (nb > 0 ? nb : 1) * 4);
    memset(charge, 0, sizeof(double) * n_lambda);
    o1_map groups;
    if (map_init(&groups, nv, 1 << 12)) return -1;
    const double rx = receivers[3 * d], ry = receivers[3 * d + 1], rz = receivers[3 * d + 2];
    const double nx = looks[3 * d], ny = looks[3 * d + 1], nz = looks[3 * d + 2];
    const double origin = origins[d];
    int64_t cursor = 0;
    while (cursor < n_pen) {
      int64_t p = cursor++;
      double dx = rx - pos[3 * p], dy = ry - pos[3 * p + 1], dz = rz - pos[3 * p + 2];
      double r = sqrt(dx * dx + dy * dy + dz * dz);
      double hx = dx / r, hy = dy / r, hz = dz / r;
      double t_emit = 0.0, tau = 0.0, log_r = log(r);
      int64_t base;
      if (screen) {
        base = ((int64_t)floor(log(r) / log_r_step) + (1ll << 20)) * 2 * theta_bins;
      } else {
        t_emit = tp[p] - origin;
        tau = t_emit + r / speed_ref;
        int64_t lr_key = (int64_t)floor(log_r / log_r_step) + (1ll << 20);
        int64_t tau_key = clamp64((int64_t)floor(tau / tau_step) + (1ll << 20), 0, (1ll << 21) - 1);
        base = (tau_key * (1ll << 21) + lr_key) * 2 * theta_bins;
      }
      double sx = dir[3 * p], sy = dir[3 * p + 1], sz = dir[3 * p + 2];
      double c1 = 1.0 * (sx * nx + sy * ny + sz * nz);
      double cosine = hx * sx + hy * sy + hz * sz;
      double px = hx - cosine * sx, py = hy - cosine * sy, pz = hz - cosine * sz;
      double sine = sqrt(px * px + py * py + pz * pz);
      double c3 = sine > 1e-300 ? (px * nx + py * ny + pz * nz) / sine : 0.0;
      double theta = atan2(sine, cosine);
      if (screen && parent[p] == -2) {
        double extent2 = var_major[p] + prep[7 * p + 6] / (r * r);
        if (theta < 0.5 * O1_PI && theta * theta < smoothing * smoothing * extent2) continue;
        cursor = next[p];
      }
      int backward = theta > 0.5 * O1_PI;
      double bound = 0.0;
      if (!backward) bound = var_major[p] + var_minor[p] + prep[7 * p + 6] / (r * r);
      double weight, weight2 = 0.0, theta2 = theta;
      int averaged;
      if (backward) {
        weight = 1.0 / r;
        averaged = 0;
      } else if (sine > 1e-300 && bound < 1e-4 * sine * sine) {
        double factor = 1.0 / sine;
        weight = factor / r;
        averaged = 0;
      } else if (screen) {
        double f0, th0, f1, th1;
        if (!radial_rule(p, r, theta, sine, hx, hy, hz, major, var_major, var_minor, prep, &P, &f0,
                         &th0, &f1, &th1, &averaged))
          continue;
        theta = th0;
        theta2 = th1;
        weight = f0 / r;
        weight2 = f1 / r;
      } else {
        double factor, teff;
        if (!shape_factor(p, r, theta, sine, hx, hy, hz, major, var_major, var_minor, prep, &P,
                          &factor, &teff, &averaged))
          continue;
        theta = teff;
        weight = factor / r;
      }
      const double first_weight = weight, first_theta = theta;
      for (int node = 0; node < (weight2 > 0.0 ? 2 : 1); ++node) {
        weight = node == 0 ? first_weight : weight2;
        theta = node == 0 ? first_theta : theta2;
        int64_t i_theta = theta_index(theta, theta_lo, log_ratio);
        int64_t key = base + (int64_t)backward * theta_bins + i_theta;
        double* row = map_row(&groups, key);
        if (!row) return -1;
        /* _fill_moments_averaged_pair */
        double wa = weight * w0p[p], wb = weight * w2p[p];
        cp[0] = 1.0;
        sp[0] = 1.0;
        double perp2 = dmax(1.0 - c1 * c1, 0.0);
        for (int q = 1; q <= max_power; ++q) {
          cp[q] = cp[q - 1] * c1;
          if (averaged) sp[q] = (q % 2 == 1) ? 0.0 : sp[q - 2] * perp2 * (q - 1.0) / q;
          else sp[q] = sp[q - 1] * c3;
        }
        for (int m = 0; m < n_mono; ++m) {
          mom0[m] = wa * cp[ipow[m]] * sp[jpow[m]];
          mom2[m] = wb * cp[ipow[m]] * sp[jpow[m]];
        }
        for (int m = 0; m < n_mono; ++m) {
          row[m] += mom0[m];
          row[n_mono + m] += mom2[m];
        }
        double omega = fabs(mom0[0]);
        row[2 * n_mono] += omega;
        row[2 * n_mono + 1] += omega * theta;
        row[2 * n_mono + 2] += omega * r;
        row[2 * n_mono + 3] += omega * t_emit;
        row[2 * n_mono + 4] += omega * tau;
        row[2 * n_mono + 5] += omega * tau * tau;
      }
    }
    /* batches: groups in key order, one batch per key / theta_bins */
    int64_t used = groups.used;
    int64_t* order = map_sorted_rows(&groups);
    int64_t start = 0, batches = 0;
    while (start < used) {
      int64_t batch_key = groups.row_keys[order[start]] / theta_bins;
      int back = batch_key % 2 == 1;
      int64_t stop = start;
      double omega_sum = 0.0, r_sum = 0.0, t_sum = 0.0, tau_sum = 0.0, tau2_sum = 0.0;
      double theta_small = O1_PI;
      while (stop < used && groups.row_keys[order[stop]] / theta_bins == batch_key) {
        const double* row = groups.values + order[stop] * nv;
        double omega = row[2 * n_mono];
        if (omega > 0.0) {
          omega_sum += omega;
          r_sum += row[2 * n_mono + 2];
          t_sum += row[2 * n_mono + 3];
          tau_sum += row[2 * n_mono + 4];
          tau2_sum += row[2 * n_mono + 5];
          theta_small = dmin(theta_small, row[2 * n_mono + 1] / omega);
        }
        stop++;
      }
      if (omega_sum > 0.0) {
        double r_b = r_sum / omega_sum;
        double t_b = t_sum / omega_sum;
        double tau_mean = tau_sum / omega_sum;
        double tau_var = dmax(tau2_sum / omega_sum - tau_mean * tau_mean, 0.0);
        theta_small = dmax(theta_small, 1e-9);
        double sigma;
        if (back)
          sigma = dmax(0.5 * r_b * sin(theta_small) * y_g, 0.25 * r_b * (1.0 - cos(theta_small)));
        else
          sigma = batch_sigma(r_b, sin(theta_small), tan(0.5 * theta_small), y_g);
        int n = screen ? batch_grid(r_b, sigma, 0.0, h, h, tail_exp, mut_min, speed_max, INFINITY,
                                    s_buf, max_nodes)
                       : batch_grid(r_b, sigma, t_b, h, h_tail, tail_exp, mut_min, speed_max,
                                    edges[nb], s_buf, max_nodes);
        for (int k = 0; k < n; ++k) g0[k] = g2[k] = 0.0;
        for (int64_t q = start; q < stop; ++q) {
          const double* row = groups.values + order[q] * nv;
          double omega = row[2 * n_mono];
          if (omega <= 0.0) continue;
          double th = dmax(row[2 * n_mono + 1] / omega, 1e-9);
          for (int m = 0; m < n_mono; ++m) {
            mom0[m] = row[m];
            mom2[m] = row[n_mono + m];
          }
          double s = sin(th);
          batch_add_moments(n, s_buf, r_b, s, cos(th), s, mom0, mom2, &P, g0, g2, back);
        }
        batch_deposit(n, s_buf, g0, g2, r_b, t_b, &P, pre, acc, charge, t_buf, h_buf,
                      sqrt(12.0 * tau_var));
        batches++;
      }
      start = stop;
    }
    if (compute_bins) {
      charge_out[d] = finalize(&P, pre, acc, charge, areas[d], bins_out + d * nb);
    } else {
      double total = 0.0;
      for (int l = 0; l < n_lambda; ++l) total += charge[l];
      charge_out[d] = areas[d] * total;
    }
    groups_out[d] = used;
    batches_out[d] = batches;
    free(order);
    map_free(&groups);
  }
  free(prep); free(pre); free(acc); free(charge);
  free(s_buf); free(t_buf); free(h_buf); free(g0); free(g2);
  return 0;
}

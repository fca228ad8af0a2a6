/*
 * lighthit_b200.h -- C ABI of the B200 (sm_100a) LightHit per-event transport path.
 *
 * The reference (NeutrinoHit/LightHit) is a Python package; its hot path is a set
 * of NumPy/Numba routines behind TransportKernel / ShowerTransport /
 * EventTransport. Each entry point below replaces one of those routines for a
 * batch of events. The Python host layer (lighthit_b200/) keeps the reference's
 * call surface and binds these symbols through ctypes.
 *
 * Conventions
 *  - Every pointer in a *_problem / *_batch struct is a DEVICE pointer owned by
 *    the caller (tables uploaded once, read-only; outputs caller-allocated),
 *    except where a field says "host".
 *  - Functions return LH_OK or an LH_E* code and never throw across the ABI.
 *  - Data-dependent conditions found on the device (an OM outside the table's
 *    radial range whose bound is above threshold, a source on an OM centre) are
 *    reported in the batch's device `status` block; the host reads it with the
 *    results and raises the reference's ValueError.
 *  - Work is enqueued on `stream` (a cudaStream_t); nothing synchronises.
 */
#ifndef LIGHTHIT_B200_H
#define LIGHTHIT_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LH_OK 0
#define LH_EINVAL 1     /* bad sizes / null pointers (reference: ValueError)   */
#define LH_ECUDA 2      /* a CUDA launch failed                                */
#define LH_ENOMEM 3     /* workspace smaller than required (reference: MemoryError) */
#define LH_ETIMEDOUT 4  /* a bounded device wait gave up                      */
#define LH_EUNSUPPORTED 5

/* status[0] flag bits written by the device */
#define LH_STATUS_COINCIDENT 1u  /* a source sits on an OM centre (transport.py:1072-1073) */
#define LH_STATUS_UNSAFE 2u      /* OM outside range above bound (transport.py:1115-1123)  */
#define LH_STATUS_TIMEOUT 4u     /* a tensor-core pipeline wait timed out                  */

/* Precision / launch modes. */
#define LH_MODE_PLAIN_FP32 0   /* CUDA-core fp32 readout: the plain GPU path          */
#define LH_MODE_SPLIT_BF16 1   /* tcgen05 BF16 hi+lo (3 products), fp32 accumulate    */
#define LH_MODE_BF16 2         /* tcgen05 single BF16 product, fp32 accumulate        */

/* ------------------------------------------------------------------ readout
 * Readout operator: bins[b] = sum_k A[k] * B[b][k] with A the relative spectrum
 * packed as (Re omega_0..n-1, Im omega_0..n-1, zero padding to k_pad).
 * Built on the host from readout.py:9-40 (inverse_bins) composed with the
 * not-a-knot cubic refinement of readout.py:55-62.
 */
typedef struct {
  int32_t n_bins;          /* N: output bins                                   */
  int32_t k_pad;           /* K padded to a multiple of 16 (>= 2*n_omega)      */
  int32_t n_tile;          /* N columns per tensor-core tile (<= 256, %16 == 0) */
  int32_t n_tiles;         /* ceil(n_bins / n_tile)                            */
  const float* b_fp32;     /* [n_bins][k_pad] row-major                        */
  const uint16_t* b_hi;    /* bf16 bits, [n_tiles][k_pad/8][n_tile][8]         */
  const uint16_t* b_lo;    /* bf16 bits, same layout (residual x - hi)         */
} lh_readout_operator;

/* Replaces readout.inverse_bins + CubicSpline refinement (readout.py:43-72) for
 * `rows` spectra already packed in the workspace layout of `mode`.
 * out[row][bin] (row stride `out_row_stride` floats). */
int lh_readout_rows(const lh_readout_operator* op, int mode, const void* a_packed, int64_t rows,
                    float* out, int64_t out_row_stride, int32_t* status, void* stream);

/* Pack `rows` complex spectra (float2, [row][n_omega]) into the A layout of `mode`. */
int lh_readout_pack(const lh_readout_operator* op, int mode, const float* spectra_c64,
                    int32_t n_omega, int64_t rows, void* a_packed, void* stream);

/* Bytes of packed A storage for `rows` rows in `mode`. */
size_t lh_readout_packed_bytes(const lh_readout_operator* op, int mode, int64_t rows);

/* ------------------------------------------------------------------ flashes
 * Replaces TransportKernel._transport_isotropic (transport.py:1061-1164) with
 * ResponseCache.acceptance_spectrum / moments_at (cache.py:294-436) for a batch
 * of monochromatic isotropic flashes sharing one wavelength table.
 */
typedef struct {
  int32_t n_om;
  const double* om_pos;        /* [n_om][3]                                        */
  const double* om_look;       /* [n_om][3] OM orientation (head-on axis)          */
  const double* om_area;       /* [n_om] effective area m^2                        */
  int32_t acc_top;             /* highest significant acceptance degree            */
  const double* alpha;         /* [acc_top+1] Legendre coefficients of acceptance  */
  double efficiency;           /* spectral weight at the flash wavelength          */
  int32_t n_omega;
  const double* omega;         /* [n_omega] rad/ns                                 */
  int32_t n_radii;
  const double* log_r;         /* [n_radii] log of table radii                     */
  const float* coef;           /* float2 [n_radii-1][acc_top+1][2][4][n_omega]    */
  double mu_a, mu_t;           /* absorption, extinction 1/m                       */
  double speed;                /* m/ns of the table's band                        */
  double origin_speed;         /* c / min group index (clock)                      */
  double r_low, r_high;        /* table radial range m                             */
  double threshold;            /* pe                                               */
  int32_t n_edges;
  const double* edges;         /* [n_edges] relative bin edges ns                  */
} lh_flash_problem;

typedef struct {
  int32_t n_flash;
  const double* pos;           /* [n_flash][3]                                     */
  const double* photons;       /* [n_flash]                                        */
  const double* time_ns;       /* [n_flash]                                        */
  float* spectrum;             /* float2 [n_flash][n_om][n_omega][3] absolute      */
  float* components;           /* [n_flash][n_om][3][n_bins]                       */
  double* charge;              /* [n_flash][n_om][3]                               */
  double* origin;              /* [n_flash][n_om]                                  */
  uint8_t* active;             /* [n_flash][n_om] bit0 active, bit1 unsafe, bit2 coincident */
  int32_t* status;             /* [4]: flags, unsafe count, max unsafe radius (double bits) */
  const int32_t* n_flash_device; /* optional: device count (<= n_flash) read by the kernel, so
                                    one captured CUDA graph sized for n_flash serves any batch;
                                    the plain FP32 path writes zero order-1/2 bins for the
                                    flashes past it, the fused path leaves them untouched */
  int32_t block_threads;       /* fused kernel CTA size: 0 (default 512), 256 or 512 */
} lh_flash_batch;

size_t lh_flash_workspace_bytes(const lh_flash_problem* p, const lh_readout_operator* op,
                                int mode, int32_t n_flash);

/* The fused modes (LH_MODE_SPLIT_BF16, LH_MODE_BF16) read op->b_hi / b_lo with
 * their K columns as (Re, Im) per frequency (the A tile's order: one bf16x2
 * store per value); LH_MODE_PLAIN_FP32 reads op->b_fp32 in the order above. */
int lh_flash_transport(const lh_flash_problem* p, const lh_readout_operator* op, int mode,
                       const lh_flash_batch* b, void* workspace, size_t workspace_bytes,
                       void* stream);

/* Broadband flashes (transport.py:1049-1164): the flash is transported at the
 * kernel's wavelength nodes, one lh_flash_transport per node with that node's
 * table and photons (_flash_nodes), the common clock of the fastest node
 * (origin_speed) and threshold +infinity (no mask, no range check); this call
 * sums the node outputs into `b` (spectrum, components, charge) and sets the
 * mask and the range check of the sum: active = inside and total charge >=
 * threshold, unsafe = outside and 10 x sum of the nodes' absorption-only
 * estimates >= threshold (status as lh_flash_transport). `p` is the problem of
 * any node with the real threshold; b->origin is not written (every node run
 * wrote the same clock). */
#define LH_FLASH_MAX_NODES 8
typedef struct {
  int32_t n_nodes;                                /* <= LH_FLASH_MAX_NODES              */
  const float* spectrum[LH_FLASH_MAX_NODES];      /* node runs, layouts of lh_flash_batch */
  const float* components[LH_FLASH_MAX_NODES];
  const double* charge[LH_FLASH_MAX_NODES];
  const double* photons[LH_FLASH_MAX_NODES];      /* [n_flash] photons at each node       */
  double efficiency[LH_FLASH_MAX_NODES];          /* detector spectral weight at the node */
  double absorption[LH_FLASH_MAX_NODES];          /* 1/m at the node                      */
} lh_flash_nodes;

int lh_flash_combine(const lh_flash_problem* p, const lh_flash_nodes* nodes,
                     const lh_flash_batch* b, void* stream);

/* ------------------------------------------------------------------ order >= 2
 * Replaces apply_folded -> apply_multi_spectral -> _apply_multi_spectral
 * (shower/ge2.py:99-119, _shower_basis.py:894-1198): node-band axial sources
 * sharing one point set, contracted with the band-folded RTE kernels. Points,
 * receivers and looks are in the source's axis frame (as apply_multi_spectral
 * rotates them); channels are already aligned to the earliest band reference.
 */
typedef struct {
  int32_t n_bands;             /* folded node bands                                   */
  int32_t n_intervals;         /* radial intervals (log-r knots - 1)                  */
  int32_t degree;              /* kernel degree L (<= 16)                             */
  int32_t acc_degree;          /* detector (acceptance) degree A (<= 4)               */
  int32_t max_m;               /* azimuthal degree min(source M, L) (<= 4)            */
  int32_t n_pairs;             /* detector pairs (<= 8)                               */
  int32_t nch;                 /* kept source channels sum_l (2 min(l, M) + 1)         */
  int32_t n_omega;             /* frequencies of the table (stride of coef)          */
  const float* coef;           /* complex64 [band][interval][l][pair][4][n_omega]     */
  const double* log_r;         /* [n_intervals + 1]                                   */
  const double* absorption;    /* [band] 1/m                                          */
  const double* speed;         /* [band] m/ns                                         */
  const double* omega;         /* [n_omega] rad/ns                                    */
  const int32_t* pair_lambda;  /* [n_pairs]                                           */
  const int32_t* pair_mu;      /* [n_pairs]                                           */
  const double* alpha;         /* [acc_degree + 1] acceptance Legendre coefficients   */
  const int32_t* starts;       /* [degree + 2] first kept channel of each source l    */
  const double* start_norm;    /* [(jmax + 1) (2 jmax + 1)] sqrt(binom(2j, j - nu))    */
  int32_t jmax;                /* max(max_m, acc_degree)                              */
  int32_t flight;              /* table phase is the flight phase                     */
} lh_ge2_table;

typedef struct {
  int32_t n_points;
  const double* points;        /* [n_points][3] axis frame                            */
  const float* channels;       /* complex64 [band][n_points][nch][n_omega_channels]   */
  int32_t n_omega_channels;    /* frequencies stored per channel (1 at zero frequency) */
  int32_t n_omega;             /* frequencies computed: the first n_omega of the table */
  int32_t n_om;
  const double* receivers;     /* [n_om][3] axis frame                                */
  const double* looks;         /* [n_om][3] axis frame                                */
  const double* out_scale;     /* [band][n_om] detector scale (effective area)        */
  double radial_low, radial_high; /* radial window m                                  */
  double reference_ns;         /* emission-time reference of the aligned channels     */
  double* result;              /* complex128 [n_om][n_omega]                          */
} lh_ge2_problem;

size_t lh_ge2_workspace_bytes(const lh_ge2_table* t, const lh_ge2_problem* p);
int lh_ge2_apply(const lh_ge2_table* t, const lh_ge2_problem* p, void* workspace,
                 size_t workspace_bytes, void* stream);

/* Many problems (the events of a batch) on one table in one set of launches:
 * the same per-problem results as n calls of lh_ge2_apply (n <= 65535; a
 * problem without points yields zeros). `host_slots` is caller host memory of
 * lh_ge2_batch_slot_bytes(n) bytes staging the per-problem table copied to the
 * workspace: pageable memory may be reused when the call returns, pinned memory
 * only after the stream has passed the call. */
size_t lh_ge2_batch_workspace_bytes(const lh_ge2_table* t, const lh_ge2_problem* p, int32_t n);
size_t lh_ge2_batch_slot_bytes(int32_t n);
int lh_ge2_apply_batch(const lh_ge2_table* t, const lh_ge2_problem* p, int32_t n,
                       void* workspace, size_t workspace_bytes, void* host_slots, void* stream);

/* The same batch contraction on the tensor cores (tcgen05, BF16 operands with
 * FP32 accumulation in TMEM; mode LH_MODE_SPLIT_BF16 splits every operand into
 * three BF16 parts, hi + mid + lo, and accumulates the six products down to
 * float32 rounding, LH_MODE_BF16 multiplies the hi parts alone). The
 * folded kernels are first packed into the tensor-core operand layout, once per
 * table: lh_ge2_tc_pack_bytes(t) bytes (0: the table's shape is not supported:
 * bands x frequencies > 256, pairs > 8 or rows x 8 too wide), filled by
 * lh_ge2_tc_pack on `stream`. Every problem must compute the table's full
 * spectrum (n_omega == t->n_omega). `status` (device int32) receives
 * LH_STATUS_TIMEOUT if a tensor-core pipeline wait gave up. */
size_t lh_ge2_tc_pack_bytes(const lh_ge2_table* t);
int lh_ge2_tc_pack(const lh_ge2_table* t, void* packed, size_t packed_bytes, void* stream);
size_t lh_ge2_tc_workspace_bytes(const lh_ge2_table* t, const lh_ge2_problem* p, int32_t n);
int lh_ge2_apply_batch_tc(const lh_ge2_table* t, const lh_ge2_problem* p, int32_t n,
                          int32_t mode, const void* packed, void* workspace,
                          size_t workspace_bytes, void* host_slots, int32_t* status,
                          void* stream);

/* ------------------------------------------------------------------ order 0
 * Replaces PreparedBallistic.charge() / .bins(ids, origins, edges)
 * (_surface_ballistic.py:95-118, the first-entry order 0 of transport_prompt,
 * prompt.py:640-660 and 896-903): direct Cherenkov light of spectral elements to
 * the first glass entry of each OM sphere, over the candidate pairs of
 * interval_candidates (_ballistic_interval_numba.py:449-519), integrated by the
 * reference's direct ray form _surface_ballistic_rays.evaluate
 * (_surface_ballistic_rays.py:36-156) at a fixed Gauss order.
 * The optical panels are those of prepare_optics(..., exact_response=True)
 * (ballistic_interval.py:64-161), built once by the reference.
 */
#define LH_STATUS_ON_TRACK 8u             /* point receiver on an emitting track        */
#define LH_STATUS_INSIDE_GLASS 16u        /* emitting segment intersects the glass      */
#define LH_STATUS_NEGATIVE_ACCEPTANCE 32u /* negative ballistic angular response        */
#define LH_STATUS_OVERFLOW 64u            /* more bin cuts in one s / phi range than the
                                             kernel holds (bins finer than the arrival
                                             spread by > 10x): result incomplete        */

typedef struct {
  int32_t n_om;
  const double* om_pos;        /* [n_om][3]                                            */
  const double* om_look;       /* [n_om][3] looks = -orientations                      */
  const double* om_area;       /* [n_om] effective area m^2                            */
  const double* om_radius;     /* [n_om] glass sphere radius m (> 0)                   */
  int32_t n_alpha;             /* acceptance Legendre coefficients (<= 8)              */
  const double* alpha;
  int32_t n_panel_edges;       /* optical panels + 1 (<= 129)                          */
  const double* panel_edges;   /* [n_panel_edges] wavelength nm                        */
  const double* phase;         /* [n_panel_edges] phase index                          */
  const double* group;         /* [n_panel_edges] group index                          */
  const double* extinction;    /* [n_panel_edges] mu_a + mu_s 1/m                      */
  int32_t eff_cols;            /* 4 (cubic) or 6 (cubic x exp(linear))                 */
  const double* efficiency;    /* [n_panel_edges - 1][eff_cols]                        */
  int32_t order;               /* Gauss-Legendre order of every quadrature (<= 64)     */
  const double* gauss_x;       /* [order] nodes on (-1, 1)                             */
  const double* gauss_w;       /* [order] weights                                      */
  /* A second, lower Gauss order evaluated in the same launch when the batch asks
   * for it (charge_check): the per-OM difference of the two charges is the
   * quadrature's error estimate (the reference doubles its order until
   * successive charges agree, _surface_ballistic.py:149-168). 0: none. */
  int32_t check_order;         /* < order                                              */
  const double* check_x;       /* [check_order] nodes                                  */
  const double* check_w;       /* [check_order] weights                                */
} lh_order0_optics;

typedef struct {
  int32_t n_events;
  const int64_t* element_offset; /* [n_events + 1] event e owns elements [off[e], off[e+1]) */
  int64_t n_elements;            /* host: element_offset[n_events]; n_elements * n_om < 2^31 */
  const double* start;           /* [n_el][3] m                                           */
  const double* direction;       /* [n_el][3] unit                                        */
  const double* length;          /* [n_el] m                                              */
  const double* c0;              /* [n_el] Cherenkov C0                                   */
  const double* c2;              /* [n_el] Cherenkov C2 (= -C0 / beta^2)                  */
  const double* beta;            /* [n_el]                                                */
  const double* t0;              /* [n_el] start ns                                       */
  const double* t1;              /* [n_el] end ns                                         */
  const double* origins;         /* [n_events][n_om] time origin ns                       */
  int32_t n_edges;               /* relative time edges; charge only: 2 edges (-1e100, 1e100) */
  const double* edges;           /* [n_edges] ns                                          */
  double* charge;                /* [n_events][n_om] pe (overwritten)                     */
  double* bins;                  /* [n_events][n_om][n_edges-1] pe (overwritten) or NULL  */
  int32_t* status;               /* [1] LH_STATUS_* flags (or-ed in)                      */
  void* workspace;               /* lh_order0_workspace_bytes bytes of device memory      */
  size_t workspace_bytes;
  double* charge_check;          /* [n_events][n_om] charge at optics->check_order
                                    (overwritten), or NULL: no check                      */
} lh_order0_batch;

/* Device scratch for one call: candidate-pair lists (4 bytes per (OM, element)). */
size_t lh_order0_workspace_bytes(const lh_order0_optics* optics, const lh_order0_batch* batch);

int lh_order0(const lh_order0_optics* optics, const lh_order0_batch* batch, void* stream);

/* ------------------------------------------------------------------ order 1
 * Replaces the grouped order 1 of transport_prompt (prompt.py:1020-1258):
 * stage A `compress` (prompt.py:1317-1402; _prompt_numba.py:1094-1232 and
 * finish_pencils :2247-2354) turns elements into (cell, pixel) pencils;
 * stage B `grouped_pencils_order1` (_prompt_numba.py:1750-2086) merges them per
 * OM into (tau, r, theta) groups and deposits each (tau, r) batch's single-
 * scattering profile into the bins. All float64.
 */
typedef struct {
  int32_t n_om;
  const double* om_pos;        /* [n_om][3]                                         */
  const double* om_look;       /* [n_om][3] looks = -orientations                   */
  const double* om_area;       /* [n_om] effective area m^2                         */
  int32_t n_bands;             /* wavelength bands of the unit (<= 8)               */
  const double* mus;           /* [n_bands] scattering 1/m                          */
  const double* mut;           /* [n_bands] extinction 1/m                          */
  const double* speed;         /* [n_bands] group speed m/ns                        */
  const double* s0w;           /* [n_bands] C0 spectral weight (prompt.py:429)      */
  const double* s2w;           /* [n_bands] C2 spectral weight                       */
  double g;                    /* Henyey-Greenstein asymmetry                        */
  int32_t n_mono;              /* acceptance monomials (prompt.py:380-399) (<= 10)   */
  const double* coef;          /* [n_mono]                                          */
  const int32_t* ipow;         /* [n_mono]                                          */
  const int32_t* jpow;         /* [n_mono]                                          */
  int32_t max_power;           /* acceptance degree (<= 4)                           */
  int32_t n_edges;
  const double* edges;         /* [n_edges] relative time edges ns                   */
  const double* eedge;         /* [n_bands][n_edges] exp(kappa edges), kappa = -mut v */
  const double* itab;          /* [n_bands][n_edges-1][3] interval_table             */
  int32_t compute_bins;        /* 0: charge only                                     */
  /* PromptConfig (prompt.py:154-196) */
  double cell_m;               /* pencil position cell                               */
  int32_t pixel_face;          /* cube-sphere pixels per face edge                   */
  int32_t ring_nodes;          /* Cherenkov ring azimuths per sub-segment            */
  double path_step, path_step_tail, tail_exponent;
  int32_t direct_bins, max_path_nodes;  /* max_path_nodes <= 2048                    */
  double smoothing_factor;
  double theta_lo, theta_ratio, tau_step, log_r_step;  /* merge_theta_min/ratio/tau/log_r */
  int32_t theta_bins;          /* 2 + int(log(pi / theta_lo) / log(1 + theta_ratio)) */
  double speed_ref;            /* max band speed                                     */
  int32_t n_gauss;             /* nodes of the Gaussian 1/theta mean (48)            */
  const double* gauss_tau;     /* [n_gauss] on [0, pi/2]                              */
  const double* gauss_w;       /* [n_gauss]                                          */
  int32_t group_capacity;      /* group table slots per OM (power of two, <= 2^20)   */
  /* The coarse charge screen (compress_screen / screen_order1,
   * _prompt_screen.py:91-503) when nonzero: stage A builds pencils at
   * pixel_face under parents at parent_face (pixel_face a multiple of it) and
   * writes parents then children with each child's parent row; stage B uses a
   * parent unless the OM lies inside its angular extent, else its children,
   * keys without the arrival time, the two-node radial rule near the pencil
   * direction and path grids without a window edge (charge only). */
  int32_t screen;
  int32_t parent_face;
} lh_order1_config;

typedef struct {
  int32_t n_el;
  int64_t n_subseg;            /* sum of max(1, ceil(length / (cell_m / 2)))         */
  const int64_t* subseg_offset;/* [n_el + 1] device                                  */
  const double* start;         /* [n_el][3]                                          */
  const double* direction;     /* [n_el][3]                                          */
  const double* length;        /* [n_el]                                             */
  const double* c0;            /* [n_el]                                             */
  const double* c2;            /* [n_el]                                             */
  const double* cone_cos;      /* [n_el] frozen cone cosine 1/(beta n_cone)          */
  const double* t0;            /* [n_el]                                             */
  const double* t1;            /* [n_el]                                             */
  double grid_origin[3];       /* host values: cell grid origin (prompt.py:1321-1326) */
  int64_t grid_dims[3];        /* host values: cells per axis                        */
} lh_order1_elements;

typedef struct {
  int32_t capacity;            /* rows allocated                                     */
  double* position;            /* [capacity][3]                                      */
  double* direction;           /* [capacity][3]                                      */
  double* w0;                  /* [capacity]                                         */
  double* w2;                  /* [capacity]                                         */
  double* time;                /* [capacity]                                         */
  double* major;               /* [capacity][3]                                      */
  double* var_major;           /* [capacity]                                         */
  double* var_minor;           /* [capacity]                                         */
  double* pos_cov;             /* [capacity][6] xx yy zz xy xz yz                    */
  int32_t* parent;             /* [capacity] screen tables: parent row of a child,
                                  -1 for a parent (NULL otherwise)                   */
} lh_order1_pencil_table;

/* Workspace for n_subseg sub-segments and n_work OMs (both stages). */
size_t lh_order1_workspace_bytes(const lh_order1_config* config, int64_t n_subseg, int32_t n_work);

/* Stage A: pencils of the elements; *n_pencils_device receives the count. */
int lh_order1_pencils(const lh_order1_config* config, const lh_order1_elements* elements,
                      const lh_order1_pencil_table* pencils, int32_t* n_pencils_device,
                      void* workspace, size_t workspace_bytes, int32_t* status, void* stream);

/* Stage B: charge[n_om] and bins[n_om][n_edges-1] of the OMs in work[n_work]
 * (others zero), clocks origins[n_om]. n_pencils bounds the table rows used;
 * n_pencils_device (optional, device) holds the stage-A count, read on the device. */
int lh_order1_grouped(const lh_order1_config* config, const lh_order1_pencil_table* pencils,
                      int32_t n_pencils, const int32_t* n_pencils_device,
                      const int32_t* work, int32_t n_work,
                      const double* origins, double* charge, double* bins, void* workspace,
                      size_t workspace_bytes, int32_t* status, void* stream);

/* ------------------------------------------------------------------ order >= 2 source
 * Replaces node_sources (shower/ge2.py:35-67) -> compile_axial_slices
 * (_shower_basis.py:188-645) with the shower basis: axial slices x cubic
 * Lagrange weights x 5-moment transverse stencil x real harmonics P_l(mu_C) Y_lm,
 * deposited on a linear time lattice and transformed to the route frequencies.
 * Every element must emit in every node band (one lattice for all bands).
 * Small per-problem tables are passed by value; pointers are device memory.
 */
typedef struct {
  int32_t n_el;
  const double* start;          /* [n_el][3]                                          */
  const double* direction;      /* [n_el][3]                                          */
  const double* length;         /* [n_el]                                             */
  const double* c0;             /* [n_el]                                             */
  const double* c2;             /* [n_el]                                             */
  const double* beta;           /* [n_el]                                             */
  const double* t0;             /* [n_el]                                             */
  const double* t1;             /* [n_el]                                             */
  int32_t n_bands;              /* node bands (<= 8)                                  */
  double band_s0[8];            /* 1 / lambda^2 (shower/ge2.py:30)                    */
  double band_s2[8];            /* 1 / (lambda^2 n^2)                                 */
  double band_phase[8];         /* phase index n of the band (cone 1 / (beta n))      */
  double band_scale[8];         /* fold scale of the band (shower/ge2.py:66)          */
  double centre[3], first[3], second[3], axis[3];  /* AxisFrame of the prompt steps     */
  int32_t degree, max_m, nch;   /* source degree, azimuthal degree, kept channels     */
  int32_t starts[18];           /* first kept channel of each degree (axial_fast._layout) */
  int32_t channel_degree[153];  /* degree l of each kept channel                      */
  double aa[85], bb[85];        /* [(degree+1)(max_m+1)] Legendre recurrences        */
  int32_t element_order;        /* Gauss nodes per chord (1 or 2)                     */
  double node_fraction[2], node_weight[2];
  double cell_m, stencil_m, stencil_threshold_m, time_step_ns;
  double reference_ns;          /* earliest emission (time lattice origin)            */
  double z_origin;              /* slice lattice origin (min node z - 2 cells)        */
  int64_t n_slices, kmax;       /* slice and tick lattice sizes                       */
  int32_t n_omega;
  const double* omega;          /* [n_omega] rad/ns                                   */
} lh_source_problem;

typedef struct {
  int64_t capacity;             /* points per band allocated (>= 5 n_slices)          */
  double* points;               /* [n_bands][capacity][3] (z, x, y) in the frame      */
  float* channels;              /* complex64 [n_bands][capacity][nch][n_omega]         */
  int32_t* n_points;            /* [n_bands] points written per band                  */
} lh_source_output;

size_t lh_source_workspace_bytes(const lh_source_problem* problem);
int lh_source_compile(const lh_source_problem* problem, const lh_source_output* output,
                      void* workspace, size_t workspace_bytes, int32_t* status, void* stream);

/* ------------------------------------------------------------------ per-OM geometry
 * Replaces min_distance_to_segments (_prompt_numba.py:2221-2243, the module
 * selection of transport_prompt, prompt.py:603-631) and
 * earliest_element_arrival (_shower_basis.py:50-78, the clock of an extended
 * source, shower/api.py:466-473), float64 bit-identical, for several events.
 */
typedef struct {
  int32_t n_om;
  const double* om_pos;          /* [n_om][3]                                         */
  int32_t n_events;              /* <= 65535                                          */
  const int64_t* element_offset; /* [n_events + 1]                                    */
  const double* start;           /* [n_el][3]                                         */
  const double* direction;       /* [n_el][3] unit                                    */
  const double* length;          /* [n_el]                                            */
  const double* start_ns;        /* [n_el]                                            */
  double group_index;            /* fastest group index (flight n_g / c)              */
  double* min_distance;          /* [n_events][n_om] or NULL                          */
  double* earliest_ns;           /* [n_events][n_om] or NULL                          */
} lh_om_geometry_problem;

int lh_om_geometry(const lh_om_geometry_problem* geometry, void* stream);

/* ------------------------------------------------------------------ radial window
 * Replaces the radial-window pass of ShowerTransport (shower/api.py:322-340 with
 * the far-tail screen of shower_basis.py:408-439): for every (event, node band,
 * OM) the number of basis points closer than radial_low and farther than
 * radial_high (float64, bit-identical to the reference's NumPy distances), and the
 * far-tail sum  sum_far photons_c exp(interp(r, att_radius, att_log)) / (4 pi r^2),
 * photons_c = photon_scale |channel_c(0, 0)| / efficiency_band.
 * Basis points are in the axis frame (z, x, y) of their event, as the source
 * compile writes them; world = ((centre + z axis) + x first) + y second. */
typedef struct {
  int32_t n_points[8];          /* basis points of each node band                     */
  int32_t capacity;             /* points stride between bands                        */
  const double* points;         /* [band][capacity][3] (z, x, y)                      */
  const float* channels;        /* complex64 [band][capacity][channel_stride/2]       */
  int32_t channel_stride;       /* floats per point (2 nch n_omega)                   */
  double centre[3], axis[3], first[3], second[3];
} lh_window_event;

typedef struct {
  int32_t n_om, n_bands;
  const double* om_pos;         /* [n_om][3]                                          */
  double radial_low, radial_high;
  int32_t n_att;
  const double* att_radius;     /* [n_att] ascending                                  */
  const double* att_log;        /* [n_att]                                            */
  double photon_scale;          /* sqrt(4 pi)                                         */
  double efficiency[8];         /* of each node band                                  */
  int32_t* n_near;              /* [event][band][n_om]                                */
  int32_t* n_far;               /* [event][band][n_om]                                */
  double* far_sum;              /* [event][band][n_om]                                */
} lh_radial_window_problem;

/* `events` (host memory, n_events <= 65535 / n_bands) is copied on the stream
 * into the workspace (lh_window_slot_bytes(n_events) bytes of device memory);
 * pageable `events` may be reused when the call returns. */
size_t lh_window_slot_bytes(int32_t n_events);
int lh_radial_window(const lh_radial_window_problem* problem, const lh_window_event* events,
                     int32_t n_events, void* workspace, size_t workspace_bytes, void* stream);

/* ------------------------------------------------------------------ near field
 * Replaces near_field_ge2 (near_field.py:91-171) with near_portions (:39-69):
 * the order >=2 light of every element portion closer than radius_m to an OM
 * (points the order >=2 tables leave out), with the Green function clamped at
 * the table's radial minimum along the same directions and the flight phase of
 * the actual distance (_cone_many_looks with clamp_low = 0,
 * muon/track_ge2_primitive.py:612-660), per unit-coefficient spectral cone
 * harmonics (near_field.py:72-88), Gauss panels of panel_m along each portion.
 * Per OM the portions are summed in element order.
 */
typedef struct {
  int32_t n_lambda;            /* kernel wavelength nodes (<= 8)                      */
  int32_t degree;              /* kernel degree L (<= 16)                             */
  int32_t acc_degree;          /* detector degree A (<= 4)                            */
  int32_t n_pairs;             /* detector pairs (<= 8)                               */
  int32_t n_omega;             /* frequencies                                         */
  const float* coef;           /* complex64 [lambda][l][pair][4][n_omega]: the first
                                  radial interval of the per-wavelength splines        */
  double log_r0, log_r1;       /* that interval in log m; exp(log_r0) is the clamp     */
  double radial_high;          /* table radial maximum m                              */
  const double* absorption;    /* [lambda] 1/m                                        */
  const double* speed;         /* [lambda] m/ns                                       */
  const double* omega;         /* [n_omega] rad/ns                                    */
  const int32_t* pair_lambda;  /* [n_pairs]                                           */
  const int32_t* pair_mu;      /* [n_pairs]                                           */
  const double* alpha;         /* [acc_degree + 1] acceptance Legendre coefficients   */
  const double* start_norm;    /* [(acc_degree + 1)(2 acc_degree + 1)] sqrt(binom(2j, j - nu)) */
  int32_t flight;              /* splines hold the flight phase                       */
  const double* wavelength_nm; /* [lambda]                                            */
  const double* phase_index;   /* [lambda] cone phase index                           */
  const double* spectral_weight; /* [lambda] wavelength weight nm x detector efficiency */
  int32_t gauss_order;         /* nodes per panel (<= 16)                             */
  const double* gauss_x;       /* [gauss_order] on (-1, 1)                            */
  const double* gauss_w;       /* [gauss_order]                                       */
  double panel_m;              /* panel length along a portion                        */
} lh_near_table;

typedef struct {
  int32_t n_om;
  const double* om_pos;        /* [n_om][3]                                           */
  const double* om_look;       /* [n_om][3] looks = -orientations                     */
  const double* om_area;       /* [n_om] effective area m^2                           */
  const double* time_origin_ns; /* [n_om] clock of the response                       */
  int32_t n_elements;
  const double* start_m;       /* [n][3]                                              */
  const double* direction;     /* [n][3] unit                                         */
  const double* length_m;      /* [n] (> 0)                                           */
  const double* coefficient0;  /* [n]                                                 */
  const double* coefficient2;  /* [n]                                                 */
  const double* beta;          /* [n]                                                 */
  const double* start_ns;      /* [n]                                                 */
  const double* end_ns;        /* [n]                                                 */
  double radius_m;             /* portions closer than this (<= exp(log_r0))          */
  double* spectrum;            /* complex128 [n_om][n_omega] relative to the OM clock  */
  double* charge;              /* [n_om] zero-frequency real part                     */
  int32_t* portions;           /* [n_om][2]: portions, portions with nonzero harmonics */
} lh_near_problem;

size_t lh_near_workspace_bytes(const lh_near_table* t, const lh_near_problem* p);
int lh_near_field(const lh_near_table* t, const lh_near_problem* p, void* workspace,
                  size_t workspace_bytes, void* stream);

/* Kernel timing for measurement runs (the reference reports per-stage wall
 * times in metadata['timings'], shower/api.py:243-420; these are the device
 * durations of the main kernels behind those stages). lh_kernel_timing(1)
 * clears the record and starts it; while on, every timed launch records a CUDA
 * event pair on its own stream (not while that stream is being captured).
 * lh_kernel_timing_read waits for the recorded events and returns per kernel
 * id the launch count and the summed milliseconds. */
enum {
  LH_KT_ORDER0 = 0,      /* order0_kernel (lh_order0)                */
  LH_KT_O1_RING = 1,     /* o1_ring_kernel (lh_order1_pencils)       */
  LH_KT_O1_GROUP = 2,    /* o1_group_kernel (lh_order1_grouped)      */
  LH_KT_O1_BATCH = 3,    /* o1_batch_kernel (lh_order1_grouped)      */
  LH_KT_GE2_APPLY = 4,   /* ge2_apply_batch_kernel (lh_ge2_apply_batch)  */
  LH_KT_SRC_GROUP = 5,   /* src_group_kernel (lh_source_compile)     */
  LH_KT_SRC_TRANSFORM = 6, /* src_transform_kernel (lh_source_compile) */
  LH_KT_READOUT = 7,     /* readout_tc_kernel (lh_readout_rows)      */
  LH_KT_FLASH = 8,       /* flash_tc_kernel (lh_flash_transport)     */
  LH_KT_GE2_TC = 9,      /* ge2_tc_kernel (lh_ge2_apply_batch_tc)    */
  LH_KT_COUNT = 10
};
int lh_kernel_timing(int enable);
int lh_kernel_timing_read(int32_t n_kernels, int64_t* launches, double* total_ms);
/* Algorithmic work units of the timed kernels, counted on the device by every
 * launch since the last lh_kernel_timing(1) (after a device synchronisation):
 * (OM, pencil) evaluations for o1_group_kernel, float32 integrand
 * evaluations (one wavelength x along-track x azimuth node of a piece) for
 * order0_kernel, (OM, point) pairs inside the radial window for the
 * tensor-core >=2 contraction, 0 for the kernels that do not count. */
int lh_kernel_units_read(int32_t n_kernels, int64_t* units);

/* Host function (no device work): the weighted centre and the lower triangle
 * of the weighted covariance of the element midpoints start + length/2 *
 * direction with weights `share` (summing to one), summed in element order
 * with every product rounded to float64 as NumPy evaluates AxisFrame.of's
 * expressions (axial_source.py:88-118). centre[3], covariance[3][3] (upper
 * triangle zero). */
int lh_axis_frame_sums(int64_t n, const double* start, const double* direction,
                       const double* length, const double* share, double* centre,
                       double* covariance);

/* Host function (no device work): low[3], high[3] = the per-coordinate minima
 * and maxima over the element starts and ends start + length * direction, the
 * box of compress's cell grid (prompt.py:1317-1402). NaN coordinates give NaN
 * bounds. */
int lh_element_box(int64_t n, const double* start, const double* direction,
                   const double* length, double* low, double* high);

/* Host function (no device work): delay[i] = (start_ns[i] - start_ns[first])
 * - |start[i] - start[first]| / c_m_per_ns, the steps' delays behind the light
 * front of step `first` in delay_groups (shower/ge2.py:122-147), rounded as
 * NumPy evaluates that expression; `distance` (may be NULL) receives
 * |start[i] - start[first]|. */
int lh_element_delays(int64_t n, const double* start, const double* start_ns, int64_t first,
                      double c_m_per_ns, double* delay, double* distance);

/* Host function (no device work): the sub-segments of compress
 * (prompt.py:1317-1402): element i is cut into max(1, ceil(length[i] / a_step))
 * pieces; offsets[0..n] are the running totals (offsets[0] = 0) and *n_sub the
 * sum. LH_EINVAL for a negative or non-finite length. */
int lh_subsegment_offsets(int64_t n, const double* length, double a_step, int64_t* offsets,
                          int64_t* n_sub);

/* Flash transport that allocates nothing (no counterpart in the reference).
 * For callers that cannot allocate device memory: processes whose device memory
 * is reserved up front by their own framework's allocator (trigger/DAQ farms),
 * and latency-critical loops where cudaMalloc/cudaFree would synchronise the
 * device. Runs the plain FP32 path (as lh_flash_transport with
 * LH_MODE_PLAIN_FP32) with its scratch in a static 4 MiB __device__ array of the
 * library: at most 2 * n_flash * n_om * k_pad * 4 bytes, e.g. 75 flashes of a
 * 48-OM array at k_pad = 144; larger batches return LH_ESCRATCH and launch
 * nothing. The caller still passes inputs and outputs. The first call on a
 * device looks up the array's device address (cudaGetSymbolAddress) with that
 * device current, so make it before any stream capture. The address is kept
 * for the life of the process: after cudaDeviceReset on a device (which ends
 * the context the address belongs to) this entry point must not be called on
 * that device again. All calls on a device share the array: calls that overlap
 * on the GPU race and must be serialised. */
#define LH_ESCRATCH 6   /* request larger than the static scratch of the entry point below */
int lh_flash_transport_noalloc(const lh_flash_problem* p, const lh_readout_operator* op,
                               const lh_flash_batch* b, void* stream);

/* Failure detection without a fault (no counterpart in the reference). Every
 * wait of the tensor-core kernels on an mbarrier gives up after 1 s of global
 * time; the kernel then sets LH_STATUS_TIMEOUT in its status word, finishes
 * its own copies, frees its tensor memory and returns, and the host raises.
 * This entry point runs one such wait, limited to `limit_ns` (0 < limit_ns
 * <= 1e9), on an mbarrier that nothing completes: `status` (device, 8-byte
 * aligned, int32[4]) gets LH_STATUS_TIMEOUT in status[0] and the nanoseconds
 * waited in status[2..3] (uint64). */
int lh_wait_selftest(int32_t* status, int64_t limit_ns, void* stream);

/* Library version string (host). */
const char* lh_version(void);

#ifdef __cplusplus
}
#endif

#endif /* LIGHTHIT_B200_H */

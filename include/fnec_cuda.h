/*
 * fnec_cuda.h -- C ABI of libfnec_cuda.so, the B200 (sm_100a) backend for
 * the Hallen method-of-moments hot path of dc0sk/fnec-rust.
 *
 * The library replaces the wgpu entry points of the reference's `nec_accel`
 * crate (crates/nec_accel/src/lib.rs:52-96, wgpu_device.rs) and adds the
 * batched / device-resident interface the CUDA path is built around.  All
 * pointers are plain host pointers; sizes are element counts; complex
 * numbers are interleaved (re, im) doubles.  Every function returns an int
 * status (FNEC_OK == 0, negative on error); there is no CPU fallback: a
 * call that cannot run on the GPU returns an error and does nothing else.
 *
 * Reference interfaces replaced (file:line within dc0sk/fnec-rust):
 *   fnec_fill_zmatrix            <- fill_zmatrix_wgpu            crates/nec_accel/src/wgpu_device.rs:832
 *   fnec_solve_hallen_resident   <- solve_hallen_gpu_resident    crates/nec_accel/src/wgpu_device.rs:1294
 *   fnec_solve_hallen            <- solve_hallen                 crates/nec_solver/src/linear.rs:672
 *   fnec_rp_farfield_batch       <- run_rp_farfield_batch_wgpu   crates/nec_accel/src/wgpu_device.rs:461
 *   fnec_radiation_pattern       <- compute_radiation_pattern    crates/nec_solver/src/farfield.rs:563
 *   fnec_integrate_radiated_power<- integrate_radiated_power     crates/nec_solver/src/farfield.rs:409
 *   fnec_near_field              <- near_e_field / near_h_field  crates/nec_solver/src/farfield.rs:154, :218
 *   fnec_microbench_zmatrix_dispatch <- microbench_zmatrix_dispatch crates/nec_accel/src/wgpu_device.rs:1087
 *   fnec_enumerate_devices       <- enumerate_compute_adapters   crates/nec_accel/src/wgpu_device.rs:24
 *   fnec_dispatch_frequency_point<- dispatch_frequency_point     crates/nec_accel/src/lib.rs:92
 *   fnec_batch_*                 <- the per-frequency loop of execute_frequency_sweep /
 *                                   solve_frequency_point (apps/nec-cli/src/solve_session.rs:1186, :1782)
 */
#ifndef FNEC_CUDA_H
#define FNEC_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---------------------------------------------------- */
#define FNEC_OK 0
#define FNEC_ERR_BAD_ARG (-1)          /* invalid argument / geometry      */
#define FNEC_ERR_NO_DEVICE (-2)        /* no CUDA device / wrong arch      */
#define FNEC_ERR_OUT_OF_MEMORY (-3)    /* device allocation failed         */
#define FNEC_ERR_CUDA (-4)             /* CUDA runtime error               */
#define FNEC_ERR_SINGULAR (-5)         /* pivot below 1e-30 (linear.rs:1354)*/
#define FNEC_ERR_SEGMENT_NOT_FOUND (-6)/* EX card without its segment      */
#define FNEC_ERR_UNSUPPORTED (-7)      /* feature not built                */
#define FNEC_ERR_TIMEOUT (-8)          /* bounded device wait expired      */
#define FNEC_ERR_BUSY (-9)             /* admission refused (HBM budget)   */
#define FNEC_ERR_TOO_LARGE (-10)       /* beyond a fixed static maximum    */

/* Per-unit status word of a batch (fnec_batch_read): 0, -(column+1) of a
 * singular pivot, or FNEC_UNIT_TIMEOUT when a wait between the CTAs of a
 * grid-wide kernel ran out of time (the unit's results are void). */
#define FNEC_UNIT_TIMEOUT 0x40000000

#define FNEC_GROUND_FREE 0             /* GroundModel::FreeSpace           */
#define FNEC_GROUND_PEC 1              /* GroundModel::PerfectConductor    */

/* pipeline phases timed by fnec_batch_phase_ms (CUDA events on the
 * context stream, recorded only while profiling is on) */
#define FNEC_N_PHASES 8
#define FNEC_PHASE_EXPAND 0   /* GW -> segments                 */
#define FNEC_PHASE_RHS 1      /* Hallen RHS and cos(k s)        */
#define FNEC_PHASE_FILL 2     /* Z fill                         */
#define FNEC_PHASE_GRAM 3     /* normal equations M^H M + lambda */
#define FNEC_PHASE_FACTOR 4   /* elimination / factorisation    */
#define FNEC_PHASE_SOLVE 5    /* back substitution / refinement */
#define FNEC_PHASE_FEED 6     /* feedpoint rows                 */
#define FNEC_PHASE_FARFIELD 7 /* pattern grid + power integral  */

#define FNEC_PRECISION_FP64 0          /* plain FP64, bit-exact operation order */
#define FNEC_PRECISION_MIXED 1         /* FP32 factor + FP64 GMRES refinement   */

/* ---- data records ----------------------------------------------------- */

/* ZSegmentInput (wgpu_device.rs:811-816) */
typedef struct {
    double midpoint[3];
    double direction[3];
    double length;
    double radius;
} fnec_zsegment;

/* GpuSegment (gpu_kernels.rs:52-59) */
typedef struct {
    double midpoint[3];
    double direction[3];
    double length;
} fnec_gpu_segment;

/* RpGpuResult (wgpu_device.rs:139-148).  axial_ratio is the Stokes axial
 * ratio of farfield.rs:659-667 (the CPU path's definition). */
typedef struct {
    double u_theta;
    double u_phi;
    double gain_total_dbi;
    double gain_theta_dbi;
    double gain_phi_dbi;
    double axial_ratio;
    double theta_deg;
    double phi_deg;
} fnec_rp_result;

/* One junction constraint I[seg_a] + sign * I[seg_b] = 0 (geometry.rs:255-262) */
typedef struct {
    uint64_t seg_a;
    uint64_t seg_b;
    double sign;
} fnec_junction;

/* One GW card (geometry.rs:710-754 expands it) */
typedef struct {
    uint32_t tag;
    uint32_t segments;
    double start[3];
    double end[3];
    double radius;
} fnec_wire;

/* One voltage-source EX card (types 0 and 5), in deck order */
typedef struct {
    uint32_t tag;
    uint32_t segment;
    double v_re;
    double v_im;
} fnec_source;

/* One RP card (farfield.rs:677-699: phi outer, theta inner) */
typedef struct {
    uint32_t n_theta;
    uint32_t n_phi;
    double theta0;
    double phi0;
    double d_theta;
    double d_phi;
} fnec_rp_card;

/* The first plane-wave EX card of a deck (EX types 1, 2, 3; card.rs ExCard
 * via planewave.rs:60-80 and solve_session.rs:313-355): the wave arrives
 * from (theta0, phi0) degrees with polarisation angle eta (F3); types 2 / 3
 * are right / left elliptic with axial ratio F6, type 1 linear.  I2 x I3 =
 * n_theta x n_phi incidence directions stepped by (d_theta, d_phi) (F4, F5)
 * form the receive sweep, theta outer, phi inner; the first direction is
 * the deck's own solve. */
typedef struct {
    uint32_t ex_type;
    uint32_t n_theta, n_phi;
    uint32_t reserved;
    double theta0, phi0, eta;
    double d_theta, d_phi;
    double axial_ratio;
} fnec_plane_wave;

/* One LD card (nec_model card.rs:265-279; applied by loads.rs:103-222 and
 * solve_session.rs:1285-1289): load type 0 series RLC, 1 parallel RLC,
 * 2 series RL, 3 series RC, 4 series R + jX, 5 wire conductivity (other
 * types are ignored, as the reference ignores them with a warning); tag 0
 * = every tag; seg_first 0 = every segment of the tag; seg_last 0 = seg_first. */
typedef struct {
    int32_t load_type;
    uint32_t tag;
    uint32_t seg_first;
    uint32_t seg_last;
    double f1, f2, f3;
} fnec_load;

/* One TL card (card.rs TlCard; stamped by tl.rs:47-183 as in
 * solve_session.rs:1290-1296): the line's ends (tag, segment; segment 0 =
 * the tag's centre segment, the lower one of an even count), sections
 * (stamped as one section), type (0 lossless with velocity factor f3 when
 * 0 < f3 <= 1, else 1; any other type lossy with f3 the matched-line loss in
 * dB), z0 (> 0) and length (> 0).  Cards that cannot stamp are ignored, as
 * the reference ignores them with a warning. */
typedef struct {
    uint32_t tag1, seg1, tag2, seg2;
    uint32_t num_segments, tl_type;
    double z0, length, f3;
} fnec_tl;

/* One NT card with its ten fields parsed (network.rs:55-142): the ends and
 * the reciprocal two-port's short-circuit admittances Y11, Y12 = Y21, Y22;
 * stamped as [Z] = [Y]^-1.  A singular [Y] or coincident ends are ignored. */
typedef struct {
    uint32_t tag1, seg1, tag2, seg2;
    double y11_re, y11_im, y12_re, y12_im, y22_re, y22_im;
} fnec_nt;

/* One antenna of a batch: its geometry, sources, ground, frequency list and
 * optional pattern request.  Each frequency is one unit (one solve). */
typedef struct {
    const fnec_wire *wires;
    uint32_t n_wires;
    const fnec_source *sources;
    uint32_t n_sources;
    int32_t ground;
    uint32_t n_freqs;
    const double *freqs_hz;
    const fnec_rp_card *rp; /* NULL: no pattern */
    /* 0: the EX cards superpose into one right-hand side (a deck's
     * semantics).  1: every card is its own right-hand side -- solved as the
     * single-source deck it stands for -- and all of them reuse the one
     * factorisation of each frequency. */
    uint32_t separate_sources;
    /* LD cards in deck order (may be NULL): their series impedances are added
     * to Z's diagonal at every frequency before the solve */
    const fnec_load *loads;
    uint32_t n_loads;
    /* TL and NT cards in deck order (may be NULL): their two-port stamps are
     * added to Z after the loads, TL first (solve_session.rs:1290-1309) */
    const fnec_tl *tls;
    uint32_t n_tls;
    const fnec_nt *nts;
    uint32_t n_nts;
    /* NULL: the voltage sources drive the antenna.  Otherwise the antenna is
     * a receiving one (solve_session.rs:262-301, linear.rs:910-1090): each
     * incidence direction of the card is one right-hand side of the
     * frequency's factorisation, with two homogeneous columns (cos, sin) per
     * wire -- or per conductor path when some degree-2 path is non-trivial;
     * other junctioned decks are FNEC_ERR_UNSUPPORTED, as the reference
     * rejects them.  n_sources must be 0; FP64 form only. */
    const fnec_plane_wave *plane_wave;
    /* Several RP cards (main.rs:292-304 concatenates their grids): the
     * (theta, phi) degree pairs of every requested direction, in the place of
     * rp (which must then be NULL); the power integral is formed as for rp. */
    const double *rp_points;
    uint32_t n_rp_points;
} fnec_antenna;

/* Per-unit shape, for sizing result buffers.  A unit is one solve: one
 * right-hand side of one (antenna, frequency) system. */
typedef struct {
    uint32_t antenna;
    uint32_t n;        /* segments (currents)            */
    uint32_t s;        /* unknowns N + W                 */
    uint32_t n_feed;   /* feedpoint rows                 */
    uint32_t n_points; /* pattern points                 */
    double freq_hz;
    uint64_t cur_off;  /* offset (complex) into the currents array of fnec_batch_read */
    uint64_t feed_off; /* offset (rows of 7 doubles) into the feed array           */
    uint64_t pat_off;  /* offset (rows of 6 doubles) into the pattern array        */
    uint32_t rhs;      /* right-hand side index within its system                  */
    uint32_t system;   /* (antenna, frequency) system index: the factorisation     */
} fnec_unit_info;

/* Batch totals. */
typedef struct {
    uint32_t n_units;
    uint32_t max_s;
    uint64_t total_currents; /* complex entries over all units */
    uint64_t total_feeds;    /* feed rows                       */
    uint64_t total_points;   /* pattern rows                    */
    uint64_t device_bytes;   /* HBM held by the batch           */
    uint64_t h2d_bytes;      /* input bytes copied by fnec_batch_upload */
    uint64_t kernel_launches;/* launches issued by one fnec_batch_run  */
    uint32_t n_systems;      /* factorisations (antenna, frequency)     */
    /* host milliseconds of fnec_batch_create: in all; the per-antenna
     * planning (segments, topology, junctions, sources; on host threads);
     * allocation in all, and its device, pinned-host and mixed-work parts
     * (the rest: tables, packing, the first upload) */
    double create_ms, antennas_ms, alloc_ms, alloc_device_ms, alloc_pinned_ms, alloc_mixed_ms;
} fnec_batch_info;

typedef struct fnec_ctx fnec_ctx;
typedef struct fnec_batch fnec_batch;

/* ---- context ---------------------------------------------------------- */
int fnec_ctx_create(int device, fnec_ctx **out);
int fnec_ctx_destroy(fnec_ctx *ctx);
/* Last error message of this context (static storage of the context). */
const char *fnec_ctx_last_error(const fnec_ctx *ctx);
/* The context's CUDA stream (cudaStream_t), for callers that order their
 * own work against the library's. */
void *fnec_ctx_stream(fnec_ctx *ctx);

/* ---- reference nec_accel entry points ---------------------------------- */

/* fill_zmatrix_wgpu: N x N Hallen matrix, row-major, interleaved complex128
 * (2*n*n doubles).  Unlike the wgpu path the fill is FP64 and supports the
 * PEC image (ground = FNEC_GROUND_PEC). */
int fnec_fill_zmatrix(fnec_ctx *ctx, const fnec_zsegment *segments, uint64_t n, double freq_hz,
                      int32_t ground, double *z_out);

/* solve_hallen_gpu_resident: fill + normal equations + GEPP on the device.
 * rhs: 2n doubles; cos_vec: n doubles; wire_endpoints: 2w uint64 (first,
 * last); junctions: nj records.  x_out: 2(n + w') doubles, w' = max(w, 1)
 * (linear.rs:691-696 falls back to one wire when w == 0).  pivots_out
 * (optional, n + w' int32) receives the pivot row of each column. */
int fnec_solve_hallen_resident(fnec_ctx *ctx, const fnec_zsegment *segments, uint64_t n,
                               const double *rhs, const double *cos_vec,
                               const uint64_t *wire_endpoints, uint64_t w,
                               const fnec_junction *junctions, uint64_t nj, double freq_hz,
                               int32_t ground, int32_t precision, double *x_out,
                               int32_t *pivots_out);

/* nec_solver::solve_hallen (linear.rs:672-797) on a caller-supplied Z
 * (2*n*n doubles, row-major): regularised normal equations + GEPP on the
 * device.  Arguments as fnec_solve_hallen_resident. */
int fnec_solve_hallen(fnec_ctx *ctx, const double *z, uint64_t n, const double *rhs,
                      const double *cos_vec, const uint64_t *wire_endpoints, uint64_t w,
                      const fnec_junction *junctions, uint64_t nj, int32_t precision,
                      double *x_out, int32_t *pivots_out);

/* run_rp_farfield_batch_wgpu: pattern at explicit (theta, phi) points with
 * a caller-supplied normalisation total_radiated (currents: 2n doubles,
 * points: 2p doubles in degrees). */
int fnec_rp_farfield_batch(fnec_ctx *ctx, const fnec_gpu_segment *segments, uint64_t n,
                           const double *currents, double k, double total_radiated,
                           const double *points, uint64_t p, fnec_rp_result *out);

/* compute_radiation_pattern: the power integral is formed on the device.
 * out: 4 doubles per point (gain_total, gain_theta, gain_phi, axial ratio);
 * total_out (optional) receives the integral. */
int fnec_radiation_pattern(fnec_ctx *ctx, const fnec_gpu_segment *segments, uint64_t n,
                           const double *currents, double freq_hz, int32_t ground,
                           const double *points, uint64_t p, double *out, double *total_out);

/* integrate_radiated_power (pec_ground != 0: 91 x 360 upper hemisphere). */
int fnec_integrate_radiated_power(fnec_ctx *ctx, const fnec_gpu_segment *segments, uint64_t n,
                                  const double *currents, double freq_hz, int32_t pec_ground,
                                  double *out);

/* ---- decks and reports ------------------------------------------------ *
 * The deck reader (nec_parser::parse, crates/nec_parser/src/lib.rs:78-418)
 * and the report contract v1 writer (nec_report::render_text_report,
 * crates/nec_report/src/lib.rs:307-484) around the batch interface: a deck's
 * text in, the CLI's text report for every FR frequency out. */
typedef struct fnec_deck fnec_deck;
typedef struct {
    uint32_t n_wires, n_sources, n_ex, n_loads, n_tls, n_nts, n_freqs, n_rp_cards, n_points, n_ne_cards;
    int32_t ground;      /* FNEC_GROUND_FREE / FNEC_GROUND_PEC as the deck's GN / GE cards select */
    uint32_t plane_wave; /* the deck's first plane-wave EX card drives it */
    uint32_t warnings;   /* unknown cards skipped by the parser */
    uint32_t runnable;   /* 0: the device path does not build this deck (why says what) */
    char why[200];       /* the reason, or the first parser warning */
} fnec_deck_info;
/* Parse a deck.  A bad or missing field is fatal (FNEC_ERR_BAD_ARG; err
 * receives "line N: ..."); unknown cards are counted and skipped.  Grids
 * beyond the maxima below are refused with FNEC_ERR_TOO_LARGE (err says
 * which card); host memory exhaustion gives FNEC_ERR_OUT_OF_MEMORY. */
#define FNEC_DECK_MAX_FREQS (1u << 20)  /* FR steps                          */
#define FNEC_DECK_MAX_POINTS (1u << 22) /* RP points over all RP cards; NE/NH */
int fnec_deck_parse(const char *text, fnec_deck **out, char *err, uint64_t err_cap);
int fnec_deck_destroy(fnec_deck *d);
int fnec_deck_get_info(const fnec_deck *d, fnec_deck_info *out);
/* The deck as one fnec_antenna (pointers into the deck, valid while it
 * lives); freqs (optional, n_freqs doubles) receives the FR frequencies. */
int fnec_deck_get_antenna(const fnec_deck *d, fnec_antenna *out, double *freqs);
/* Solve every FR frequency in one batch and render the report of each
 * (FEEDPOINTS, SOURCES, LOADS, CURRENTS with the last PT card's filter,
 * RADIATION_PATTERN, RECEIVE_PATTERN, NEAR_FIELD, NEAR_H_FIELD,
 * NORMALIZED_PATTERN, AVERAGE_POWER_GAIN), separated by blank lines as the
 * CLI prints them.  *report is owned by the deck (until the next solve or
 * destroy).  FNEC_ERR_UNSUPPORTED for decks the device path does not build,
 * FNEC_ERR_SINGULAR when a solve fails. */
int fnec_deck_solve(fnec_ctx *ctx, fnec_deck *d, int32_t precision, const char **report, uint64_t *len);

/* sizeof of the public structs, in this order, for bindings to check their
 * layouts against: fnec_wire, fnec_source, fnec_rp_card, fnec_plane_wave,
 * fnec_load, fnec_tl, fnec_nt, fnec_antenna, fnec_unit_info,
 * fnec_batch_info, fnec_deck_info, fnec_server_config, fnec_request_out,
 * fnec_request_info, fnec_request_result, fnec_server_stats_t,
 * fnec_schedule, fnec_tune_report, fnec_zsegment, fnec_gpu_segment,
 * fnec_rp_result, fnec_junction.  Returns how many there are; writes at
 * most cap. */
uint32_t fnec_abi_struct_sizes(uint64_t *out, uint32_t cap);

/* build_geometry (geometry.rs:676-754): the segments of GW cards in card
 * order, on the host, as the device expands them.  out may be NULL (count
 * only); *n_out receives the segment count; cap < count writes nothing. */
int fnec_build_geometry(const fnec_wire *wires, uint32_t n_wires, fnec_zsegment *out, uint64_t cap,
                        uint64_t *n_out);

/* near_e_field / near_h_field: the near electric and magnetic fields at p
 * points (3p doubles, metres) as the sum over the n segments of Hertzian
 * elements I_n L_n at their midpoints, free space, segments within 1e-9 m of
 * a point skipped.  currents: 2n doubles.  e_out / h_out: 6p doubles each
 * (Ex, Ey, Ez complex), either may be null but not both. */
int fnec_near_field(fnec_ctx *ctx, const fnec_gpu_segment *segments, uint64_t n, const double *currents,
                    double freq_hz, const double *points, uint64_t p, double *e_out, double *h_out);

/* microbench_zmatrix_dispatch: device-init vs dispatch split (microseconds). */
int fnec_microbench_zmatrix_dispatch(int device, uint64_t n_segments, uint32_t n_dispatches,
                                     uint64_t *device_init_us, uint64_t *dispatch_min_us,
                                     uint64_t *dispatch_median_us);

/* enumerate_compute_adapters: number of CUDA devices and, for index `i`,
 * its name into `name` (NUL-terminated, at most `cap` bytes). */
int fnec_enumerate_devices(int *count, int index, char *name, uint64_t cap);

/* dispatch_frequency_point: 1 = RunOnGpu (a device is present), 0 = none. */
int fnec_dispatch_frequency_point(int request_kind, double freq_hz);

/* FP64 pipe peaks of this GPU (no counterpart in the reference): fused
 * DFMA and separately rounded DMUL+DADD throughput in TFLOP/s, used as the
 * roofline denominators of the FP64-bound kernels. */
int fnec_measure_fp64_peak(int device, double *fma_tflops, double *muladd_tflops);
/* FP32 FFMA throughput in TFLOP/s (no counterpart in the reference): the
 * roofline denominator of the mixed form's FP32 factorisation. */
int fnec_measure_fp32_peak(int device, double *ffma_tflops);

/* ---- serving: continuous batching of solve requests -------------------
 * No counterpart in the reference (its sweep loop calls the backend once
 * per frequency).  A server owns `lanes` CUDA streams and a host thread:
 * submitted requests (one fnec_antenna deck each; every voltage source a
 * separate right-hand side when separate_sources is set) queue in arrival
 * order; whenever a lane (each driven by its own host thread) is free it
 * admits queued requests while the device bytes of the batches in flight
 * (each request's admission estimate, fnec_request_info.device_bytes) stay
 * within hbm_budget_bytes, solves them as one batch -- Z and its factor stay
 * on the device for all of a request's right-hand sides and its pattern --
 * and delivers the results: copied into the request's output arrays when it
 * gave some, else readable in place in the server's page-locked memory
 * (fnec_server_result) until fnec_server_release.  Requests arriving while
 * batches run are admitted as lanes and memory free up; the lanes' planning,
 * kernels and copies overlap.  With more than one lane the grid-wide
 * (cooperative) kernels are not used.  At creation the server maps its HBM
 * budget (at most the device's free memory less 2 GiB) into the device's
 * stream-ordered pool, so that admission under load suballocates instead of
 * waiting for the driver to map memory. */
typedef struct fnec_server fnec_server;

typedef struct {
    int32_t precision;         /* FNEC_PRECISION_FP64 or FNEC_PRECISION_MIXED */
    int32_t lanes;             /* concurrent batches (streams), 1..16        */
    uint64_t hbm_budget_bytes; /* device bytes the batches in flight may use */
    uint32_t max_batch;        /* requests per batch                          */
    uint32_t queue_cap;        /* queued requests before submit is BUSY (0: 2^20) */
} fnec_server_config;

/* Output arrays of one request, caller-owned, written before the request
 * reports DONE (any may be NULL).  Solve k = frequency * n_rhs + rhs. */
typedef struct {
    double *currents; /* n_solves x n_segments complex (interleaved)         */
    double *feeds;    /* n_feed_rows x 7 (as fnec_batch_read), solve order    */
    double *pattern;  /* n_solves x n_points x 6 (as fnec_batch_read)         */
    int32_t *status;  /* n_solves: 0, -(column+1) singular, or an error code  */
} fnec_request_out;

typedef struct {
    uint32_t n_segments;
    uint32_t n_rhs;
    uint32_t n_solves;
    uint32_t n_feed_rows;
    uint32_t n_points;
    uint32_t pad;
    uint64_t device_bytes; /* admission estimate (upper bound) of the footprint */
} fnec_request_info;

typedef struct {
    uint64_t submitted, completed, failed;
    uint64_t solves;          /* right-hand sides of completed requests */
    uint64_t batches;
    uint64_t queued;
    uint64_t in_flight_bytes, peak_in_flight_bytes;
    uint64_t max_batch;       /* largest batch formed                      */
    uint64_t kernel_launches; /* kernels launched for the completed batches */
    uint64_t h2d_bytes, d2h_bytes; /* host <-> device bytes of those batches */
    double plan_ms, launch_ms, collect_ms; /* the lanes' host time: batch planning,
                                              enqueueing, result delivery */
    double alloc_ms;                       /* of plan_ms: allocations          */
    double alloc_device_ms, alloc_upload_ms, alloc_pinned_ms, alloc_mixed_ms; /* its parts */
    double p50_ms, p99_ms, mean_ms, max_ms; /* submit -> results delivered */
} fnec_server_stats_t;

#define FNEC_REQ_QUEUED 0
#define FNEC_REQ_RUNNING 1
#define FNEC_REQ_DONE 2

int fnec_server_create(fnec_ctx *ctx, const fnec_server_config *cfg, fnec_server **out);
/* Finishes every queued and running request, then releases the server. */
int fnec_server_destroy(fnec_server *s);
/* Output sizes and admission footprint of a request (host planning only). */
int fnec_request_shape(fnec_ctx *ctx, const fnec_antenna *req, int32_t precision, fnec_request_info *out);
/* Queue a request; BUSY when the queue is full, TOO_LARGE when it alone
 * exceeds the budget.  The deck is copied.  out (may be NULL): output
 * arrays, which must stay valid until the request is done.  info (may be
 * NULL) receives the request's shape. */
int fnec_server_submit(fnec_server *s, const fnec_antenna *req, const fnec_request_out *out, uint64_t *ticket,
                       fnec_request_info *info);
/* state: FNEC_REQ_* or a negative error. */
int fnec_server_poll(fnec_server *s, uint64_t ticket, int32_t *state, double *latency_ms);
int fnec_server_wait(fnec_server *s, uint64_t ticket, double timeout_ms, int32_t *state, double *latency_ms);

/* The next finished request (done or failed) in completion order; each
 * finished request not yet released is reported once here, whatever
 * poll/wait also saw. */
int fnec_server_next_done(fnec_server *s, double timeout_ms, uint64_t *ticket);

/* A finished request's results, in place in the server's page-locked
 * memory (NULL arrays when it was submitted with output arrays, or failed);
 * valid until fnec_server_release.  Solve k's currents start at
 * currents + 2 * k * cur_stride doubles (n_segments complex values). */
typedef struct {
    const double *currents;
    uint64_t cur_stride;
    const double *feeds;   /* n_feed_rows x 7  */
    const double *pattern; /* n_solves x n_points x 6 */
    const int32_t *status; /* n_solves         */
    uint32_t n_solves, n_segments, n_feed_rows, n_points;
} fnec_request_result;
int fnec_server_result(fnec_server *s, uint64_t ticket, fnec_request_result *out);
/* Forget a finished request (BUSY while it runs); its in-place results go.
 * Requests read in place hold their batch's result slab: a server keeps at
 * most lanes + 4 slabs (allocated up front), so lanes wait for releases when
 * all are held. */
int fnec_server_release(fnec_server *s, uint64_t ticket);
/* The server's most recent failure (valid until the next call). */
const char *fnec_server_last_error(fnec_server *s);
/* Latency percentiles over completed requests since the last reset. */
int fnec_server_stats(fnec_server *s, fnec_server_stats_t *out, int32_t reset);

/* Page-locked host memory (no counterpart in the reference).  Result arrays
 * passed to fnec_batch_read in such memory are written by direct device
 * copies, without the staging copy pageable memory needs.  Freed blocks
 * (these and the batches' input / result arenas) are kept for reuse, up to
 * 1 GiB in all: pinning pages is the slowest part of planning a batch.
 * fnec_host_cache_release frees the kept blocks (*released: their bytes). */
int fnec_host_alloc(uint64_t bytes, void **out);
int fnec_host_free(void *p);
int fnec_host_cache_release(uint64_t *released);

/* Device memory of batches comes from the device's stream-ordered pool, which
 * keeps what a destroyed batch frees for the next batch (mapping and
 * unmapping a large batch's memory costs tens of milliseconds).
 * fnec_device_cache_release waits for the context's stream and returns the
 * pool's unused memory to the driver (*released: its bytes), e.g. before
 * another library on the device allocates. */
int fnec_device_cache_release(fnec_ctx *ctx, uint64_t *released);

/* Self-test of the 3xTF32 tensor-core GEMM that forms the mixed form's
 * Gram matrix (no counterpart in the reference): C = A B^T with A (m x k),
 * B (n x k) and C (m x n) row-major FP32 host arrays.  m, n, k <= 65536. */
int fnec_selftest_tf32x3_gemm(int32_t device, uint64_t m, uint64_t n, uint64_t k, const float *a,
                              const float *b, float *c);

/* Self-tests of the failure paths (no counterpart in the reference; test
 * use).  fnec_selftest_wait_timeout makes one bounded device wait run out
 * on purpose and reports the status word the kernel left:
 *   which 0  a cooperative launch of 8 CTAs whose CTA 3 never reaches the
 *            grid barrier: the others give up after wait_ns and mark
 *            FNEC_UNIT_TIMEOUT;
 *   which 1  the same launch with every CTA arriving: status 0;
 *   which 2  the tcgen05 GEMM with its loads stopped after 2 of 8 k-blocks:
 *            the MMA warp's wait runs out, the CTA drains its copies and
 *            MMAs, frees TMEM and marks FNEC_UNIT_TIMEOUT.
 * wait_ns is 1 .. 2e9.  Returns FNEC_OK when the kernel ran to its end;
 * *elapsed_ms is the launch's duration.  The context stays usable.
 * fnec_test_fail_device_allocation(n): the n-th batch device allocation
 * from now on fails as if the device were full (once); -1 disarms. */
int fnec_selftest_wait_timeout(int32_t device, int32_t which, uint64_t wait_ns, int32_t *unit_status,
                               double *elapsed_ms);
int fnec_test_fail_device_allocation(int32_t after);
/* The mixed form's fill evaluates its samples' phase with its own
 * sin(pi x), cos(pi x) (quadrant reduction, Taylor series; the same source
 * is compiled for the host): fnec_test_fill_sincospi runs it on the host
 * for n arguments 0 <= x < 2^50 (test use). */
int fnec_test_fill_sincospi(const double *x, uint64_t n, double *sin_out, double *cos_out);
/* The fill's reciprocal square root (a single-precision guess and two
 * Newton steps), run on the current device for n <= 2^20 normal, finite,
 * positive arguments (test use; allocates its own device memory). */
int fnec_test_fill_rsqrt(const double *x, uint64_t n, double *out);

/* Radiation pattern that allocates no device memory.  No counterpart in
 * the reference: it serves callers that cannot call cudaMalloc -- a host
 * framework that owns all device memory through its own pool, a plugin held
 * to a fixed memory budget, or a real-time loop that cannot take the
 * implicit synchronisation of cudaMalloc/cudaFree.
 * Same computation as fnec_radiation_pattern (compute_radiation_pattern
 * semantics, power integral on the device), but every pointer is a DEVICE
 * pointer owned by the caller: d_segments (n records), d_currents (2n
 * doubles), d_points (2p doubles, degrees), d_out (4p doubles: gain_total,
 * gain_theta, gain_phi, axial_ratio) and d_total (1 double, optional).  The
 * work is enqueued on `stream` (a cudaStream_t; NULL = legacy default) of
 * the current device; the caller synchronises.
 * Scratch lives in a fixed static device array of about 5.6 MB held by
 * every GPU that loads the library until exit.  With CUDA's lazy module
 * loading the array (and the kernels) are committed on a device at the
 * first call there, which also looks the array's address up
 * (cudaGetSymbolAddress): make that first call before the host framework
 * reserves its memory pool and before any stream capture.  Calls that
 * overlap on the GPU (other streams, other threads) race on the shared
 * scratch and must be serialised.  A CUDA error already pending on the
 * calling thread is returned as FNEC_ERR_CUDA (and left pending) with
 * nothing launched.
 * Limits: n <= FNEC_NOALLOC_MAX_SEGMENTS, p <= FNEC_NOALLOC_MAX_POINTS;
 * larger sizes return FNEC_ERR_TOO_LARGE without touching the device. */
#define FNEC_NOALLOC_MAX_SEGMENTS 4096
#define FNEC_NOALLOC_MAX_POINTS 65536
int fnec_radiation_pattern_noalloc(const fnec_gpu_segment *d_segments, uint64_t n,
                                   const double *d_currents, double freq_hz, int32_t ground,
                                   const double *d_points, uint64_t p, double *d_out,
                                   double *d_total, void *stream);

/* ---- batched, device-resident interface ------------------------------- */

/* Plan a batch: host-side topology (endpoints, collinear merge, junctions,
 * constraint rows, resolved sources, wire runs), device allocation and a
 * first upload.  Units are ordered antenna-major, frequency-minor. */
int fnec_batch_create(fnec_ctx *ctx, const fnec_antenna *antennas, uint32_t n_antennas,
                      int32_t precision, fnec_batch **out);
int fnec_batch_destroy(fnec_batch *b);
int fnec_batch_get_info(const fnec_batch *b, fnec_batch_info *out);
int fnec_batch_get_unit_info(const fnec_batch *b, uint32_t unit, fnec_unit_info *out);
/* Re-copy the batch's host inputs (wires, tables, frequencies) to the
 * device (the host->device half of an end-to-end step). */
int fnec_batch_upload(fnec_batch *b);
/* Enqueue the whole pipeline on the context stream: segment expansion,
 * Hallen RHS, Z fill, Gram, factorisation, solve, feedpoints, pattern. */
int fnec_batch_run(fnec_batch *b);
/* Wait for the batch (and report per-unit failures as the first error). */
int fnec_batch_sync(fnec_batch *b);
/* Copy results to host arrays (any may be NULL):
 *   currents: 2 * total_currents doubles (unit blocks at cur_off)
 *   feeds:    7 * total_feeds doubles (seg, V re/im, I re/im, Zin re/im)
 *   pattern:  6 * total_points doubles (gain_total, gain_theta, gain_phi,
 *             axial_ratio, u_theta, u_phi)
 *   status:   n_units int32 (0, -(column+1) of a singular pivot, or
 *             FNEC_UNIT_TIMEOUT)
 *   total_radiated: n_units doubles */
int fnec_batch_read(fnec_batch *b, double *currents, double *feeds, double *pattern,
                    int32_t *status, double *total_radiated);
/* Record CUDA events around each pipeline phase of later runs (on != 0). */
int fnec_batch_set_profiling(fnec_batch *b, int on);
/* Milliseconds of each phase of the last profiled run (FNEC_N_PHASES
 * doubles); waits for that run to finish. */
int fnec_batch_phase_ms(fnec_batch *b, double *ms);

/* Per-unit solution vector x (currents then homogeneous constants), 2*s
 * doubles, and the pivot rows (s int32), for parity checks. */
int fnec_batch_read_unit(fnec_batch *b, uint32_t unit, double *x, int32_t *pivots);
/* The report's results only (what render_text_report prints): currents,
 * feeds and status as fnec_batch_read; pattern4 receives 4 doubles per point
 * (gain_total, gain_theta, gain_phi, axial_ratio), packed on the device, so
 * the copy is two thirds of the 6-column rows.  pattern4 must be page-locked
 * (fnec_host_alloc). */
int fnec_batch_read_report(fnec_batch *b, double *currents, double *feeds, double *pattern4, int32_t *status);
/* Run the batch with the report's pattern columns streamed out: the far
 * field runs in chunks of solves and each chunk's 4 columns are copied to
 * pattern4 (page-locked, 4 doubles per point) while the next chunk
 * computes.  Launched eagerly (not from the batch's graph).  Follow with
 * fnec_batch_read_report(b, currents, feeds, NULL, status), which waits for
 * the copies too. */
int fnec_batch_run_report(fnec_batch *b, double *pattern4);
/* Receive pattern of plane-wave units (solve_session.rs:313-375
 * plane_wave_receive_sweep): 3 doubles per unit -- theta, phi (degrees)
 * and 20 log10(peak |I| / the largest peak of the unit's system) dB,
 * -999.99 for a zero peak; units without a plane wave get NaNs.  The peak
 * is formed on the device. */
int fnec_batch_read_receive(fnec_batch *b, double *out);
/* Mixed-precision batches: per-unit GMRES iterations (n_units int32) and
 * final preconditioned relative residual (n_units doubles) of the last run. */
int fnec_batch_read_refinement(fnec_batch *b, int32_t *iters, double *resid);
/* Z matrix (2*n*n doubles) and the augmented normal-equation matrix before
 * elimination is not kept; the Z of a unit can be read after a run. */
int fnec_batch_read_z(fnec_batch *b, uint32_t unit, double *z);
/* Resident systems (no counterpart in the reference, whose accelerator
 * keeps no device state between calls): after a run, a batch keeps every
 * system's Z and factorisation on the device.  fnec_batch_set_sources
 * replaces the voltage sources of one antenna (resolved against its
 * segments as at planning); every right-hand side must keep its planned
 * numbers of resolved sources and feed rows.  fnec_batch_resolve then
 * solves every unit again on the stored factorisations -- right-hand
 * sides, substitution (plain: bit-identical to a fresh batch with those
 * sources) or refinement (mixed), feedpoints and pattern -- without the
 * fill, the normal equations or the factorisation.  Results are read as
 * after fnec_batch_run. */
int fnec_batch_set_sources(fnec_batch *b, uint32_t antenna, const fnec_source *sources, uint32_t n_sources);
int fnec_batch_resolve(fnec_batch *b);

/* ---- schedules, CUDA graphs and the autotuner --------------------------
 *
 * How a batch's pipeline is launched.  None of these choices changes a
 * result bit of the plain FP64 form (its per-unit arithmetic is the same
 * under every schedule); the mixed form stays within its refinement
 * tolerance under every schedule. */
typedef struct {
    int32_t grid_panels;   /* 1: panels too tall for one CTA's shared memory are
                              factored grid-wide (cooperative launch); 0: one CTA
                              from global memory                                  */
    int32_t class_shift;   /* panel and trailing launches group units whose
                              remaining heights share a 2^class_shift size class
                              (1 or 2)                                            */
    int32_t gram_tensor;   /* mixed: 1 Gram Z^H Z as 3xTF32 tcgen05 tiles; 0 FP32
                              SIMT tiles                                          */
    int32_t gmres_cluster; /* mixed: CTAs per refinement solve (1, 2, 4 or 8; a
                              thread-block cluster when > 1)                      */
    int32_t grid_gmres;    /* mixed: 1 very large solves refine grid-wide        */
    int32_t graph;         /* 0 launch eagerly; 1 capture the pipeline as a CUDA
                              graph at the second run and replay it afterwards;
                              2 capture at the first run                          */
    int32_t factor_streams;/* mixed: the factor's units in 1, 2 or 4 groups of
                              about equal work, each on its own stream (parallel
                              branches of the graph)                              */
    int32_t unit_factor;   /* mixed: units with S <= 256 (1), 384 (2) or 512 (3)
                              are factored whole, one CTA each, in one launch
                              beside the per-step launches of the larger units;
                              0 none                                              */
    int32_t block_inverse; /* mixed: 1 the refinement applies the factor's 32x32
                              diagonal blocks through their FP64 inverses (block
                              products); 0 by substitution in one warp            */
    int32_t tensor_trailing;/* mixed: 1 trailing updates of >= 192 rows run on
                              tcgen05 (3xTF32, complex as one real GEMM of K 64;
                              for the Hermitian factor only the tiles on and
                              below the diagonal); 0 all as FP32 SIMT tiles, one
                              pass per step; 2 (GEPP only) SIMT tiles once per
                              two steps (the first step updates only the next
                              panel's columns)                                   */
    int32_t gmres_ctas_per_sm;/* mixed: 3 or 4 refinement CTAs per SM (the
                              register budget of the one-CTA-per-solve kernel)    */
    int32_t factor_pivoting;/* mixed: 0 the FP32 factor of the Hermitian normal
                              equations without row exchanges (lower-triangle
                              trailing updates, U12 mirrored from L21); 1 GEPP
                              with partial pivoting (row exchanges and U12
                              solves; tensor_trailing 2 applies to it only)     */
} fnec_schedule;

/* Graph state of a batch (fnec_batch_graph_state). */
#define FNEC_GRAPH_NONE 0     /* not captured (eager launches)                 */
#define FNEC_GRAPH_READY 1    /* runs replay the captured graph                */
#define FNEC_GRAPH_FAILED (-1)/* capture was refused; runs launch eagerly      */

typedef struct {
    fnec_schedule best;     /* the schedule set on the batch                  */
    double default_ms;      /* device ms of one run under the starting schedule */
    double best_ms;         /* ... under the chosen one                       */
    uint32_t candidates;    /* schedules timed                                 */
    uint32_t from_cache;    /* 1: the batch's shape was already in the cache   */
    char key[96];           /* shape key of the tuning cache                   */
} fnec_tune_report;

int fnec_batch_get_schedule(const fnec_batch *b, fnec_schedule *out);
/* Change the schedule (validated: FNEC_ERR_BAD_ARG for values out of range;
 * cluster sizes above what the batch planned for are lowered); drops a
 * captured graph. */
int fnec_batch_set_schedule(fnec_batch *b, const fnec_schedule *s);
/* state: FNEC_GRAPH_*; nodes: kernel launches one replay issues. */
int fnec_batch_graph_state(const fnec_batch *b, int32_t *state, uint64_t *nodes);
/* Time the batch under candidate schedules (coordinate descent over the
 * fields above, two passes; reps timed runs each after one warm-up, median device time
 * on the batch stream), set the fastest and record it in the process-wide
 * tuning cache under the batch's shape key.  Batches created later with
 * the same key start from the cached schedule.  With reps == 0 the cached
 * schedule is applied if present and nothing is timed. */
int fnec_batch_tune(fnec_batch *b, uint32_t reps, fnec_tune_report *out);
/* The tuning cache as a text file: one "key field=value ..." line per
 * shape.  load merges (later lines win); clear empties the cache. */
int fnec_tune_cache_save(const char *path);
int fnec_tune_cache_load(const char *path);
int fnec_tune_cache_clear(void);
/* Number of cached shapes. */
int fnec_tune_cache_size(uint32_t *n);

#ifdef __cplusplus
}
#endif
#endif

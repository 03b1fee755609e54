/*
 * fnec_oracle.h -- CPU oracle for the Hallen method-of-moments hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference
 * CPU path of dc0sk/fnec-rust (crates/nec_solver, apps/nec-cli) used as the
 * checker for the CUDA library.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / reference arm of bench.py may load it; the product library
 * (libfnec_cuda.so) never links or calls it.
 *
 * Faithfulness rules: every function follows the cited reference function
 * operation by operation, compiled with -O2 -ffp-contract=off (no FMA
 * contraction, like rustc), against glibc libm (the libm Rust's f64::sin,
 * cos, sqrt, ln, hypot, log10, asin and tan call on linux-gnu).  Complex
 * arithmetic follows num-complex 0.4.6 (the version pinned in the
 * reference's Cargo.lock): mul (ac-bd, ad+bc); div ((ac+bd)/|w|^2,
 * (bc-ad)/|w|^2); norm = hypot; exp(0+jt) = (cos t, sin t).
 *
 * Parity pin: the golden values of corpus/reference-results.json (feedpoint
 * impedances to 6 decimals, current samples, pattern samples to 4 decimals)
 * are checked by tests/test_oracle_golden.py against this oracle.
 */
#ifndef FNEC_ORACLE_H
#define FNEC_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* One wire segment; mirrors nec_solver::geometry::Segment (geometry.rs:115-134). */
typedef struct {
    uint32_t tag;
    uint32_t tag_index;   /* 1-based index within the tag */
    double start[3];
    double end[3];
    double mid[3];
    double dir[3];
    double length;
    double radius;
} or_seg;

/* One GW card (geometry.rs:710-754 consumes these fields). */
typedef struct {
    uint32_t tag;
    uint32_t segments;
    double start[3];
    double end[3];
    double radius;
} or_wire;

/* One voltage-source EX card (types 0/5), in deck order. */
typedef struct {
    uint32_t tag;
    uint32_t segment;
    double v_re;
    double v_im;
} or_source;

enum { OR_GROUND_FREE = 0, OR_GROUND_PEC = 1 };
enum {
    OR_OK = 0,
    OR_ERR_SINGULAR = -1,
    OR_ERR_ZERO_SEGMENTS = -2,
    OR_ERR_ZERO_LENGTH = -3,
    OR_ERR_NO_WIRES = -4,
    OR_ERR_SEGMENT_NOT_FOUND = -5,
    OR_ERR_CAPACITY = -6,
    OR_ERR_DIM = -7,
    OR_ERR_JUNCTION = -8 /* planewave.rs:131-133 JunctionedGeometryNotSupported */
};

/* geometry.rs:676-754 (GW only). Returns N, or a negative error. */
int64_t or_build_geometry(const or_wire *wires, int64_t nw, or_seg *out, int64_t cap);
/* geometry.rs:168-185. out holds 2*cap int64 (first,last). Returns count. */
int64_t or_wire_endpoints(const or_seg *segs, int64_t n, int64_t *out, int64_t cap);
/* geometry.rs:200-225. */
int64_t or_merge_collinear(const or_seg *segs, int64_t n, int64_t *out, int64_t cap);
/* geometry.rs:274-339. Returns the number of junctions (may exceed cap:
 * only the first cap are written). */
int64_t or_detect_junctions(const or_seg *segs, const int64_t *ep, int64_t w, double tol,
                            int64_t *ja, int64_t *jb, double *jsign, int64_t cap);
/* solve_session.rs:1386-1400: merged endpoints + cross-component junctions. */
int64_t or_cli_junctions(const or_seg *segs, int64_t n, const int64_t *merged, int64_t w,
                         int64_t *ja, int64_t *jb, double *jsign, int64_t cap);
/* excitation.rs:119-244.  rhs: 2n doubles (re,im); cosv: n doubles. */
int or_hallen_rhs(const or_seg *segs, int64_t n, double freq_hz, const or_source *src,
                  int64_t ns, double *rhs, double *cosv);
/* excitation.rs:78-90 / :450-482 (V/dl per segment).  v: 2n doubles. */
int or_excitation(const or_seg *segs, int64_t n, const or_source *src, int64_t ns, double *v);
/* matrix.rs:186-218.  z: 2*n*n doubles, row-major, interleaved re/im. */
void or_assemble_z(const or_seg *segs, int64_t n, double freq_hz, int ground, double *z);
/* One element: matrix.rs:297-331 (elem) + image (:265-279) when ground=PEC. */
void or_z_element(const or_seg *obs, const or_seg *src, double freq_hz, int ground,
                  int is_self, double *out2);
/* linear.rs:672-797 + :1321-1383.  x: 2*(n+w) doubles.  pivots (optional):
 * n+w int32 pivot rows.  gram (optional): 2*S*(S+1) doubles, the augmented
 * [A|b] before elimination.  naive != 0 runs the literal dense triple loop
 * over M; naive == 0 skips structural zeros (value-identical, see .c). */
/* geometry.rs:404-584 build_conductor_paths.  Per segment: path index,
 * traversal sign, signed arc length from the path centre; free_ends: 2 per
 * path (capacity 2n).  Returns the path count, -1 for None (degree >= 3,
 * closed loop).  *nontrivial: some path is reversed or non-contiguous. */
int64_t or_conductor_paths(const or_seg *segs, int64_t n, int64_t *path_of, double *sign,
                           double *s_mid, int64_t *free_ends, int *nontrivial);
/* excitation.rs:264-341 build_hallen_rhs_paths. */
int or_hallen_rhs_paths(const or_seg *segs, int64_t n, double freq_hz, const or_source *src,
                        int64_t ns, const int64_t *path_of, const double *sign, const double *s_mid,
                        double *rhs, double *cosv);
/* linear.rs:823-894 solve_hallen_paths; x holds n + paths complex values. */
int or_solve_hallen_paths(const double *z, int64_t n, const double *rhs, const double *cosv,
                          const int64_t *path_of, const int64_t *free_ends, int64_t n_free, double *x,
                          int32_t *pivots, double *gram, int naive, int nthreads);
int or_solve_hallen(const double *z, int64_t n, const double *rhs, const double *cosv,
                    const int64_t *ep, int64_t w, const int64_t *ja, const int64_t *jb,
                    const double *jsign, int64_t nj, double *x, int32_t *pivots,
                    double *gram, int naive, int nthreads);
/* linear.rs:1321-1383 on a dense S x S matrix a (2*S*S) and b (2*S).
 * a and b are overwritten.  x: 2*S.  pivots optional. */
int or_solve_square(double *a, double *b, int64_t s, double *x, int32_t *pivots, int nthreads);
/* solve_session.rs:846-947 (voltage sources only): per EX card with a
 * matching segment, (seg index, V, I, Zin).  out: 7 doubles per row
 * (idx, v_re, v_im, i_re, i_im, z_re, z_im).  Returns row count. */
int64_t or_feedpoints(const or_seg *segs, int64_t n, const or_source *src, int64_t ns,
                      const double *cur, double *out, int64_t cap);
/* farfield.rs:422-464 (PEC or free). */
double or_integrate_power(const or_seg *segs, int64_t n, const double *cur, double freq_hz,
                          int ground);
/* farfield.rs:563-647.  pts: 2p (theta,phi deg).  out: 4 doubles per point
 * (gain_total, gain_theta, gain_phi, axial_ratio).  total_out optional.
 * uf_out optional: 4 doubles per point (F_theta re,im, F_phi re,im). */
void or_radiation_pattern(const or_seg *segs, int64_t n, const double *cur, double freq_hz,
                          int ground, const double *pts, int64_t p, double *out,
                          double *total_out, double *uf_out);
/* farfield.rs:677-699. pts: 2*max(nt,1)*max(np,1). Returns count. */
int64_t or_rp_card_points(uint32_t n_theta, uint32_t n_phi, double theta0, double phi0,
                          double d_theta, double d_phi, double *pts);

/* One LD card (nec_model card.rs:265-279): load type 0-5, tag (0 = every
 * tag), first and last segment (0 = every segment of the tag; last 0 =
 * first), F1..F3. */
typedef struct {
    int32_t load_type;
    uint32_t tag;
    uint32_t seg_first;
    uint32_t seg_last;
    double f1, f2, f3;
} or_load;

/* loads.rs:103-222 build_loads: the series load impedance of every segment
 * (2*n doubles) summed over the cards in deck order.  Returns the number of
 * cards (or card/segment pairs for type 5 with sigma <= 0) ignored with a
 * warning by the reference. */
int64_t or_build_loads(const or_seg *segs, int64_t n, double freq_hz, const or_load *ld, int64_t nl,
                       double *out);

/* One TL card (card.rs TlCard; tl.rs:47-183): ends (tag, segment; segment 0
 * = the tag's centre segment), sections, type (0 lossless; else lossy with
 * F3 the matched-line loss in dB), Z0, length, F3 (velocity factor of a
 * lossless line; parsed default 1). */
typedef struct {
    uint32_t tag1, seg1, tag2, seg2, num_segments, tl_type;
    double z0, length, f3;
} or_tl;
/* One NT card with its 10 fields parsed (network.rs:55-142): ends and the
 * reciprocal two-port's short-circuit admittances Y11, Y12 (= Y21), Y22. */
typedef struct {
    uint32_t tag1, seg1, tag2, seg2;
    double y11r, y11i, y12r, y12i, y22r, y22i;
} or_nt;
/* tl.rs:47-183 build_tl_stamps / network.rs:55-142 build_nt_stamps: the
 * (row, col, delta) stamps in order (4 per applied card; cap entries).
 * Returns the stamp count. */
int64_t or_tl_stamps(const or_seg *segs, int64_t n, double freq_hz, const or_tl *tl, int64_t ntl, int64_t *rows,
                     int64_t *cols, double *vals, int64_t cap);
int64_t or_nt_stamps(const or_seg *segs, int64_t n, const or_nt *nt, int64_t nnt, int64_t *rows, int64_t *cols,
                     double *vals, int64_t cap);

/* farfield.rs:154-261 near_e_field / near_h_field: the Hertzian-element sum
 * of the segment currents (2n doubles) at p points (3p doubles, metres);
 * e_out / h_out (6p doubles: x, y, z complex components) may be NULL. */
void or_near_field(const or_seg *segs, int64_t n, const double *cur, double freq_hz, const double *pts, int64_t p,
                   double *e_out, double *h_out);
/* solve_session.rs:645-688 near_field_grid_points of one NE/NH card
 * (coord_type 0 rectangular x/y/z, else spherical R/phi/theta); returns the
 * point count, writes 3 doubles per point when pts != NULL. */
int64_t or_near_field_points(uint32_t coord_type, uint32_t nx, uint32_t ny, uint32_t nz, double x0, double y0,
                             double z0, double dx, double dy, double dz, double *pts);

/* An incident plane wave (planewave.rs:37-105, EX types 1/2/3): it arrives
 * from (theta, phi) degrees with polarisation angle eta; types 2 / 3 are
 * right / left elliptic with the given axial ratio, type 1 linear. */
typedef struct {
    int32_t ex_type;
    double theta_deg, phi_deg, eta_deg, axial_ratio;
} or_wave;

/* planewave.rs:162-254 build_planewave_hallen (path_of == NULL: per-tag
 * wires; returns OR_ERR_JUNCTION when any two wire ends touch) and
 * :278-348 build_planewave_hallen_paths (path_of, sign, s_mid from
 * or_conductor_paths): the forcing (2n doubles) and the cos / sin
 * homogeneous columns (n doubles each). */
int or_planewave_rhs(const or_seg *segs, int64_t n, double freq_hz, const or_wave *wave, const int64_t *path_of,
                     const double *sign, const double *s_mid, double *rhs, double *cosv, double *sinv);
/* linear.rs:910-993 solve_hallen_planewave (free_ends == NULL: I = 0 at
 * both ends of each per-tag wire) and :1024-1090 solve_hallen_planewave_paths
 * (the listed free-end rows): two homogeneous columns (cos, sin) per wire or
 * path, the same regularised normal equations and GEPP; x: 2(n + 2w). */
int or_solve_hallen_planewave(const double *z, int64_t n, const double *rhs, const double *cosv,
                              const double *sinv, const int64_t *row_wire, int64_t w, const int64_t *free_ends,
                              int64_t n_free, double *x, int32_t *pivots, double *gram, int naive);

/* A whole per-frequency solve of the CLI standard Hallen branch
 * (solve_session.rs:1186-1437 + :1645): geometry -> rhs -> Z -> merged
 * endpoints + junctions -> solve_hallen -> feedpoints -> pattern.  */
typedef struct {
    const or_wire *wires;
    int64_t n_wires;
    const or_source *sources;
    int64_t n_sources;
    int ground;
    double freq_hz;
    const double *points; /* 2*n_points (theta, phi) deg; may be NULL */
    int64_t n_points;
    /* outputs (caller-allocated) */
    double *currents;     /* 2*N */
    double *feed;         /* 7 * n_sources */
    int64_t *n_feed;
    double *pattern;      /* 4 * n_points */
    int32_t *pivots;      /* S, optional */
    int status;
    const or_load *loads; /* LD cards in deck order; may be NULL */
    int64_t n_loads;
    const or_tl *tls;     /* TL cards in deck order; may be NULL */
    int64_t n_tls;
    const or_nt *nts;     /* NT cards in deck order; may be NULL */
    int64_t n_nts;
    /* the first plane-wave EX card, or NULL: with it the problem is the CLI's
     * receive solve (solve_session.rs:262-301); voltage sources are then not
     * used and no feed rows are produced */
    const or_wave *wave;
} or_problem;

/* Solve one problem; returns its status. */
int or_solve_problem(or_problem *p);
/* Solve many independent problems on nthreads host threads (one problem per
 * thread at a time), mirroring the reference's rayon per-frequency
 * parallelism.  Each solve is single-threaded, as in the reference. */
void or_solve_problems(or_problem *ps, int64_t count, int nthreads);

#ifdef __cplusplus
}
#endif
#endif

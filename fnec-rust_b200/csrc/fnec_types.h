// fnec_types.h -- device-side data layout of a Hallen batch.
//
// A batch holds A antennas (geometries) and U units; a unit is one
// (antenna, frequency) solve.  Everything the kernels touch lives in a few
// flat device arrays addressed through the descriptors below:
//
//   segments   DevSeg[total_segments]          128 B each, one cache line
//   Z          complex128 N*N per unit          row-major
//   A          complex128 S*(S+1) per unit      augmented [A | b], row-major
//   x          complex128 S per unit            solution (currents, C_hom)
//   rhs, cosv  complex128 N / f64 N per unit    Hallen RHS and cos(k s)
//
// S = N + W where W is the number of (merged) wire endpoint pairs.
#pragma once
#include <stdint.h>

namespace fnec {

struct DevSeg {          // nec_solver::geometry::Segment (geometry.rs:115-134)
    double mid[3];
    double dir[3];
    double len;
    double rad;
    double start[3];
    double end[3];
    uint32_t tag;
    uint32_t tag_index;
    // 2 ln((len/2 + sqrt((len/2)^2 + rad^2)) / rad): the analytic part of
    // the self term (matrix.rs:297-331), evaluated on the host with the
    // platform libm so that the exact fill uses the reference's value
    double self_log;
};
static_assert(sizeof(DevSeg) == 128, "DevSeg is one 128-byte line");

struct DevWire {         // one GW card, expanded by k_expand_segments
    double start[3];
    double end[3];
    double radius;
    uint32_t tag;
    uint32_t nseg;
    int64_t seg_off;     // global index of its first segment
    double self_log;     // DevSeg::self_log of its segments (all equal)
};

// A straight run of segments whose midpoints advance by a constant step
// (every GW card expands into one).  Used by the far-field Horner sum.
struct DevRun {
    double mid0[3];      // midpoint of the first segment
    double step[3];      // midpoint increment between consecutive segments
    double dir[3];
    double len;
    int32_t first;       // antenna-local index of the first segment
    int32_t count;
};

struct AntDesc {
    int64_t seg_off;     // into segments
    int32_t n;           // segments
    int32_t w;           // homogeneous columns (merged wires)
    int64_t rowwire_off; // int32[n]: wire column of each row (linear.rs:728-733)
    int64_t wrow_off;    // CSR: int32 rows of each wire column, wrow_ptr
    int64_t wptr_off;    // int32[w+1]
    int64_t comp_off;    // int32[2n]: merged component (first,last) of each segment
    int64_t src_off;     // DevSource[n_src] (resolved BTreeMap order), grouped by right-hand side
    int32_t n_src;
    int32_t n_rhs;       // right-hand sides per system
    int64_t sptr_off;    // int32[n_rhs+1]: sources of right-hand side r = srcs[sptr[r] .. sptr[r+1])
    int64_t fptr_off;    // int32[n_rhs+1]: feed rows of right-hand side r
    int32_t n_con;       // constraint pair groups
    int64_t con_off;     // DevConstraint groups
    int64_t conv_off;    // int32 value codes for each group (row order)
    int64_t feed_off;    // DevFeed[n_feed]
    int32_t n_feed;
    int32_t ground;      // 0 free space, 1 PEC image
    int64_t run_off;     // DevRun[n_run]
    int32_t n_run;
    int32_t n_crow;      // constraint rows of M (free ends, then junctions)
    int64_t crow_off;    // DevConRow[n_crow]
    int64_t ccptr_off;   // int32[n+1]: CSR of the constraint rows touching each column
    int64_t ccq_off;     // int32: those rows (ascending), ccptr-indexed
    // degree-2 conductor paths (solve_session.rs:1338-1378): one column per
    // path (rowwire), I = 0 rows at the two free ends of each path, and
    // cos / source terms along the signed arc length of each path
    int32_t paths;       // 1: the path form; 0: merged straight wires
    // plane-wave form (linear.rs:910-1090): two homogeneous columns per wire
    // or path, cos (2q) then sin (2q + 1); cos(k s) then sin(k s) per system
    // (2n doubles); the arc table holds s and sign for both layouts
    int32_t hom2;
    int64_t arc_off;     // doubles: s_mid[n] (signed arc length), then sign[n]
    int64_t wave_off;    // doubles: 10 per right-hand side (r_hat, pol re, pol im, pad)
    int64_t koff_off;    // int32[n]: row m's entry of the system's sin(k |s_m - s_p|) table
};

// One constraint row of M (linear.rs:744-762): M[N+q][c0] = 1 and, for a
// junction row, M[N+q][c1] = v1 (c1 = -1 for a free-end I = 0 row).
struct DevConRow {
    int32_t c0, c1;
    double v1;
};

struct DevSource {       // one resolved delta-gap source (excitation.rs:171-187)
    int32_t feed;        // antenna-local segment index
    int32_t comp_first;  // merged component of the feed segment (path form: unused)
    int32_t comp_last;
    int32_t pad;
    double v_re, v_im;
};

struct DevFeed {         // one EX card row of build_feedpoint_rows
    int32_t seg;
    int32_t pad;
    double vdl_re, vdl_im;   // v_vec[idx] = sum of V/dl on that segment
};

// One (i, j) entry of the Gram touched by constraint rows; its
// contributions, in row order, are codes in conv[begin .. begin+count):
// each code packs (u_val, v_val) with values in {1, -1}.
struct DevConstraint {
    int32_t i, j;
    int32_t begin, count;
};

// A system is one (antenna, frequency): one Z, one normal-equation matrix,
// one factorisation.  A solve is one right-hand side of a system (the
// superposed EX cards of a deck, or -- for served requests -- each source
// position separately); solves share their system's factor.  Kernels that
// work per system and kernels that work per solve both take UnitDesc
// arrays: a solve's descriptor is its system's with the per-solve offsets.
struct UnitDesc {
    int32_t ant;
    int32_t n;
    int32_t s;           // n + w
    int32_t rhs;         // right-hand side index of a solve (0 for a system)
    double freq;
    double k_fill;       // 2*pi*f/c (matrix.rs:194, excitation.rs:165)
    double k_rp;         // 2*pi/(c/f) (farfield.rs:570-571)
    int64_t z_off;       // complex elements of Z (per system)
    int64_t a_off;       // complex elements of [A|b] (per system)
    int64_t x_off;       // complex elements of the solution (per solve; a system: its solve 0)
    int64_t rhs_off;     // complex elements of the Hallen RHS (per solve; a system: its solve 0)
    int64_t cos_off;     // doubles of cos(k s) (per system)
    int64_t piv_off;     // int32 pivot rows (per system)
    int64_t pat_off;     // requested pattern points (per solve)
    int32_t n_rhs;       // right-hand sides of the system
    int32_t sys;         // system index of a solve
};

// Requested pattern points of one antenna: an RP card grid (phi outer,
// theta inner, farfield.rs:677-699) or an explicit (theta, phi) list.
struct DevRp {
    int32_t n_theta, n_phi;
    double theta0, phi0, d_theta, d_phi;
    int64_t pts_off;      // >= 0: explicit list of n_pts (theta, phi) pairs
    int32_t n_pts;
    int32_t skip_integral;  // 1: use total_given instead of integrating
    double total_given;
    // Requested points that coincide with a power-integration direction
    // reuse its field: i2r (int32[n_int], -1 = none) maps integration
    // directions to requested points; the other requested points are
    // listed in xr (int32[n_xr]).  i2r_off < 0: no maps, every requested
    // point is computed on its own (n_xr = all of them, in order).
    int64_t i2r_off;
    int64_t xr_off;
    int32_t n_xr;
    int32_t pad_rp;
};

// One stamp: Z[index] += (re, im) on a system's Z (matrix.rs:131-139
// add_to_diagonal of the LD loads, matrix.rs add_to_entry of the TL / NT
// two-ports).  Stamps on one entry are consecutive, in the reference's
// order (loads, then TL cards, then NT cards); `first` marks the first of
// each entry's run.
struct DevStamp {
    int64_t index;  // complex element of the batch's Z
    double re, im;
    int32_t first;  // 1 on the first stamp of an entry
    int32_t count;  // on the first: the run's length
};

// Constraint-row contribution codes: bit 1 set -> the conj side is -1,
// bit 0 set -> the other side is -1 (values are 1 or the junction sign).
inline int32_t con_code(double u, double v) { return (u < 0 ? 2 : 0) | (v < 0 ? 1 : 0); }

}  // namespace fnec

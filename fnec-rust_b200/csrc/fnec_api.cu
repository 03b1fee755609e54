// fnec_api.cu -- host orchestration and the C ABI of libfnec_cuda.so.
//
// Host work is the small, branchy topology of a geometry (wire endpoint
// runs, collinear merge, junction pairs, constraint rows, resolved sources,
// feedpoint rows, wire runs for the far field); it follows the reference
// functions cited inline with the same IEEE arithmetic (built with
// -ffp-contract=off).  Everything proportional to N^2 or N^3 runs on the
// device: segment expansion, Hallen RHS, Z fill, Gram, factorisation,
// solve, feedpoints and the pattern grid.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <tuple>
#include <vector>

#include "fnec_cuda.h"
#include "fnec_kernels.h"
#include "fnec_mixed.h"

using namespace fnec;

namespace {

constexpr double PI = 3.14159265358979323846;
constexpr double C0 = 299792458.0;

struct Err {
    int code;
    std::string msg;
};

}  // namespace

struct fnec_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::string err;
};

static int fail(fnec_ctx *c, int code, const std::string &msg) {
    if (c) c->err = msg;
    return code;
}

#define CUDA_TRY(ctx, call)                                                                   \
    do {                                                                                      \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess) {                                                              \
            int code_ = (e_ == cudaErrorMemoryAllocation) ? FNEC_ERR_OUT_OF_MEMORY : FNEC_ERR_CUDA; \
            return fail((ctx), code_, std::string(#call) + ": " + cudaGetErrorString(e_));   \
        }                                                                                     \
    } while (0)

// ---------------------------------------------------------------------------
// host restatements needed for topology (same arithmetic as k_expand_segments)
// ---------------------------------------------------------------------------
// The analytic part of the self term, 2 ln((h + sqrt(h^2 + a^2)) / a) with
// h = len / 2 (matrix.rs:297-331), in the reference's operation order and
// with the host libm's ln -- the library the reference's f64::ln calls.
static double self_log_term(double len, double rad) {
    double half = len * 0.5;
    double r_end = std::sqrt(half * half + rad * rad);
    return 2.0 * std::log((half + r_end) / rad);
}

static DevSeg host_seg(const fnec_wire &gw, uint32_t i) {
    double dx = gw.end[0] - gw.start[0], dy = gw.end[1] - gw.start[1], dz = gw.end[2] - gw.start[2];
    double wl = std::sqrt(dx * dx + dy * dy + dz * dz);
    double nn = (double)gw.segments;
    double t0 = (double)i / nn, t1 = ((double)i + 1.0) / nn, tm = (t0 + t1) * 0.5;
    DevSeg s;
    s.start[0] = gw.start[0] + dx * t0;
    s.start[1] = gw.start[1] + dy * t0;
    s.start[2] = gw.start[2] + dz * t0;
    s.end[0] = gw.start[0] + dx * t1;
    s.end[1] = gw.start[1] + dy * t1;
    s.end[2] = gw.start[2] + dz * t1;
    s.mid[0] = gw.start[0] + dx * tm;
    s.mid[1] = gw.start[1] + dy * tm;
    s.mid[2] = gw.start[2] + dz * tm;
    s.dir[0] = dx / wl;
    s.dir[1] = dy / wl;
    s.dir[2] = dz / wl;
    s.len = wl / nn;
    s.rad = gw.radius;
    s.tag = gw.tag;
    s.tag_index = i + 1;
    s.self_log = self_log_term(s.len, s.rad);
    return s;
}

static double dist2(const double *a, const double *b) {
    double d0 = a[0] - b[0], d1 = a[1] - b[1], d2 = a[2] - b[2];
    return d0 * d0 + d1 * d1 + d2 * d2;
}

// geometry.rs:227-236
static bool dir_aligned(const double *a, const double *b, double tol) {
    double cr[3] = {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
    double zero[3] = {0, 0, 0};
    double dot = a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
    return dist2(cr, zero) < tol * tol && dot > 0.0;
}

namespace {

// Everything the device needs for one antenna, before packing.
struct HostAnt {
    std::vector<DevWire> wires;     // empty for caller-provided segments
    std::vector<DevSeg> segs;       // host copies of the segments
    int ground = 0;
    std::vector<std::pair<int64_t, int64_t>> ep;  // column wires (first, last)
    std::vector<int32_t> comp;      // 2n merged component (first, last) per segment
    std::vector<int64_t> ja, jb;    // junction rows
    std::vector<double> js;
    std::vector<std::vector<DevSource>> rhs_srcs;  // sources of each right-hand side
    std::vector<std::vector<DevFeed>> rhs_feeds;   // feed rows of each right-hand side
    std::vector<DevRun> runs;
    DevRp rp{};
    std::vector<double> pts;        // explicit points (theta, phi)
    std::vector<double> freqs;
    bool rhs_given = false;         // caller supplies rhs/cos (one unit)
    std::vector<double> rhs, cosv;  // 2n, n
    std::vector<double> z;          // caller-supplied Z (2 n^2), else filled on the device
    // degree-2 conductor-path form (solve_session.rs:1338-1378)
    bool paths = false;
    std::vector<int32_t> path_of;   // column (path) of each row
    std::vector<double> arc;        // 2n: signed arc length of each midpoint, then its sign
    std::vector<int64_t> free_ends; // 2 per path: I = 0 rows
    // plane-wave receive form: two homogeneous columns per wire or path, one
    // right-hand side per incidence direction (theta, phi) with its r_hat and
    // polarisation vector (10 doubles)
    bool planewave = false;
    std::vector<double> dirs;       // 2 per right-hand side
    std::vector<double> waves;      // 10 per right-hand side
    int64_t cols() const {
        const int64_t c = paths ? (int64_t)free_ends.size() / 2 : (int64_t)ep.size();
        return planewave ? 2 * c : c;
    }
    std::vector<fnec_load> loads;   // LD cards, deck order
    std::vector<fnec_tl> tls;       // TL cards, deck order
    std::vector<fnec_nt> nts;       // NT cards, deck order
    bool stamped() const { return !loads.empty() || !tls.empty() || !nts.empty(); }
};

// num-complex 0.4.6 arithmetic on the host, each operation separately
// rounded (this file is built without FMA contraction)
struct HC {
    double re, im;
};
inline HC hc_add(HC a, HC b) { return {a.re + b.re, a.im + b.im}; }
inline HC hc_mul(HC a, HC b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
inline HC hc_div(HC a, HC b) {
    const double n = b.re * b.re + b.im * b.im;
    return {(a.re * b.re + a.im * b.im) / n, (a.im * b.re - a.re * b.im) / n};
}
inline HC hc_scale(HC a, double s) { return {a.re * s, a.im * s}; }
inline HC hc_divr(HC a, double s) { return {a.re / s, a.im / s}; }
inline double hc_norm(HC a) { return std::hypot(a.re, a.im); }

// I0(z)/I1(z) (loads.rs:34-57): power series up to |z| = 15, the
// asymptotic expansion beyond.
HC bessel_i0_over_i1(HC z) {
    if (hc_norm(z) > 15.0) {
        const HC inv = hc_div({1.0, 0.0}, z);
        return hc_add(hc_add({1.0, 0.0}, hc_scale(inv, 0.5)), hc_scale(hc_mul(inv, inv), 0.375));
    }
    const HC half = hc_scale(z, 0.5), half_sq = hc_mul(half, half);
    HC i0{1.0, 0.0}, t0{1.0, 0.0}, i1 = half, t1 = half;
    for (int k = 1; k < 300; ++k) {
        const double kf = (double)k;
        t0 = hc_mul(t0, hc_divr(half_sq, kf * kf));
        i0 = hc_add(i0, t0);
        t1 = hc_mul(t1, hc_divr(half_sq, kf * (kf + 1.0)));
        i1 = hc_add(i1, t1);
        if (hc_norm(t0) <= 1e-17 * hc_norm(i0) && hc_norm(t1) <= 1e-17 * hc_norm(i1)) break;
    }
    return hc_div(i0, i1);
}

// tl.rs:186-241 find_segment_index: segment 0 is the tag's centre segment
// (the middle one of an odd count, the lower centre of an even count).
int64_t tl_segment(const std::vector<DevSeg> &s, uint32_t tag, uint32_t seg) {
    if (seg != 0) {
        for (size_t i = 0; i < s.size(); ++i)
            if (s[i].tag == tag && s[i].tag_index == seg) return (int64_t)i;
        return -1;
    }
    std::vector<size_t> tagged;
    for (size_t i = 0; i < s.size(); ++i)
        if (s[i].tag == tag) tagged.push_back(i);
    if (tagged.empty()) return -1;
    size_t pick = tagged.size() / 2;
    if (tagged.size() % 2 == 0) {
        const uint32_t lower = (uint32_t)(tagged.size() / 2);
        pick = tagged.size() / 2 - 1;
        for (size_t q = 0; q < tagged.size(); ++q)
            if (s[tagged[q]].tag_index == lower) {
                pick = q;
                break;
            }
    }
    return (int64_t)tagged[pick];
}

struct Stamp {
    int64_t row, col;
    HC v;
};

// The two-port stamps of the TL cards (tl.rs:47-183) then the NT cards
// (network.rs:55-142) at one frequency, in order, 4 per applied card.
void network_stamps(const HostAnt &h, double freq_hz, std::vector<Stamp> &out) {
    const double PI_ = 3.14159265358979323846, C0_ = 299792458.0;
    const double k = 2.0 * PI_ * freq_hz / C0_;
    auto put4 = [&](int64_t i1, int64_t i2, HC d1, HC d2, HC o12, HC o21) {
        out.push_back({i1, i1, d1});
        out.push_back({i2, i2, d2});
        out.push_back({i1, i2, o12});
        out.push_back({i2, i1, o21});
    };
    for (const fnec_tl &T : h.tls) {
        const int64_t i1 = tl_segment(h.segs, T.tag1, T.seg1);
        if (i1 < 0) continue;
        const int64_t i2 = tl_segment(h.segs, T.tag2, T.seg2);
        if (i2 < 0 || i1 == i2 || T.z0 <= 0.0 || T.length <= 0.0) continue;
        if (T.tl_type != 0) {  // lossy: Z0 coth(gl), Z0 csch(gl)
            const double beta_l = k * T.length, alpha_l = T.f3 * 2.302585092994046 / 20.0;  // ln 10
            const HC sh{std::sinh(alpha_l) * std::cos(beta_l), std::cosh(alpha_l) * std::sin(beta_l)};
            const HC ch{std::cosh(alpha_l) * std::cos(beta_l), std::sinh(alpha_l) * std::sin(beta_l)};
            if (hc_norm(sh) < 1e-9) continue;
            const HC z0c{T.z0, 0.0};
            const HC zd = hc_div(hc_mul(z0c, ch), sh), zo = hc_div(z0c, sh);
            put4(i1, i2, zd, zd, zo, zo);
            continue;
        }
        const double vf = (T.f3 >= 0.0 && T.f3 <= 1.0 && T.f3 > 0.0) ? T.f3 : 1.0;
        const double theta = k * T.length / vf, sin_t = std::sin(theta);
        if (std::fabs(sin_t) < 1e-9) continue;
        const double cot = std::cos(theta) / sin_t, csc = 1.0 / sin_t;
        const HC zd{0.0, -T.z0 * cot}, zo{0.0, -T.z0 * csc};
        put4(i1, i2, zd, zd, zo, zo);
    }
    for (const fnec_nt &N : h.nts) {
        const HC y11{N.y11_re, N.y11_im}, y12{N.y12_re, N.y12_im}, y21 = y12, y22{N.y22_re, N.y22_im};
        const int64_t i1 = tl_segment(h.segs, N.tag1, N.seg1);
        if (i1 < 0) continue;
        const int64_t i2 = tl_segment(h.segs, N.tag2, N.seg2);
        if (i2 < 0 || i1 == i2) continue;
        const HC p = hc_mul(y11, y22), q = hc_mul(y12, y21);
        const HC det{p.re - q.re, p.im - q.im};
        if (hc_norm(det) < 1e-30) continue;
        put4(i1, i2, hc_div(y22, det), hc_div(y11, det), hc_div({-y12.re, -y12.im}, det),
             hc_div({-y21.re, -y21.im}, det));
    }
}

// Series load impedance of every segment at one frequency (loads.rs:103-222,
// the cards summed in deck order); exact zeros where no card applies.
void segment_loads(const HostAnt &h, double freq_hz, std::vector<HC> &out) {
    const double PI_ = 3.14159265358979323846;
    const double TWO_PI = 2.0 * PI_, MU0 = 4.0 * PI_ * 1e-7;
    const double omega = TWO_PI * freq_hz;
    out.assign(h.segs.size(), HC{0.0, 0.0});
    for (const fnec_load &L : h.loads) {
        if (L.load_type < 0 || L.load_type > 5) continue;  // the reference warns and ignores it
        if (L.load_type == 5 && L.f1 <= 0.0) continue;     // sigma <= 0: likewise
        for (size_t i = 0; i < h.segs.size(); ++i) {
            const DevSeg &s = h.segs[i];
            if (L.tag != 0 && s.tag != L.tag) continue;  // segment_matches (loads.rs:209-222)
            if (L.seg_first != 0) {
                const uint32_t last = L.seg_last == 0 ? L.seg_first : L.seg_last;
                if (s.tag_index < L.seg_first || s.tag_index > last) continue;
            }
            HC z{0.0, 0.0};
            switch (L.load_type) {
            case 0:
                z = {L.f1, omega * L.f2 - (L.f3 > 0.0 ? 1.0 / (omega * L.f3) : 0.0)};
                break;
            case 1: {
                HC y{0.0, 0.0};
                if (L.f1 > 0.0) y = hc_add(y, {1.0 / L.f1, 0.0});
                if (L.f2 > 0.0) y = hc_add(y, {0.0, -1.0 / (omega * L.f2)});
                if (L.f3 > 0.0) y = hc_add(y, {0.0, omega * L.f3});
                z = hc_norm(y) < 1e-30 ? HC{0.0, 0.0} : hc_div({1.0, 0.0}, y);
                break;
            }
            case 2: z = {L.f1, omega * L.f2}; break;
            case 3: z = {L.f1, -(L.f3 > 0.0 ? 1.0 / (omega * L.f3) : 0.0)}; break;
            case 4: z = {L.f1, L.f2}; break;
            default: {  // 5: round-wire skin-effect impedance (loads.rs:73-81)
                const double sigma = L.f1, rad = s.rad, dl = s.len;
                if (omega <= 0.0) {
                    z = {dl / (sigma * PI_ * rad * rad), 0.0};
                } else {
                    const double delta = std::sqrt(2.0 / (omega * MU0 * sigma));
                    const HC gamma{1.0 / delta, 1.0 / delta};
                    z = hc_scale(hc_mul(hc_divr(gamma, TWO_PI * rad * sigma), bessel_i0_over_i1(hc_scale(gamma, rad))),
                                 dl);
                }
                break;
            }
            }
            out[i] = hc_add(out[i], z);
        }
    }
}

}  // namespace

// geometry.rs:168-185 over the segment list
static std::vector<std::pair<int64_t, int64_t>> wire_endpoints(const std::vector<DevSeg> &s) {
    std::vector<std::pair<int64_t, int64_t>> out;
    uint32_t cur = UINT32_MAX;
    int64_t first = 0;
    for (int64_t i = 0; i < (int64_t)s.size(); ++i) {
        if (s[i].tag != cur) {
            if (cur != UINT32_MAX) out.push_back({first, i - 1});
            cur = s[i].tag;
            first = i;
        }
    }
    if (cur != UINT32_MAX) out.push_back({first, (int64_t)s.size() - 1});
    return out;
}

// geometry.rs:200-225
static std::vector<std::pair<int64_t, int64_t>> merge_collinear(const std::vector<DevSeg> &s) {
    auto base = wire_endpoints(s);
    if (base.size() < 2) return base;
    const double POS_TOL = 1e-6, DIR_TOL = 1e-6;
    std::vector<std::pair<int64_t, int64_t>> merged;
    auto cur = base[0];
    for (size_t k = 1; k < base.size(); ++k) {
        auto nx = base[k];
        const DevSeg &a = s[cur.second];
        const DevSeg &b = s[nx.first];
        bool contiguous = cur.second + 1 == nx.first;
        bool connects = dist2(a.end, b.start) < POS_TOL * POS_TOL;
        bool collinear = dir_aligned(a.dir, b.dir, DIR_TOL);
        bool same_radius = std::fabs(a.rad - b.rad) < POS_TOL;
        if (contiguous && connects && collinear && same_radius) {
            cur.second = nx.second;
        } else {
            merged.push_back(cur);
            cur = nx;
        }
    }
    merged.push_back(cur);
    return merged;
}

// geometry.rs:274-339 + solve_session.rs:1386-1400 (cross-component pairs)
static void cli_junctions(const std::vector<DevSeg> &s,
                          const std::vector<std::pair<int64_t, int64_t>> &ep, HostAnt &h) {
    size_t nn = 2 * ep.size();
    std::vector<int64_t> comp(s.size(), 0);
    for (size_t c = 0; c < ep.size(); ++c)
        for (int64_t m = ep[c].first; m <= ep[c].second; ++m) comp[m] = (int64_t)c;
    for (size_t i = 0; i < nn; ++i) {
        int64_t si = (i % 2 == 0) ? ep[i / 2].first : ep[i / 2].second;
        bool st_i = i % 2 == 0;
        const double *pi = st_i ? s[si].start : s[si].end;
        for (size_t j = i + 1; j < nn; ++j) {
            int64_t sj = (j % 2 == 0) ? ep[j / 2].first : ep[j / 2].second;
            if (si == sj) continue;
            bool st_j = j % 2 == 0;
            const double *pj = st_j ? s[sj].start : s[sj].end;
            double dx = pi[0] - pj[0], dy = pi[1] - pj[1], dz = pi[2] - pj[2];
            if (std::sqrt(dx * dx + dy * dy + dz * dz) > 1e-6) continue;
            if (comp[si] == comp[sj]) continue;
            h.ja.push_back(si);
            h.jb.push_back(sj);
            h.js.push_back(st_i == st_j ? 1.0 : -1.0);
        }
    }
}

// geometry.rs:404-584 (build_conductor_paths) and the guard of
// solve_session.rs:1338-1340: the per-tag wires are joined through
// endpoint nodes where exactly two ends meet (within 1e-6 m) into open
// chains.  Returns true -- and fills the path form of h -- only when every
// node has degree <= 2, no chain is closed, and some chain is not a plain
// forward run of ascending segments; otherwise h is left as it was.
static bool conductor_paths(HostAnt &h) {
    const auto &s = h.segs;
    const auto wires = wire_endpoints(s);
    const int64_t nw = (int64_t)wires.size(), n = (int64_t)s.size();
    if (nw == 0) return false;
    auto point = [&](int64_t id) -> const double * {  // endpoint id = 2 wire + (0 start, 1 end)
        return id % 2 == 0 ? s[wires[id / 2].first].start : s[wires[id / 2].second].end;
    };
    // nodes: coincident endpoints, numbered in order of their first endpoint
    std::vector<int64_t> node(2 * nw, -1);
    std::vector<std::vector<int64_t>> members;
    for (int64_t id = 0; id < 2 * nw; ++id) {
        if (node[id] >= 0) continue;
        node[id] = (int64_t)members.size();
        members.push_back({id});
        for (int64_t j = 0; j < 2 * nw; ++j)
            if (node[j] < 0 && dist2(point(id), point(j)) < 1e-6 * 1e-6) {
                node[j] = node[id];
                members.back().push_back(j);
            }
    }
    std::vector<int64_t> up(nw);
    for (int64_t i = 0; i < nw; ++i) up[i] = i;
    auto root = [&](int64_t x) {
        while (up[x] != x) x = up[x];
        return x;
    };
    for (auto &m : members) {
        if (m.size() >= 3) return false;  // T/Y junction
        if (m.size() == 2) {
            if (m[0] / 2 == m[1] / 2) return false;  // a wire closed on itself
            up[root(m[0] / 2)] = root(m[1] / 2);
        }
    }
    std::vector<int32_t> path_of(n, 0);
    std::vector<double> smid(n, 0.0), sgn(n, 1.0);
    std::vector<int64_t> fends;
    std::vector<char> seen(nw, 0);
    bool nontrivial = false;
    int32_t np = 0;
    std::vector<int64_t> roots(nw);
    for (int64_t i = 0; i < nw; ++i) roots[i] = root(i);
    for (int64_t r = 0; r < nw; ++r) {  // chains in ascending order of their root wire
        std::vector<int64_t> ends;
        for (int64_t wi = 0; wi < nw; ++wi)
            if (roots[wi] == r)
                for (int e = 0; e < 2; ++e)
                    if (members[node[2 * wi + e]].size() == 1) ends.push_back(2 * wi + e);
        bool any = false;
        for (int64_t wi = 0; wi < nw && !any; ++wi) any = roots[wi] == r;
        if (!any) continue;
        if (ends.size() != 2) return false;  // a closed chain
        std::vector<int64_t> order;
        double arc = 0.0;
        int64_t cur = ends[0] / 2, enter = ends[0] % 2;
        for (;;) {
            seen[cur] = 1;
            const double sg = enter == 0 ? 1.0 : -1.0;
            const int64_t f = wires[cur].first, l = wires[cur].second;
            for (int64_t t = 0; t <= l - f; ++t) {
                const int64_t m = enter == 0 ? f + t : l - t;
                if (sg != 1.0 || (!order.empty() && m != order.back() + 1)) nontrivial = true;
                smid[m] = arc + s[m].len * 0.5;
                arc += s[m].len;
                sgn[m] = sg;
                path_of[m] = np;
                order.push_back(m);
            }
            const auto &at = members[node[2 * cur + (1 - enter)]];
            if (at.size() == 1) break;
            int64_t next = -1;
            for (int64_t id : at)
                if (id / 2 != cur && !seen[id / 2]) next = id;
            if (next < 0) break;
            cur = next / 2;
            enter = next % 2;
        }
        for (int64_t m : order) smid[m] = smid[m] - arc * 0.5;
        fends.push_back(order.front());
        fends.push_back(order.back());
        ++np;
    }
    if (!nontrivial) return false;
    h.paths = true;
    h.path_of = std::move(path_of);
    h.arc.assign(smid.begin(), smid.end());
    h.arc.insert(h.arc.end(), sgn.begin(), sgn.end());
    h.free_ends = std::move(fends);
    return true;
}

static int64_t find_seg(const std::vector<DevSeg> &s, uint32_t tag, uint32_t idx) {
    for (int64_t i = 0; i < (int64_t)s.size(); ++i)
        if (s[i].tag == tag && s[i].tag_index == idx) return i;
    return -1;
}

// Wire runs for the far-field Horner sum: consecutive segments with the
// same direction and length whose midpoints advance by a constant step.
static void build_runs(HostAnt &h) {
    const auto &s = h.segs;
    int64_t n = (int64_t)s.size();
    int64_t i = 0;
    while (i < n) {
        int64_t j = i + 1;
        double step[3] = {0, 0, 0};
        if (j < n) {
            for (int c = 0; c < 3; ++c) step[c] = s[j].mid[c] - s[i].mid[c];
        }
        double sl = std::sqrt(step[0] * step[0] + step[1] * step[1] + step[2] * step[2]);
        while (j < n) {
            bool same = s[j].dir[0] == s[i].dir[0] && s[j].dir[1] == s[i].dir[1] &&
                        s[j].dir[2] == s[i].dir[2] && s[j].len == s[i].len;
            double e = 0;
            for (int c = 0; c < 3; ++c) {
                double pred = s[i].mid[c] + step[c] * (double)(j - i);
                e = std::max(e, std::fabs(pred - s[j].mid[c]));
            }
            double scale = std::max(1.0, std::fabs(s[j].mid[0]) + std::fabs(s[j].mid[1]) + std::fabs(s[j].mid[2]));
            if (!same || sl == 0.0 || e > 1e-12 * scale) break;
            ++j;
        }
        DevRun r{};
        for (int c = 0; c < 3; ++c) {
            r.mid0[c] = s[i].mid[c];
            r.step[c] = (j - i > 1) ? step[c] : 0.0;
            r.dir[c] = s[i].dir[c];
        }
        r.len = s[i].len;
        r.first = (int32_t)i;
        r.count = (int32_t)(j - i);
        h.runs.push_back(r);
        i = j;
    }
}

// excitation.rs:119-187 source resolution and :78-90 / solve_session.rs:846-917
// feed rows.  With separate == false the EX cards superpose into one
// right-hand side (a deck); with separate == true every card is its own
// right-hand side, solved as the single-source deck it stands for.
static void superposed_rhs(HostAnt &h, const std::vector<int64_t> &idx, const fnec_source *src, uint32_t ns,
                           std::vector<DevSource> &out_src, std::vector<DevFeed> &out_feed) {
    const auto &s = h.segs;
    uint32_t driven = s[idx[0]].tag;
    std::map<uint32_t, std::pair<int64_t, std::pair<double, double>>> by_tag;
    by_tag[driven] = {idx[0], {src[0].v_re, src[0].v_im}};
    for (uint32_t e = 0; e < ns; ++e) {
        if (src[e].tag == driven) continue;
        by_tag[src[e].tag] = {idx[e], {src[e].v_re, src[e].v_im}};
    }
    for (auto &kv : by_tag) {
        DevSource d{};
        d.feed = (int32_t)kv.second.first;
        d.comp_first = h.comp[2 * d.feed];
        d.comp_last = h.comp[2 * d.feed + 1];
        d.v_re = kv.second.second.first;
        d.v_im = kv.second.second.second;
        out_src.push_back(d);
    }
    // v_vec[idx] accumulates V/dl of every card on that segment
    for (uint32_t e = 0; e < ns; ++e) {
        DevFeed f{};
        f.seg = (int32_t)idx[e];
        double re = 0.0, im = 0.0;
        for (uint32_t q = 0; q < ns; ++q) {
            if (idx[q] != idx[e]) continue;
            double dl = s[idx[q]].len;
            re = re + src[q].v_re / dl;
            im = im + src[q].v_im / dl;
        }
        f.vdl_re = re;
        f.vdl_im = im;
        out_feed.push_back(f);
    }
}

static int resolve_sources(HostAnt &h, const fnec_source *src, uint32_t ns, bool separate, std::string &why) {
    const auto &s = h.segs;
    std::vector<int64_t> idx(ns);
    for (uint32_t e = 0; e < ns; ++e) {
        idx[e] = find_seg(s, src[e].tag, src[e].segment);
        if (idx[e] < 0) {
            why = "EX: no segment with tag " + std::to_string(src[e].tag) + ", index " +
                  std::to_string(src[e].segment);
            return FNEC_ERR_SEGMENT_NOT_FOUND;
        }
    }
    if (h.paths) {
        // excitation.rs:303-333: every voltage card, in deck order, drives
        // its own path (no per-tag merging); feed rows as in the plain form
        std::vector<DevSource> all;
        for (uint32_t e = 0; e < ns; ++e) {
            DevSource d{};
            d.feed = (int32_t)idx[e];
            d.comp_first = d.comp_last = -1;
            d.v_re = src[e].v_re;
            d.v_im = src[e].v_im;
            all.push_back(d);
        }
        std::vector<DevSource> none;
        if (ns == 0 || !separate) {
            h.rhs_srcs.assign(1, all);
            h.rhs_feeds.assign(1, {});
            if (ns > 0) superposed_rhs(h, idx, src, ns, none, h.rhs_feeds[0]);
            return FNEC_OK;
        }
        h.rhs_srcs.assign(ns, {});
        h.rhs_feeds.assign(ns, {});
        for (uint32_t e = 0; e < ns; ++e) {
            h.rhs_srcs[e] = {all[e]};
            std::vector<int64_t> one = {idx[e]};
            superposed_rhs(h, one, &src[e], 1, none, h.rhs_feeds[e]);
            none.clear();
        }
        return FNEC_OK;
    }
    if (ns == 0 || !separate) {
        h.rhs_srcs.assign(1, {});
        h.rhs_feeds.assign(1, {});
        if (ns > 0) superposed_rhs(h, idx, src, ns, h.rhs_srcs[0], h.rhs_feeds[0]);
        return FNEC_OK;
    }
    h.rhs_srcs.assign(ns, {});
    h.rhs_feeds.assign(ns, {});
    for (uint32_t e = 0; e < ns; ++e) {
        std::vector<int64_t> one = {idx[e]};
        superposed_rhs(h, one, &src[e], 1, h.rhs_srcs[e], h.rhs_feeds[e]);
    }
    return FNEC_OK;
}

static void set_comp(HostAnt &h, const std::vector<std::pair<int64_t, int64_t>> &merged) {
    h.comp.assign(2 * h.segs.size(), 0);
    for (auto &c : merged)
        for (int64_t m = c.first; m <= c.second; ++m) {
            h.comp[2 * m] = (int32_t)c.first;
            h.comp[2 * m + 1] = (int32_t)c.second;
        }
}

// ---------------------------------------------------------------------------
// batch
// ---------------------------------------------------------------------------
struct fnec_batch {
    fnec_ctx *ctx = nullptr;
    int precision = 0;
    // packed host tables
    std::vector<DevWire> wires;
    std::vector<DevSeg> segs;  // uploaded when the batch has no wires
    bool from_wires = true;
    std::vector<AntDesc> ants;
    std::vector<UnitDesc> units;   // systems (one factorisation each)
    std::vector<UnitDesc> solves;  // right-hand sides
    std::vector<int32_t> ibuf;
    std::vector<DevSource> srcs;
    std::vector<DevFeed> feeds;
    std::vector<DevConstraint> cons;
    std::vector<int32_t> codes;
    std::vector<DevConRow> crows;
    std::vector<DevRun> runs;
    std::vector<DevRp> rps;
    std::vector<double> pts;
    std::vector<int4> fill_units, gram_tiles;  // fill_units: (unit, tiles per side, first tile, 0)
    int64_t n_fill = 0;                         // 16x16 fill tiles, listed on the device (k_fill_tile_list)
    std::vector<int64_t> feed_row_off;
    std::vector<double> rhs_given;   // 2 * total rhs
    std::vector<double> cos_given;
    bool rhs_given_flag = false;
    std::vector<double> z_given;  // caller-supplied Z for every unit (fill skipped)
    std::vector<DevStamp> stamps; // LD load stamps on the filled Z
    std::vector<fnec_unit_info> uinfo;
    int max_s = 0, max_n = 0;
    int64_t tot_seg = 0, z_el = 0, a_el = 0, x_el = 0, rhs_el = 0, pat_el = 0, feed_rows = 0, cos_el = 0,
            piv_el = 0;
    int max_rhs = 1;
    int max_w = 0;
    int ff_blocks = 0;
    size_t ff_smem = 0;
    uint64_t launches = 0;
    uint64_t h2d = 0;
    // device
    DevWire *d_wires = nullptr;
    DevSeg *d_segs = nullptr;
    AntDesc *d_ants = nullptr;
    UnitDesc *d_units = nullptr;
    UnitDesc *d_solves = nullptr;
    int32_t *d_ibuf = nullptr;
    DevSource *d_srcs = nullptr;
    DevFeed *d_feeds = nullptr;
    DevConstraint *d_cons = nullptr;
    DevConRow *d_crows = nullptr;
    int32_t *d_codes = nullptr;
    DevRun *d_runs = nullptr;
    DevRp *d_rps = nullptr;
    double *d_pts = nullptr;
    int4 *d_fill_tiles = nullptr, *d_gram_tiles = nullptr, *d_fill_units = nullptr;
    int64_t *d_feed_row_off = nullptr;
    double *d_rhs_given = nullptr, *d_cos_given = nullptr, *d_z_given = nullptr;
    DevStamp *d_stamps = nullptr;
    cx *d_z = nullptr, *d_a = nullptr, *d_x = nullptr, *d_rhs = nullptr;
    double *d_cos = nullptr;
    int32_t *d_piv = nullptr, *d_status = nullptr;
    double *d_feed_out = nullptr, *d_fld = nullptr, *d_partials = nullptr, *d_pat = nullptr,
           *d_total = nullptr;
    cx *d_cur = nullptr;           // compact currents (read into pinned memory)
    int64_t *d_cur_off = nullptr;  // per solve: its first entry in d_cur
    // plane-wave antennas: per solve its incidence (theta, phi) or NaNs, and
    // the device's peak |I| of each solve
    bool has_wave = false;
    std::vector<double> recv_dirs;
    double *d_peak = nullptr;
    // right-hand sides beyond each system's first, in groups of up to 32
    // solves: (system, first solve, count, 0)
    std::vector<int4> rhs_groups;
    int4 *d_rhs_groups = nullptr;
    // a second stream for the first right-hand sides' back substitution,
    // which runs beside the grouped kernels of the others
    cudaStream_t side = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    // fnec_batch_run_report: the page-locked destination of the report's
    // pattern columns, copied chunk by chunk behind the far field
    double *sink = nullptr;
    cudaStream_t copy_st = nullptr;
    std::vector<cudaEvent_t> ev_chunk;
    cudaEvent_t ev_copy = nullptr;
    MixedWork mixed;
    GridPlan grid;
    // execution: the stream every operation of the batch is enqueued on.
    // Device memory comes from the device's stream-ordered pool (dev_pool),
    // which keeps what a destroyed batch freed for the next one; pooled
    // batches also borrow their pinned host arenas (the server's lanes)
    cudaStream_t st = nullptr;
    bool pooled = false;
    bool dev_pool = true;
    bool allow_grid = true;
    unsigned char *stage = nullptr;  // page-locked staging of uploads (pooled batches)
    size_t stage_cap = 0, stage_used = 0;
    double alloc_ms = 0;  // host time spent allocating (device pool, pinned arenas, mixed work)
    double create_ms = 0, antennas_ms = 0;  // fnec_batch_create in all, and its per-antenna planning
    double t_dev = 0, t_copy = 0, t_pinned = 0, t_mixed = 0;  // its parts: device allocations,
                                                             // table uploads, pinned arenas, mixed work
    std::vector<int32_t> grid_order;
    size_t dev_bytes = 0;
    std::vector<void *> allocs;
    // packed input arena: one pinned host buffer mirrored by one device buffer
    unsigned char *h_in = nullptr;
    unsigned char *d_in = nullptr;
    size_t in_bytes = 0;
    // pinned staging of the results
    unsigned char *h_out = nullptr;
    size_t out_bytes = 0;
    // per-phase CUDA events (profiling on)
    bool profile = false;
    cudaEvent_t ev[FNEC_N_PHASES + 1] = {};
    bool ev_made = false;
    // schedule and its CUDA graph
    fnec_schedule sched = {1, 1, 1, 1, 1, 1, 1, 1, 1, 0, 3, 0};
    cudaGraphExec_t gexec = nullptr;
    int graph_state = FNEC_GRAPH_NONE;
    uint64_t graph_launches = 0;  // launches the graph replays
    uint64_t n_runs = 0;  // fnec_batch_run calls
    std::string graph_why;        // why capture was refused
};

// Test hook for the allocation-failure path (fnec_test_fail_device_allocation):
// the n-th batch device allocation from now on fails as if the device were
// out of memory (once); -1 = off.
static std::atomic<int> g_fail_alloc_after{-1};
static bool take_injected_alloc_failure() {
    int v = g_fail_alloc_after.load();
    while (v >= 0) {
        if (g_fail_alloc_after.compare_exchange_weak(v, v - 1)) return v == 0;
    }
    return false;
}

template <typename T>
static cudaError_t dalloc(fnec_batch *b, T **p, size_t count) {
    *p = nullptr;
    if (count == 0) count = 1;
    if (take_injected_alloc_failure()) return cudaErrorMemoryAllocation;
    const auto t0 = std::chrono::steady_clock::now();
    cudaError_t e = b->dev_pool ? cudaMallocAsync((void **)p, sizeof(T) * count, b->st)
                                : cudaMalloc((void **)p, sizeof(T) * count);
    b->t_dev += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    if (e == cudaSuccess) {
        b->allocs.push_back(*p);
        b->dev_bytes += sizeof(T) * count;
    }
    return e;
}

template <typename T>
static cudaError_t up(fnec_batch *b, T *d, const std::vector<T> &h) {
    if (h.empty()) return cudaSuccess;
    b->h2d += sizeof(T) * h.size();
    const auto t0 = std::chrono::steady_clock::now();
    DevAlloc dev{b->st, b->dev_pool, b->stage, b->stage_cap, &b->stage_used};
    cudaError_t e = dev.upload(d, h.data(), sizeof(T) * h.size());
    b->t_copy += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return e;
}

// Page-locked host blocks kept for reuse: pinning pages is the slowest part
// of planning a batch (tens of milliseconds for its input arena), and a
// caller that plans a new batch per request frees and asks again for
// blocks of the same sizes.  A request takes the smallest cached block of
// at least its size and at most twice it (plus 4 MB); freed blocks are kept
// while the cache holds at most PIN_CACHE_MAX bytes.  Blocks are rounded up
// to 1 MB.  fnec_host_cache_release frees what is cached.
constexpr size_t PIN_CACHE_MAX = (size_t)1 << 30;
static std::mutex g_pin_mu;
static std::multimap<size_t, void *> g_pin_free;   // capacity -> block
static std::map<void *, size_t> g_pin_cap;          // every block handed out -> capacity
static size_t g_pin_cached = 0;

static cudaError_t pin_alloc(void **p, size_t bytes) {
    const size_t need = ((bytes ? bytes : 1) + ((size_t)1 << 20) - 1) & ~(((size_t)1 << 20) - 1);
    {
        std::lock_guard<std::mutex> lk(g_pin_mu);
        auto it = g_pin_free.lower_bound(need);
        if (it != g_pin_free.end() && it->first <= 2 * need + ((size_t)4 << 20)) {
            *p = it->second;
            g_pin_cached -= it->first;
            g_pin_cap[*p] = it->first;
            g_pin_free.erase(it);
            return cudaSuccess;
        }
    }
    cudaError_t e = cudaMallocHost(p, need);
    if (e != cudaSuccess) {
        *p = nullptr;
        return e;
    }
    std::lock_guard<std::mutex> lk(g_pin_mu);
    g_pin_cap[*p] = need;
    return cudaSuccess;
}

// false: p is not a block of this cache
static bool pin_free(void *p) {
    if (!p) return true;
    size_t cap = 0;
    {
        std::lock_guard<std::mutex> lk(g_pin_mu);
        auto it = g_pin_cap.find(p);
        if (it == g_pin_cap.end()) return false;
        cap = it->second;
        g_pin_cap.erase(it);
        if (g_pin_cached + cap <= PIN_CACHE_MAX) {
            g_pin_free.emplace(cap, p);
            g_pin_cached += cap;
            return true;
        }
    }
    cudaFreeHost(p);
    return true;
}

static void free_batch(fnec_batch *b) {
    for (void *p : b->allocs) {
        if (b->dev_pool) cudaFreeAsync(p, b->st);
        else cudaFree(p);
    }
    b->allocs.clear();
    if (!b->pooled) {  // pooled batches borrow their lane's pinned arenas
        pin_free(b->h_in);
        pin_free(b->h_out);
    }
    b->h_in = b->h_out = nullptr;
    if (b->gexec) cudaGraphExecDestroy(b->gexec);
    b->gexec = nullptr;
    if (b->ev_made)
        for (auto &e : b->ev) cudaEventDestroy(e);
    b->ev_made = false;
    for (auto e : b->ev_chunk) cudaEventDestroy(e);
    b->ev_chunk.clear();
    if (b->ev_copy) cudaEventDestroy(b->ev_copy);
    if (b->copy_st) cudaStreamDestroy(b->copy_st);
    b->ev_copy = nullptr;
    b->copy_st = nullptr;
    if (b->ev_fork) cudaEventDestroy(b->ev_fork);
    if (b->ev_join) cudaEventDestroy(b->ev_join);
    if (b->side) cudaStreamDestroy(b->side);
    b->ev_fork = b->ev_join = nullptr;
    b->side = nullptr;
    free_mixed(b->mixed, DevAlloc{b->st, b->dev_pool});
}

// Carve the packed input arena: every host table gets a 256-byte aligned
// slot; the device pointer of the table is the same offset in d_in.
struct Packer {
    std::vector<std::pair<const void *, size_t>> parts;
    std::vector<size_t> offs;
    size_t total = 0;
    template <typename T>
    size_t add(const std::vector<T> &v) {
        size_t off = total;
        parts.push_back({v.data(), sizeof(T) * v.size()});
        offs.push_back(off);
        total += (sizeof(T) * v.size() + 255) / 256 * 256;
        return off;
    }
};

// Pack host antennas into flat tables and allocate the device side.
// Far-field coverage maps (see DevRp): requested points whose (theta, phi)
// equal a power-integration direction's -- evaluated with the same
// expressions as the far-field kernel -- reuse that direction's field.
// Integration rows with sin(theta) == 0 are never evaluated (theta = 0), and
// the last row is left out as well; PEC points below the horizon need no
// field at all.
static void ff_cover_maps(const DevRp &rp, const double *pts, int ground, std::vector<int32_t> &i2r,
                          std::vector<int32_t> &xr) {
    const bool pec = ground == 1;
    const int n_th = pec ? 91 : 181;
    const double th_max = pec ? 90.0 : 180.0;
    const int n_int = rp.skip_integral ? 0 : n_th * 360;
    const int n_req = rp.pts_off >= 0 ? rp.n_pts : rp.n_theta * rp.n_phi;
    i2r.assign(n_int, -1);
    xr.clear();
    for (int p = 0; p < n_req; ++p) {
        double th, ph;
        if (rp.pts_off >= 0) {
            th = pts[2 * p];
            ph = pts[2 * p + 1];
        } else {
            int ip = p / rp.n_theta, it = p % rp.n_theta;
            th = rp.theta0 + (double)it * rp.d_theta;
            ph = rp.phi0 + (double)ip * rp.d_phi;
        }
        if (pec && th > 90.0) continue;  // clamped to -999.99 without a field
        bool covered = false;
        if (n_int > 0 && th >= 0.0 && ph >= 0.0 && ph < 360.0) {
            double step = th_max / ((double)n_th - 1.0);
            long it = std::lround(th / step), ip = std::lround(ph);
            if (it >= 1 && it < n_th - 1 && ip >= 0 && ip < 360) {
                double th_i = (double)it * th_max / ((double)n_th - 1.0), ph_i = (double)ip;
                int d = (int)(it * 360 + ip);
                if (th_i == th && ph_i == ph && i2r[d] < 0) {
                    i2r[d] = p;
                    covered = true;
                }
            }
        }
        if (!covered) xr.push_back(p);
    }
}

// Where a batch runs: the context's stream with its own allocations (the
// default), or a server lane's stream with pooled device memory and the
// lane's pinned arenas.
struct PinnedArena {
    unsigned char *p = nullptr;
    size_t cap = 0;
    cudaError_t ensure(size_t need) {
        if (need <= cap) return cudaSuccess;
        if (p) cudaFreeHost(p);
        p = nullptr;
        cap = 0;
        size_t grow = need + need / 2;  // geometric growth: few reallocations
        cudaError_t e = cudaMallocHost((void **)&p, grow);
        if (e == cudaSuccess) cap = grow;
        return e;
    }
    void release() {
        if (p) cudaFreeHost(p);
        p = nullptr;
        cap = 0;
    }
};
extern "C" {
static void schedule_from_cache(fnec_batch *b);  // defined with the C API below
static void apply_schedule(fnec_batch *b, const fnec_schedule &s);
}

struct BatchPlace {
    cudaStream_t st = nullptr;  // null: the context's stream
    bool pooled = false;
    bool allow_grid = true;
    PinnedArena *in = nullptr, *out = nullptr;  // pooled only
    PinnedArena *aux = nullptr;                 // pooled only: staging of the other uploads
};

static int build_batch(fnec_ctx *ctx, std::vector<HostAnt> &hs, int precision, fnec_batch **out,
                       bool need_solve = true, const BatchPlace &place = BatchPlace()) {
    int64_t n_solves = 0;
    for (const HostAnt &h : hs) {
        if (h.planewave && precision == FNEC_PRECISION_MIXED)
            return fail(ctx, FNEC_ERR_UNSUPPORTED, "plane-wave antennas solve in the FP64 form");
        n_solves += (int64_t)h.freqs.size() * (int64_t)std::max<size_t>(h.rhs_srcs.size(), 1);
    }
    if (n_solves > 65535) return fail(ctx, FNEC_ERR_TOO_LARGE, "a batch holds at most 65535 solves");
    fnec_batch *b = new fnec_batch();
    b->ctx = ctx;
    b->st = place.st ? place.st : ctx->stream;
    b->pooled = place.pooled;
    b->allow_grid = place.allow_grid;
    if (place.aux) {
        b->stage = place.aux->p;
        b->stage_cap = place.aux->cap;
    }
    b->precision = precision;
    b->from_wires = !hs.empty() && !hs[0].wires.empty();
    int64_t ff_req_max = 0, ff_int_max = 0;
    size_t smem_max = 0;
    std::map<std::tuple<int32_t, int32_t, double, double, double, double, int32_t, int>, DevRp> map_cache;
    for (size_t ai = 0; ai < hs.size(); ++ai) {
        HostAnt &h = hs[ai];
        AntDesc a{};
        a.seg_off = b->tot_seg;
        a.n = (int32_t)h.segs.size();
        a.w = (int32_t)h.cols();
        a.ground = h.ground;
        int n = a.n;
        // wires
        for (auto w : h.wires) {
            w.seg_off += b->tot_seg;
            b->wires.push_back(w);
        }
        if (!b->from_wires) b->segs.insert(b->segs.end(), h.segs.begin(), h.segs.end());
        // row_wire (linear.rs:728-733) and the CSR of rows per wire column
        std::vector<int32_t> row_wire(n, 0);
        for (size_t q = 0; q < h.ep.size(); ++q)
            for (int64_t r = h.ep[q].first; r <= h.ep[q].second; ++r) row_wire[r] = (int32_t)q;
        if (h.paths) row_wire = h.path_of;  // linear.rs:851-856: one column per path
        if (h.planewave)  // linear.rs:955-961: the cos column 2q, the sin column 2q + 1
            for (auto &c : row_wire) c *= 2;
        a.hom2 = h.planewave ? 1 : 0;
        a.rowwire_off = (int64_t)b->ibuf.size();
        b->ibuf.insert(b->ibuf.end(), row_wire.begin(), row_wire.end());
        std::vector<std::vector<int32_t>> rows_of(a.w);
        for (int r = 0; r < n; ++r) {
            rows_of[row_wire[r]].push_back(r);
            if (h.planewave) rows_of[row_wire[r] + 1].push_back(r);
        }
        int64_t ktab = 0;  // plane-wave form: each row's sin(k |s_m - s_p|) entries over its wire's rows
        if (h.planewave) {
            a.koff_off = (int64_t)b->ibuf.size();
            for (int r = 0; r < n; ++r) {
                b->ibuf.push_back((int32_t)ktab);
                ktab += (int64_t)rows_of[row_wire[r]].size();
            }
        }
        a.wptr_off = (int64_t)b->ibuf.size();
        int32_t acc = 0;
        b->ibuf.push_back(0);
        for (auto &v : rows_of) {
            acc += (int32_t)v.size();
            b->ibuf.push_back(acc);
        }
        a.wrow_off = (int64_t)b->ibuf.size();
        for (auto &v : rows_of) b->ibuf.insert(b->ibuf.end(), v.begin(), v.end());
        a.comp_off = (int64_t)b->ibuf.size();
        if (h.comp.empty()) h.comp.assign(2 * n, 0);
        b->ibuf.insert(b->ibuf.end(), h.comp.begin(), h.comp.end());
        // constraint rows (linear.rs:744-762): free endpoints first (first,
        // then last, per wire; skipping junction endpoints), then junctions.
        std::vector<char> injunc(n, 0);
        for (size_t t = 0; t < h.ja.size(); ++t) {
            injunc[h.ja[t]] = 1;
            injunc[h.jb[t]] = 1;
        }
        struct Ent {
            int64_t col;
            double val;
        };
        std::vector<std::vector<Ent>> crow;
        for (auto &e : h.ep) {
            if (!injunc[e.first]) crow.push_back({{e.first, 1.0}});
            if (!injunc[e.second]) crow.push_back({{e.second, 1.0}});
        }
        for (int64_t fe : h.free_ends) crow.push_back({{fe, 1.0}});  // linear.rs:859-864 (path form)
        for (size_t t = 0; t < h.ja.size(); ++t) {
            if (h.ja[t] == h.jb[t]) crow.push_back({{h.jb[t], h.js[t]}});
            else crow.push_back({{h.ja[t], 1.0}, {h.jb[t], h.js[t]}});
        }
        a.crow_off = (int64_t)b->crows.size();
        a.n_crow = (int32_t)crow.size();
        for (auto &r : crow) {
            DevConRow d{(int32_t)r[0].col, r.size() > 1 ? (int32_t)r[1].col : -1, r.size() > 1 ? r[1].val : 0.0};
            if (r.size() == 1 && r[0].val != 1.0) {  // a junction row with seg_a == seg_b
                d.c1 = d.c0;
                d.v1 = r[0].val - 1.0;
            }
            b->crows.push_back(d);
        }
        {
            // transpose: the constraint rows touching each segment column
            std::vector<std::vector<int32_t>> cc(a.n);
            for (int32_t q = 0; q < a.n_crow; ++q) {
                const DevConRow &d = b->crows[a.crow_off + q];
                cc[d.c0].push_back(q);
                if (d.c1 >= 0 && d.c1 != d.c0) cc[d.c1].push_back(q);
            }
            a.ccptr_off = (int64_t)b->ibuf.size();
            int32_t acc = 0;
            b->ibuf.push_back(0);
            for (auto &v : cc) b->ibuf.push_back(acc += (int32_t)v.size());
            a.ccq_off = (int64_t)b->ibuf.size();
            for (auto &v : cc) b->ibuf.insert(b->ibuf.end(), v.begin(), v.end());
        }
        struct Contrib {
            int64_t i, j, row;
            int32_t code;
        };
        std::vector<Contrib> cl;
        for (size_t r = 0; r < crow.size(); ++r)
            for (auto &u : crow[r])
                for (auto &v : crow[r]) cl.push_back({u.col, v.col, (int64_t)r, con_code(u.val, v.val)});
        std::stable_sort(cl.begin(), cl.end(), [](const Contrib &x, const Contrib &y) {
            return x.i != y.i ? x.i < y.i : (x.j != y.j ? x.j < y.j : x.row < y.row);
        });
        a.con_off = (int64_t)b->cons.size();
        a.conv_off = (int64_t)b->codes.size();
        int32_t base = 0;
        for (size_t q = 0; q < cl.size();) {
            size_t e = q;
            while (e < cl.size() && cl[e].i == cl[q].i && cl[e].j == cl[q].j) ++e;
            DevConstraint c{(int32_t)cl[q].i, (int32_t)cl[q].j, base, (int32_t)(e - q)};
            for (size_t t = q; t < e; ++t) b->codes.push_back(cl[t].code);
            base += (int32_t)(e - q);
            b->cons.push_back(c);
            q = e;
        }
        a.n_con = (int32_t)(b->cons.size() - a.con_off);
        // sources and feed rows, grouped by right-hand side (CSR in ibuf)
        if (h.rhs_srcs.empty()) {
            h.rhs_srcs.assign(1, {});
            h.rhs_feeds.assign(1, {});
        }
        a.n_rhs = (int32_t)h.rhs_srcs.size();
        a.src_off = (int64_t)b->srcs.size();
        a.feed_off = (int64_t)b->feeds.size();
        a.sptr_off = (int64_t)b->ibuf.size();
        int32_t cnt = 0;
        b->ibuf.push_back(0);
        for (auto &v : h.rhs_srcs) {
            b->srcs.insert(b->srcs.end(), v.begin(), v.end());
            cnt += (int32_t)v.size();
            b->ibuf.push_back(cnt);
        }
        a.n_src = cnt;
        a.fptr_off = (int64_t)b->ibuf.size();
        cnt = 0;
        b->ibuf.push_back(0);
        for (auto &v : h.rhs_feeds) {
            b->feeds.insert(b->feeds.end(), v.begin(), v.end());
            cnt += (int32_t)v.size();
            b->ibuf.push_back(cnt);
        }
        a.n_feed = cnt;
        a.run_off = (int64_t)b->runs.size();
        a.n_run = (int32_t)h.runs.size();
        b->runs.insert(b->runs.end(), h.runs.begin(), h.runs.end());
        DevRp rp = h.rp;
        if (!h.pts.empty()) {
            rp.pts_off = (int64_t)b->pts.size() / 2;
            rp.n_pts = (int32_t)(h.pts.size() / 2);
            b->pts.insert(b->pts.end(), h.pts.begin(), h.pts.end());
        }
        {
            // antennas with the same RP card and ground share one copy of the maps
            const bool card = rp.pts_off < 0;
            const auto key = std::make_tuple(rp.n_theta, rp.n_phi, rp.theta0, rp.phi0, rp.d_theta, rp.d_phi,
                                             rp.skip_integral, h.ground);
            auto hit = card ? map_cache.find(key) : map_cache.end();
            if (hit != map_cache.end()) {
                rp.i2r_off = hit->second.i2r_off;
                rp.xr_off = hit->second.xr_off;
                rp.n_xr = hit->second.n_xr;
            } else {
                std::vector<int32_t> i2r, xr;
                ff_cover_maps(rp, h.pts.data(), h.ground, i2r, xr);
                rp.i2r_off = (int64_t)b->ibuf.size();
                b->ibuf.insert(b->ibuf.end(), i2r.begin(), i2r.end());
                rp.xr_off = (int64_t)b->ibuf.size();
                b->ibuf.insert(b->ibuf.end(), xr.begin(), xr.end());
                rp.n_xr = (int32_t)xr.size();
                if (card) map_cache[key] = rp;
            }
        }
        b->rps.push_back(rp);
        int64_t n_req = rp.pts_off >= 0 ? rp.n_pts : (int64_t)rp.n_theta * rp.n_phi;
        int64_t n_int = rp.skip_integral ? 0 : (h.ground == 1 ? 91 : 181) * 360;
        ff_req_max = std::max(ff_req_max, n_req);
        ff_int_max = std::max(ff_int_max, n_int);
        smem_max = std::max(smem_max, sizeof(DevRun) * h.runs.size() + sizeof(cx) * (size_t)n);
        if (h.paths) a.paths = 1;
        if (!h.arc.empty()) {
            a.arc_off = (int64_t)b->pts.size();  // 2n doubles (n arc lengths, n signs): pairs stay aligned
            b->pts.insert(b->pts.end(), h.arc.begin(), h.arc.end());
        }
        if (h.planewave) {
            a.wave_off = (int64_t)b->pts.size();  // 10 doubles per direction: pairs stay aligned
            b->pts.insert(b->pts.end(), h.waves.begin(), h.waves.end());
            b->has_wave = true;
        }
        b->ants.push_back(a);
        b->max_w = std::max(b->max_w, (int)a.w);
        // systems (one per frequency) and their solves (one per right-hand side)
        int s = n + a.w;
        for (size_t fi = 0; fi < h.freqs.size(); ++fi) {
            double f = h.freqs[fi];
            UnitDesc u{};
            u.ant = (int32_t)ai;
            u.n = n;
            u.s = s;
            u.rhs = 0;
            u.freq = f;
            u.k_fill = 2.0 * PI * f / C0;
            u.k_rp = 2.0 * PI / (C0 / f);
            u.z_off = b->z_el;
            u.a_off = b->a_el;
            u.cos_off = b->cos_el;
            u.piv_off = b->piv_el;
            u.n_rhs = a.n_rhs;
            u.sys = (int32_t)b->units.size();
            if (need_solve && h.stamped()) {
                // this system's stamps in the reference's order: the LD loads on
                // the diagonal, then the TL and NT two-ports; runs per entry
                std::vector<Stamp> sv;
                if (!h.loads.empty()) {
                    std::vector<HC> lv;
                    segment_loads(h, f, lv);
                    for (int i = 0; i < n; ++i)
                        if (lv[i].re != 0.0 || lv[i].im != 0.0)  // adding an exact zero changes nothing
                            sv.push_back({i, i, lv[i]});
                }
                network_stamps(h, f, sv);
                std::stable_sort(sv.begin(), sv.end(), [](const Stamp &x, const Stamp &y) {
                    return x.row != y.row ? x.row < y.row : x.col < y.col;
                });
                for (size_t q = 0; q < sv.size();) {
                    size_t e = q;
                    while (e < sv.size() && sv[e].row == sv[q].row && sv[e].col == sv[q].col) ++e;
                    for (size_t t = q; t < e; ++t)
                        b->stamps.push_back(DevStamp{u.z_off + sv[t].row * n + sv[t].col, sv[t].v.re, sv[t].v.im,
                                                     t == q ? 1 : 0, t == q ? (int32_t)(e - q) : 0});
                    q = e;
                }
            }
            if (need_solve) {
                b->z_el += (int64_t)n * n;
                b->a_el += (int64_t)s * (s + 1);
            }
            b->cos_el += h.planewave ? 2 * (int64_t)n + ktab : n;
            b->piv_el += s;
            b->max_s = std::max(b->max_s, s);
            b->max_n = std::max(b->max_n, n);
            b->max_rhs = std::max(b->max_rhs, (int)a.n_rhs);
            int32_t uidx = u.sys;
            const int32_t first_solve = (int32_t)b->solves.size();
            for (int r0 = 1; r0 < a.n_rhs; r0 += 32)
                b->rhs_groups.push_back(make_int4(uidx, first_solve + r0, std::min(32, a.n_rhs - r0), 0));
            const int32_t *fptr = &b->ibuf[a.fptr_off];
            for (int r = 0; r < a.n_rhs; ++r) {
                UnitDesc v = u;
                v.rhs = r;
                v.x_off = b->x_el;
                v.rhs_off = b->rhs_el;
                v.pat_off = b->pat_el;
                if (r == 0) {  // the system points at its first right-hand side
                    u.x_off = v.x_off;
                    u.rhs_off = v.rhs_off;
                    u.pat_off = v.pat_off;
                }
                b->x_el += s;
                b->rhs_el += n;
                b->pat_el += n_req;
                int nf = fptr[r + 1] - fptr[r];
                fnec_unit_info ui{};
                ui.antenna = (uint32_t)ai;
                ui.n = (uint32_t)n;
                ui.s = (uint32_t)s;
                ui.n_feed = (uint32_t)nf;
                ui.n_points = (uint32_t)n_req;
                ui.freq_hz = f;
                ui.pat_off = (uint64_t)v.pat_off;
                ui.feed_off = (uint64_t)b->feed_rows;
                ui.cur_off = b->uinfo.empty() ? 0 : b->uinfo.back().cur_off + b->uinfo.back().n;
                ui.rhs = (uint32_t)r;
                ui.system = (uint32_t)uidx;
                b->feed_row_off.push_back(b->feed_rows);
                b->feed_rows += nf;
                b->uinfo.push_back(ui);
                b->recv_dirs.push_back(h.planewave ? h.dirs[2 * r] : std::nan(""));
                b->recv_dirs.push_back(h.planewave ? h.dirs[2 * r + 1] : std::nan(""));
                b->solves.push_back(v);
            }
            b->units.push_back(u);
            if (need_solve) {
                const int nt = (n + 15) / 16;
                b->fill_units.push_back(make_int4(uidx, nt, (int)b->n_fill, 0));
                b->n_fill += (int64_t)nt * nt;
                for (int i0 = 0; i0 < n; i0 += 64)
                    for (int j0 = 0; j0 <= n; j0 += 64) b->gram_tiles.push_back(make_int4(uidx, i0, j0, 0));
            }
            if (!h.z.empty()) b->z_given.insert(b->z_given.end(), h.z.begin(), h.z.end());
            if (h.rhs_given) {
                b->rhs_given_flag = true;
                b->rhs_given.insert(b->rhs_given.end(), h.rhs.begin(), h.rhs.end());
                b->cos_given.insert(b->cos_given.end(), h.cosv.begin(), h.cosv.end());
            }
        }
        b->tot_seg += n;
    }
    b->ff_blocks = farfield_max_blocks((int)ff_int_max, (int)ff_req_max);
    b->ff_smem = smem_max;
    int nu = (int)b->units.size();
    cudaError_t e = cudaSuccess;
    Packer pk;
    size_t o_wires = pk.add(b->wires), o_segs = pk.add(b->segs), o_ants = pk.add(b->ants),
           o_units = pk.add(b->units), o_solves = pk.add(b->solves), o_ibuf = pk.add(b->ibuf), o_srcs = pk.add(b->srcs),
           o_feeds = pk.add(b->feeds), o_cons = pk.add(b->cons), o_codes = pk.add(b->codes),
           o_runs = pk.add(b->runs), o_rps = pk.add(b->rps), o_pts = pk.add(b->pts),
           o_ft = pk.add(b->fill_units), o_crows = pk.add(b->crows), o_gt = pk.add(b->gram_tiles), o_fro = pk.add(b->feed_row_off),
           o_rhs = pk.add(b->rhs_given), o_cos = pk.add(b->cos_given), o_z = pk.add(b->z_given),
           o_st = pk.add(b->stamps), o_rg = pk.add(b->rhs_groups);
    b->in_bytes = pk.total > 0 ? pk.total : 256;
    const auto ta0 = std::chrono::steady_clock::now();
    if (b->pooled) {
        e = place.in->ensure(b->in_bytes);
        b->h_in = place.in->p;
        b->t_pinned += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - ta0).count();
    } else {
        e = pin_alloc((void **)&b->h_in, b->in_bytes);
    }
    if (e == cudaSuccess) e = dalloc(b, &b->d_in, b->in_bytes);
    if (e == cudaSuccess) {
        for (size_t q = 0; q < pk.parts.size(); ++q)
            if (pk.parts[q].second) std::memcpy(b->h_in + pk.offs[q], pk.parts[q].first, pk.parts[q].second);
        b->d_wires = (DevWire *)(b->d_in + o_wires);
        b->d_ants = (AntDesc *)(b->d_in + o_ants);
        b->d_units = (UnitDesc *)(b->d_in + o_units);
        b->d_solves = (UnitDesc *)(b->d_in + o_solves);
        b->d_ibuf = (int32_t *)(b->d_in + o_ibuf);
        b->d_srcs = (DevSource *)(b->d_in + o_srcs);
        b->d_feeds = (DevFeed *)(b->d_in + o_feeds);
        b->d_cons = (DevConstraint *)(b->d_in + o_cons);
        b->d_codes = (int32_t *)(b->d_in + o_codes);
        b->d_runs = (DevRun *)(b->d_in + o_runs);
        b->d_rps = (DevRp *)(b->d_in + o_rps);
        b->d_pts = (double *)(b->d_in + o_pts);
        b->d_fill_units = (int4 *)(b->d_in + o_ft);
        b->d_crows = (DevConRow *)(b->d_in + o_crows);
        b->d_gram_tiles = (int4 *)(b->d_in + o_gt);
        b->d_feed_row_off = (int64_t *)(b->d_in + o_fro);
        b->d_rhs_given = (double *)(b->d_in + o_rhs);
        b->d_cos_given = (double *)(b->d_in + o_cos);
        b->d_z_given = (double *)(b->d_in + o_z);
        b->d_stamps = (DevStamp *)(b->d_in + o_st);
        b->d_rhs_groups = (int4 *)(b->d_in + o_rg);
    }
    // segments: uploaded with the arena for caller-provided geometry,
    // expanded on the device from the wires otherwise
    if (!b->from_wires) b->d_segs = (DevSeg *)(b->d_in + o_segs);
#define DA(p, n)                                             \
    if (e == cudaSuccess) e = dalloc(b, &b->p, (size_t)(n));
    if (b->from_wires) DA(d_segs, b->tot_seg);
    DA(d_fill_tiles, b->n_fill);
    DA(d_z, b->z_el);
    DA(d_a, precision == FNEC_PRECISION_MIXED ? 1 : b->a_el);  // the mixed form factors in FP32
    DA(d_x, b->x_el);
    DA(d_rhs, b->rhs_el);
    DA(d_cos, b->cos_el);
    DA(d_piv, b->piv_el);
    DA(d_status, nu);
    DA(d_feed_out, 7 * b->feed_rows);
    DA(d_fld, 4 * b->pat_el);
    DA(d_partials, (int64_t)b->ff_blocks * (int64_t)b->solves.size());
    DA(d_pat, PAT_STRIDE * b->pat_el);
    DA(d_total, b->solves.size());
    DA(d_peak, b->has_wave ? b->solves.size() : 1);
    {
        int64_t tc = b->uinfo.empty() ? 0 : b->uinfo.back().cur_off + b->uinfo.back().n;
        std::vector<int64_t> co(b->uinfo.size());
        for (size_t u = 0; u < co.size(); ++u) co[u] = b->uinfo[u].cur_off;
        DA(d_cur, tc);
        DA(d_cur_off, co.size());
        if (e == cudaSuccess) e = up(b, b->d_cur_off, co);
    }
    {
        // grid-wide panels: units by s, tallest first
        std::vector<int32_t> &ord = b->grid_order;
        ord.resize(nu);
        for (int i = 0; i < nu; ++i) ord[i] = i;
        std::stable_sort(ord.begin(), ord.end(), [&](int32_t x, int32_t y) { return b->units[x].s > b->units[y].s; });
        b->grid.s_desc.resize(nu);
        for (int i = 0; i < nu; ++i) b->grid.s_desc[i] = b->units[ord[i]].s;
        b->grid.steps = (b->max_s + 31) / 32;
        cudaDeviceGetAttribute(&b->grid.sms, cudaDevAttrMultiProcessorCount, ctx->device);
        if (e == cudaSuccess) e = dalloc(b, &b->grid.d_order, (size_t)nu);
        if (e == cudaSuccess) e = up(b, b->grid.d_order, ord);
        if (b->max_s > 380 && b->allow_grid) {  // some panel may outgrow one CTA's shared memory
            unsigned char *xg = nullptr, *sy = nullptr;
            if (e == cudaSuccess) e = dalloc(b, &xg, grid_xchg_bytes());
            if (e == cudaSuccess) e = dalloc(b, &sy, grid_sync_bytes(b->grid.steps));
            b->grid.d_xchg = xg;
            b->grid.d_sync = sy;
        }
    }
#undef DA
    b->out_bytes = sizeof(cx) * (size_t)b->x_el + sizeof(double) * 7 * (size_t)b->feed_rows +
                   sizeof(double) * PAT_STRIDE * (size_t)b->pat_el +
                   (sizeof(int32_t) + sizeof(double)) * (size_t)(nu + b->solves.size()) + 64;
    if (e == cudaSuccess) {
        if (b->pooled) {
            const auto tp = std::chrono::steady_clock::now();
            e = place.out->ensure(b->out_bytes);
            b->h_out = place.out->p;
            b->t_pinned += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - tp).count();
        } else {
            e = pin_alloc((void **)&b->h_out, b->out_bytes);
        }
    }
    if (e == cudaSuccess && precision == FNEC_PRECISION_MIXED) {
        const auto tm = std::chrono::steady_clock::now();
        e = alloc_mixed(b->mixed, b->units, b->solves, b->ants, b->max_s,
                        DevAlloc{b->st, b->dev_pool, b->stage, b->stage_cap, &b->stage_used}, b->allow_grid);
        b->t_mixed += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - tm).count();
    }
    b->alloc_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - ta0).count();
    if (e == cudaSuccess && precision == FNEC_PRECISION_MIXED) {
        b->dev_bytes += b->mixed.bytes;
    }
    if (e != cudaSuccess) {
        free_batch(b);
        delete b;
        return fail(ctx, e == cudaErrorMemoryAllocation ? FNEC_ERR_OUT_OF_MEMORY : FNEC_ERR_CUDA,
                    std::string("batch allocation: ") + cudaGetErrorString(e));
    }
    *out = b;
    // the default for many systems: every unit up to S 512 factored whole,
    // one CTA each (enough of them to fill the GPU), and 4 refinement CTAs
    // per SM (more solves in flight)
    if (precision == FNEC_PRECISION_MIXED && (int64_t)b->units.size() >= 2 * (int64_t)b->grid.sms) {
        fnec_schedule s = b->sched;
        s.unit_factor = 3;
        if ((int64_t)b->solves.size() >= 8 * (int64_t)b->grid.sms) s.gmres_ctas_per_sm = 4;
        apply_schedule(b, s);
    }
    schedule_from_cache(b);
    int st = fnec_batch_upload(b);
    if (st != FNEC_OK) {
        free_batch(b);
        delete b;
        *out = nullptr;
        return st;
    }
    return FNEC_OK;
}

// planewave.rs:86-105 r_hat and pol_hat of one incidence direction, with the
// platform sin/cos as the reference calls them (this file is built without
// contraction): 10 doubles, r_hat[3], pol re[3], pol im[3], 0.
static void wave_vectors(uint32_t ex_type, double theta_deg, double phi_deg, double eta_deg, double ar_card,
                         double *out) {
    const double rad = PI / 180.0;  // f64::to_radians
    const double t = theta_deg * rad, p = phi_deg * rad, eta = eta_deg * rad;
    out[0] = std::sin(t) * std::cos(p);
    out[1] = std::sin(t) * std::sin(p);
    out[2] = std::cos(t);
    const double th[3] = {std::cos(t) * std::cos(p), std::cos(t) * std::sin(p), -std::sin(t)};
    const double ph[3] = {-std::sin(p), std::cos(p), 0.0};
    const double ce = std::cos(eta), se = std::sin(eta);
    double ar = 0.0, sense = 0.0;  // planewave.rs:62-67
    if (ex_type == 2) {
        ar = ar_card;
        sense = 1.0;
    } else if (ex_type == 3) {
        ar = ar_card;
        sense = -1.0;
    }
    const HC jminor{0.0, sense * ar};
    for (int i = 0; i < 3; ++i) {
        const double major = ce * th[i] + se * ph[i];
        const double minor = -se * th[i] + ce * ph[i];
        const HC v = hc_add({major, 0.0}, hc_scale(jminor, minor));
        out[3 + i] = v.re;
        out[6 + i] = v.im;
    }
    out[9] = 0.0;
}

// solve_session.rs:262-301 and :313-355: the receive form of a deck with a
// plane-wave EX card.  A non-trivial degree-2 conductor path takes the path
// form (build_planewave_hallen_paths); otherwise the per-tag wires, which
// must not touch (planewave.rs:176-180, detect_wire_junctions within 1e-6 m
// between ends of different segments).  The arc table carries the
// along-wire coordinate from each wire's geometric midpoint (sign 1).
static int plane_wave_form(const fnec_antenna &A, HostAnt &h, std::string &why) {
    const fnec_plane_wave &pw = *A.plane_wave;
    if (pw.ex_type < 1 || pw.ex_type > 3) {
        why = "plane wave: EX type must be 1, 2 or 3";
        return FNEC_ERR_BAD_ARG;
    }
    if (A.n_sources != 0) {
        why = "a plane-wave antenna takes no voltage sources";
        return FNEC_ERR_BAD_ARG;
    }
    if (h.segs.size() > 46340) {  // the sin(k |s_m - s_p|) table is indexed in int32
        why = "plane wave: at most 46340 segments";
        return FNEC_ERR_TOO_LARGE;
    }
    h.planewave = true;
    if (!conductor_paths(h)) {
        const auto wires = wire_endpoints(h.segs);
        for (size_t i = 0; i < 2 * wires.size(); ++i) {
            const int64_t si = i % 2 == 0 ? wires[i / 2].first : wires[i / 2].second;
            const double *pi = i % 2 == 0 ? h.segs[si].start : h.segs[si].end;
            for (size_t j = i + 1; j < 2 * wires.size(); ++j) {
                const int64_t sj = j % 2 == 0 ? wires[j / 2].first : wires[j / 2].second;
                if (si == sj) continue;
                const double *pj = j % 2 == 0 ? h.segs[sj].start : h.segs[sj].end;
                const double dx = pi[0] - pj[0], dy = pi[1] - pj[1], dz = pi[2] - pj[2];
                if (std::sqrt(dx * dx + dy * dy + dz * dz) <= 1e-6) {
                    why = "EX: incident plane wave is supported on straight, non-junctioned wires; junctioned "
                          "geometry is not yet supported";
                    return FNEC_ERR_UNSUPPORTED;
                }
            }
        }
        h.ep = wires;
        set_comp(h, wires);
        const int64_t n = (int64_t)h.segs.size();
        h.arc.assign(2 * n, 1.0);
        for (const auto &w : wires) {
            const double *a = h.segs[w.first].mid, *b = h.segs[w.second].mid, *dir = h.segs[w.first].dir;
            const double wm[3] = {(a[0] + b[0]) / 2.0, (a[1] + b[1]) / 2.0, (a[2] + b[2]) / 2.0};
            for (int64_t i = w.first; i <= w.second; ++i) {
                const double d[3] = {h.segs[i].mid[0] - wm[0], h.segs[i].mid[1] - wm[1], h.segs[i].mid[2] - wm[2]};
                h.arc[i] = d[0] * dir[0] + d[1] * dir[1] + d[2] * dir[2];
            }
        }
    }
    const uint32_t nt = std::max<uint32_t>(pw.n_theta, 1), np = std::max<uint32_t>(pw.n_phi, 1);
    const uint64_t nd = (uint64_t)nt * np;
    if (nd > 65535) {
        why = "plane wave: at most 65535 incidence directions";
        return FNEC_ERR_TOO_LARGE;
    }
    for (uint32_t it = 0; it < nt; ++it)
        for (uint32_t ip = 0; ip < np; ++ip) {
            // the first direction is the deck's own (theta0, phi0) as given
            const double th = it == 0 ? pw.theta0 : pw.theta0 + (double)it * pw.d_theta;
            const double ph = ip == 0 ? pw.phi0 : pw.phi0 + (double)ip * pw.d_phi;
            h.dirs.push_back(th);
            h.dirs.push_back(ph);
            double v[10];
            wave_vectors(pw.ex_type, th, ph, pw.eta, pw.axial_ratio, v);
            h.waves.insert(h.waves.end(), v, v + 10);
        }
    h.rhs_srcs.assign(nd, {});
    h.rhs_feeds.assign(nd, {});
    return FNEC_OK;
}

// HostAnt from GW/EX/RP cards: the CLI standard Hallen branch topology
// (solve_session.rs:1379-1400).
static int antenna_from_cards(const fnec_antenna &A, HostAnt &h, std::string &why) {
    if (A.n_wires == 0 || !A.wires) {
        why = "deck contains no GW (wire) cards";
        return FNEC_ERR_BAD_ARG;
    }
    if (A.ground != FNEC_GROUND_FREE && A.ground != FNEC_GROUND_PEC) {
        why = "ground must be free space or PEC";
        return FNEC_ERR_BAD_ARG;
    }
    if (A.n_freqs == 0 || !A.freqs_hz) {
        why = "no frequencies";
        return FNEC_ERR_BAD_ARG;
    }
    for (uint32_t f = 0; f < A.n_freqs; ++f)
        if (!std::isfinite(A.freqs_hz[f]) || !(A.freqs_hz[f] > 0.0)) {
            why = "frequency " + std::to_string(f) + " is not a finite positive number";
            return FNEC_ERR_BAD_ARG;
        }
    h.ground = A.ground;
    int64_t off = 0;
    for (uint32_t w = 0; w < A.n_wires; ++w) {
        const fnec_wire &gw = A.wires[w];
        if (gw.segments == 0) {
            why = "GW tag " + std::to_string(gw.tag) + ": segment count must be >= 1";
            return FNEC_ERR_BAD_ARG;
        }
        // a NaN or infinite coordinate or radius is refused here, at the
        // boundary, so that no kernel sees it
        bool finite = std::isfinite(gw.radius);
        for (int c = 0; c < 3; ++c) finite = finite && std::isfinite(gw.start[c]) && std::isfinite(gw.end[c]);
        if (!finite) {
            why = "GW tag " + std::to_string(gw.tag) + ": non-finite coordinate or radius";
            return FNEC_ERR_BAD_ARG;
        }
        double dx = gw.end[0] - gw.start[0], dy = gw.end[1] - gw.start[1], dz = gw.end[2] - gw.start[2];
        if (std::sqrt(dx * dx + dy * dy + dz * dz) == 0.0) {
            why = "GW tag " + std::to_string(gw.tag) + ": wire has zero length";
            return FNEC_ERR_BAD_ARG;
        }
        DevWire d{};
        for (int c = 0; c < 3; ++c) {
            d.start[c] = gw.start[c];
            d.end[c] = gw.end[c];
        }
        d.radius = gw.radius;
        d.tag = gw.tag;
        d.nseg = gw.segments;
        d.seg_off = off;
        for (uint32_t i = 0; i < gw.segments; ++i) h.segs.push_back(host_seg(gw, i));
        d.self_log = h.segs.back().self_log;
        h.wires.push_back(d);
        off += gw.segments;
    }
    auto merged = merge_collinear(h.segs);
    set_comp(h, merged);
    if (A.plane_wave) {
        int st = plane_wave_form(A, h, why);
        if (st != FNEC_OK) return st;
    } else if (!conductor_paths(h)) {  // the standard branch (solve_session.rs:1379-1400)
        h.ep = merged;
        cli_junctions(h.segs, merged, h);
    }
    int st = A.plane_wave ? FNEC_OK : resolve_sources(h, A.sources, A.n_sources, A.separate_sources != 0, why);
    if (st != FNEC_OK) return st;
    build_runs(h);
    h.rp.pts_off = -1;
    if (A.rp_points && A.n_rp_points > 0) {
        if (A.rp) {
            why = "rp and rp_points are exclusive";
            return FNEC_ERR_BAD_ARG;
        }
        h.pts.assign(A.rp_points, A.rp_points + 2 * (size_t)A.n_rp_points);
    } else if (A.rp) {
        h.rp.n_theta = (int32_t)std::max<uint32_t>(A.rp->n_theta, 1);
        h.rp.n_phi = (int32_t)std::max<uint32_t>(A.rp->n_phi, 1);
        h.rp.theta0 = A.rp->theta0;
        h.rp.phi0 = A.rp->phi0;
        h.rp.d_theta = A.rp->d_theta;
        h.rp.d_phi = A.rp->d_phi;
    } else {
        h.rp.n_theta = 0;
        h.rp.n_phi = 0;
        h.rp.skip_integral = 1;
    }
    h.freqs.assign(A.freqs_hz, A.freqs_hz + A.n_freqs);
    if (A.n_loads > 0) {
        if (!A.loads) {
            why = "n_loads > 0 without loads";
            return FNEC_ERR_BAD_ARG;
        }
        h.loads.assign(A.loads, A.loads + A.n_loads);
    }
    if ((A.n_tls > 0 && !A.tls) || (A.n_nts > 0 && !A.nts)) {
        why = "n_tls / n_nts > 0 without their cards";
        return FNEC_ERR_BAD_ARG;
    }
    if (A.n_tls > 0) h.tls.assign(A.tls, A.tls + A.n_tls);
    if (A.n_nts > 0) h.nts.assign(A.nts, A.nts + A.n_nts);
    return FNEC_OK;
}

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" {

int fnec_ctx_create(int device, fnec_ctx **out) {
    if (!out) return FNEC_ERR_BAD_ARG;
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) return FNEC_ERR_NO_DEVICE;
    if (device < 0 || device >= count) return FNEC_ERR_BAD_ARG;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return FNEC_ERR_NO_DEVICE;
    if (prop.major != 10) return FNEC_ERR_NO_DEVICE;  // built for sm_100a only
    if (cudaSetDevice(device) != cudaSuccess) return FNEC_ERR_CUDA;
    fnec_ctx *c = new fnec_ctx();
    c->device = device;
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete c;
        return FNEC_ERR_CUDA;
    }
    // batches allocate from the device's stream-ordered pool: keep what a
    // destroyed batch frees there for the next batch (unmapping and mapping
    // device memory again costs tens of milliseconds for a large batch);
    // fnec_device_cache_release gives it back
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
        uint64_t keep = UINT64_MAX;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    *out = c;
    return FNEC_OK;
}

int fnec_device_cache_release(fnec_ctx *ctx, uint64_t *released) {
    if (!ctx) return FNEC_ERR_BAD_ARG;
    if (released) *released = 0;
    cudaSetDevice(ctx->device);
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, ctx->device) != cudaSuccess) return FNEC_ERR_CUDA;
    if (cudaStreamSynchronize(ctx->stream) != cudaSuccess) return FNEC_ERR_CUDA;
    uint64_t before = 0, after = 0;
    cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &before);
    if (cudaMemPoolTrimTo(pool, 0) != cudaSuccess) return FNEC_ERR_CUDA;
    cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &after);
    if (released) *released = before > after ? before - after : 0;
    return FNEC_OK;
}

int fnec_ctx_destroy(fnec_ctx *ctx) {
    if (!ctx) return FNEC_ERR_BAD_ARG;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    cudaStreamDestroy(ctx->stream);
    delete ctx;
    return FNEC_OK;
}

const char *fnec_ctx_last_error(const fnec_ctx *ctx) { return ctx ? ctx->err.c_str() : ""; }

void *fnec_ctx_stream(fnec_ctx *ctx) { return ctx ? (void *)ctx->stream : nullptr; }

int fnec_batch_create(fnec_ctx *ctx, const fnec_antenna *antennas, uint32_t n_antennas,
                      int32_t precision, fnec_batch **out) {
    if (!ctx || !out || (!antennas && n_antennas)) return FNEC_ERR_BAD_ARG;
    *out = nullptr;
    if (precision != FNEC_PRECISION_FP64 && precision != FNEC_PRECISION_MIXED)
        return fail(ctx, FNEC_ERR_BAD_ARG, "unknown precision");
    if (precision == FNEC_PRECISION_MIXED && !mixed_available())
        return fail(ctx, FNEC_ERR_UNSUPPORTED, "mixed precision path not built");
    cudaSetDevice(ctx->device);
    const auto tc0 = std::chrono::steady_clock::now();
    std::vector<HostAnt> hs(n_antennas);
    // each antenna's host planning (segments, topology, junctions, sources)
    // is independent: spread over host threads for large batches
    std::vector<int> st_of(n_antennas, FNEC_OK);
    std::vector<std::string> why_of(n_antennas);
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    const unsigned nt = n_antennas >= 256 ? std::min(hw, 16u) : 1u;
    auto work = [&](unsigned k) {
        for (uint32_t a = k; a < n_antennas; a += nt) st_of[a] = antenna_from_cards(antennas[a], hs[a], why_of[a]);
    };
    if (nt > 1) {
        std::vector<std::thread> pool;
        for (unsigned k = 1; k < nt; ++k) pool.emplace_back(work, k);
        work(0);
        for (auto &t : pool) t.join();
    } else {
        work(0);
    }
    for (uint32_t a = 0; a < n_antennas; ++a)
        if (st_of[a] != FNEC_OK) return fail(ctx, st_of[a], "antenna " + std::to_string(a) + ": " + why_of[a]);
    const double ant_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - tc0).count();
    const int rc = build_batch(ctx, hs, precision, out);
    if (rc == FNEC_OK && *out) {
        (*out)->antennas_ms = ant_ms;
        (*out)->create_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - tc0).count();
    }
    return rc;
}

int fnec_batch_destroy(fnec_batch *b) {
    if (!b) return FNEC_ERR_BAD_ARG;
    cudaSetDevice(b->ctx->device);
    cudaStreamSynchronize(b->st);
    free_batch(b);
    delete b;
    return FNEC_OK;
}

int fnec_batch_get_info(const fnec_batch *b, fnec_batch_info *out) {
    if (!b || !out) return FNEC_ERR_BAD_ARG;
    out->n_units = (uint32_t)b->solves.size();
    out->n_systems = (uint32_t)b->units.size();
    out->max_s = (uint32_t)b->max_s;
    out->total_currents = b->uinfo.empty() ? 0 : b->uinfo.back().cur_off + b->uinfo.back().n;
    out->total_feeds = (uint64_t)b->feed_rows;
    out->total_points = (uint64_t)b->pat_el;
    out->device_bytes = b->dev_bytes;
    out->h2d_bytes = b->h2d;
    out->kernel_launches = b->launches;
    out->create_ms = b->create_ms;
    out->antennas_ms = b->antennas_ms;
    out->alloc_ms = b->alloc_ms;
    out->alloc_device_ms = b->t_dev;
    out->alloc_pinned_ms = b->t_pinned;
    out->alloc_mixed_ms = b->t_mixed;
    return FNEC_OK;
}

int fnec_batch_get_unit_info(const fnec_batch *b, uint32_t unit, fnec_unit_info *out) {
    if (!b || !out || unit >= b->uinfo.size()) return FNEC_ERR_BAD_ARG;
    *out = b->uinfo[unit];
    return FNEC_OK;
}

// Entry q of the fill list covers unit fu.x with fu.y tiles per side from
// tile fu.z on: tile fu.z + i fu.y + j is (unit, 16 i, 16 j) -- the list the
// host would otherwise upload, formed in place.
__global__ void k_fill_tile_list(const int4 *__restrict__ fill_units, int4 *tiles) {
    const int4 fu = fill_units[blockIdx.y];
    const int64_t cnt = (int64_t)fu.y * fu.y;
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < cnt; k += (int64_t)gridDim.x * blockDim.x)
        tiles[fu.z + k] = make_int4(fu.x, (int)(k / fu.y) * 16, (int)(k % fu.y) * 16, 0);
}

int fnec_batch_upload(fnec_batch *b) {
    if (!b) return FNEC_ERR_BAD_ARG;
    fnec_ctx *ctx = b->ctx;
    cudaSetDevice(ctx->device);
    // one pinned host -> device copy of every input table
    b->h2d = b->in_bytes;
    CUDA_TRY(ctx, cudaMemcpyAsync(b->d_in, b->h_in, b->in_bytes, cudaMemcpyHostToDevice, b->st));
    if (!b->fill_units.empty()) {  // the 16x16 fill tiles, from each unit's tiles per side
        k_fill_tile_list<<<dim3(64, (unsigned)b->fill_units.size()), 256, 0, b->st>>>(b->d_fill_units, b->d_fill_tiles);
        CUDA_TRY(ctx, cudaPeekAtLastError());
    }
    if (!b->z_given.empty())
        CUDA_TRY(ctx, cudaMemcpyAsync(b->d_z, b->d_z_given, sizeof(double) * b->z_given.size(),
                                      cudaMemcpyDeviceToDevice, b->st));
    if (b->rhs_given_flag) {
        CUDA_TRY(ctx, cudaMemcpyAsync(b->d_rhs, b->d_rhs_given, sizeof(double) * b->rhs_given.size(),
                                      cudaMemcpyDeviceToDevice, b->st));
        CUDA_TRY(ctx, cudaMemcpyAsync(b->d_cos, b->d_cos_given, sizeof(double) * b->cos_given.size(),
                                      cudaMemcpyDeviceToDevice, b->st));
    }
    return FNEC_OK;
}

// Enqueue the pipeline's launches on the batch stream (eagerly, or into
// the graph being captured on it).
// The report's pattern columns (gain_total, gain_theta, gain_phi, axial
// ratio) of every point, packed from the 6-column rows into 4.
__global__ void k_pack_report(const double *__restrict__ pat, int64_t n_points, double *__restrict__ out) {
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < 4 * n_points;
         t += (int64_t)gridDim.x * blockDim.x)
        out[t] = pat[PAT_STRIDE * (t / 4) + t % 4];
}


static int run_pipeline(fnec_batch *b) {
    fnec_ctx *ctx = b->ctx;
    cudaStream_t st = b->st;
    int nu = (int)b->units.size();
    int ns = (int)b->solves.size();
    uint64_t L = 0;
    if (nu == 0) return FNEC_OK;
    auto mark = [&](int k) {
        if (b->profile) cudaEventRecord(b->ev[k], st);
    };
    const char *failed = nullptr;  // the first phase whose launches failed
    std::string detail;
    auto check = [&](const char *phase) {
        if (!failed && cudaPeekAtLastError() != cudaSuccess) failed = phase;
    };
    {
        cudaError_t pre = cudaGetLastError();
        if (pre != cudaSuccess)
            return fail(ctx, FNEC_ERR_CUDA, std::string("an earlier call left an error: ") + cudaGetErrorString(pre));
    }
    CUDA_TRY(ctx, cudaMemsetAsync(b->d_status, 0, sizeof(int32_t) * nu, st));
    CUDA_TRY(ctx, cudaMemsetAsync(b->d_total, 0, sizeof(double) * ns, st));
    mark(0);
    if (b->from_wires) {
        launch_expand_segments(b->d_wires, (int)b->wires.size(), b->d_segs, st);
        ++L;
    }
    mark(1);
    if (!b->rhs_given_flag) {
        const double MU0 = 4.0 * PI * 1e-7;
        const double ETA0 = MU0 * C0;
        launch_hallen_rhs(b->d_solves, ns, b->d_ants, b->d_segs, b->d_ibuf, b->d_srcs, b->d_pts, b->d_rhs, b->d_cos,
                          2.0 * PI / ETA0, st);
        ++L;
        if (b->has_wave) {
            launch_planewave_rhs(b->d_solves, ns, b->max_n, b->d_ants, b->d_segs, b->d_ibuf, b->d_pts, b->d_x,
                                 b->d_rhs, b->d_cos, 2.0 * PI / ETA0, st);
            L += 2;
        }
    }
    mark(2);
    if (b->precision == FNEC_PRECISION_MIXED) {
        check("segments and right-hand sides");
        MixedMarks mm{b->profile ? &b->ev[3] : nullptr};
        L += run_mixed(b->mixed, b->d_units, nu, b->d_solves, ns, b->d_ants, b->d_segs, b->d_fill_tiles,
                       (int)b->n_fill, b->d_gram_tiles, (int)b->gram_tiles.size(), b->d_ibuf,
                       b->d_crows, b->d_z, b->d_rhs, b->d_cos, b->d_x, b->d_piv, b->d_status, b->max_s,
                       b->z_given.empty(), b->max_w, b->grid, mm, st, b->d_stamps, (int)b->stamps.size());
        if (!failed && mm.failed_phase) failed = mm.failed_phase;
        if (mm.detail[0]) detail = mm.detail;
    } else {
        if (b->z_given.empty()) {
            launch_fill_exact(b->d_units, b->d_ants, b->d_segs, b->d_fill_tiles, (int)b->n_fill,
                              b->d_z, st);
            ++L;
            if (!b->stamps.empty()) {
                launch_stamps(b->d_stamps, (int)b->stamps.size(), b->d_z, st);
                ++L;
            }
        }
        mark(3);
        launch_gram_exact(b->d_units, nu, b->max_w, b->d_ants, b->d_gram_tiles, (int)b->gram_tiles.size(), b->d_ibuf,
                          b->d_cons, b->d_codes, b->d_z, b->d_rhs, b->d_cos, b->d_a, st);
        mark(4);
        L += launch_factor_exact(b->d_units, nu, b->max_s, b->grid, b->d_a, b->d_piv, b->d_status, st);
        mark(5);
        // many right-hand sides per factorisation (receive sweeps): the grouped
        // kernels, with the first right-hand sides' back substitution beside
        // them on the side stream (they read the same factor, write other x)
        const bool grouped = b->max_rhs >= 8;
        bool forked = false;
        if (grouped) {
            if (!b->side && (cudaStreamCreateWithFlags(&b->side, cudaStreamNonBlocking) != cudaSuccess ||
                             cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
                             cudaEventCreateWithFlags(&b->ev_join, cudaEventDisableTiming) != cudaSuccess)) {
                (void)cudaGetLastError();  // no side stream: both run on st
            }
            forked = b->side && b->ev_fork && b->ev_join && cudaEventRecord(b->ev_fork, st) == cudaSuccess &&
                     cudaStreamWaitEvent(b->side, b->ev_fork, 0) == cudaSuccess;
        }
        launch_backsub(b->d_units, nu, b->max_s, b->d_a, b->d_x, b->d_status, forked ? b->side : st);
        if (b->max_rhs > 1) {
            launch_extra_rhs_exact(b->d_solves, ns, b->max_s, b->d_ants, b->d_ibuf, b->d_z, b->d_rhs, b->d_cos,
                                   b->d_a, b->d_piv, b->d_x, b->d_status, st, grouped ? b->d_rhs_groups : nullptr,
                                   grouped ? (int)b->rhs_groups.size() : 0);
            L += 2;
        }
        if (forked) {
            cudaEventRecord(b->ev_join, b->side);
            cudaStreamWaitEvent(st, b->ev_join, 0);
        }
        mark(6);
        L += 3 + 1;  // Gram (3 kernels) and the back substitution
        check("fill, Gram, factor and solve");
    }
    launch_feedpoints(b->d_solves, ns, b->d_ants, b->d_segs, b->d_ibuf, b->d_feeds, b->d_x, b->d_status,
                      b->d_feed_out, b->d_feed_row_off, st);
    ++L;
    if (b->has_wave) {
        launch_receive_peaks(b->d_solves, ns, b->d_ants, b->d_x, b->d_status, b->d_peak, st);
        ++L;
    }
    check("feedpoints");
    mark(7);
    if (b->ff_blocks > 0) {
        // with a report sink the far field runs in chunks of solves, each
        // chunk's report columns packed and copied on the copy stream while
        // the next chunk computes (the kernels index solves, partials and
        // totals by the launch's own solve index)
        constexpr int K_CHUNKS = 8;
        bool chunked = false;
        if (b->sink) {
            if (!b->copy_st) {
                bool ok = cudaStreamCreateWithFlags(&b->copy_st, cudaStreamNonBlocking) == cudaSuccess &&
                          cudaEventCreateWithFlags(&b->ev_copy, cudaEventDisableTiming) == cudaSuccess;
                for (int k = 0; ok && k < K_CHUNKS; ++k) {
                    cudaEvent_t e = nullptr;
                    ok = cudaEventCreateWithFlags(&e, cudaEventDisableTiming) == cudaSuccess;
                    if (ok) b->ev_chunk.push_back(e);
                }
                if (!ok) (void)cudaGetLastError();
            }
            chunked = b->copy_st && b->ev_copy && (int)b->ev_chunk.size() == K_CHUNKS;
        }
        const int k_n = chunked ? std::min(ns, K_CHUNKS) : 1, cs = (ns + k_n - 1) / k_n;
        for (int s0 = 0, k = 0; s0 < ns; s0 += cs, ++k) {
            const int s1 = std::min(ns, s0 + cs);
            launch_farfield(b->d_solves + s0, s1 - s0, b->d_ants, b->d_runs, b->d_rps, b->d_pts, b->d_ibuf, b->d_x,
                            b->d_status, b->d_fld, b->d_partials + (int64_t)s0 * b->ff_blocks, b->ff_blocks, b->ff_smem,
                            b->d_pat, b->d_total + s0, st);
            L += 2;
            if (chunked) {
                const int64_t p0 = (int64_t)b->uinfo[s0].pat_off;
                const int64_t p1 = (int64_t)b->uinfo[s1 - 1].pat_off + b->uinfo[s1 - 1].n_points;
                if (p1 > p0) {
                    cudaEventRecord(b->ev_chunk[k], st);
                    cudaStreamWaitEvent(b->copy_st, b->ev_chunk[k], 0);
                    // the chunk's field scratch is dead after its gains: the packed rows go there
                    k_pack_report<<<(int)std::min<int64_t>((4 * (p1 - p0) + 255) / 256, 148 * 16), 256, 0,
                                    b->copy_st>>>(b->d_pat + PAT_STRIDE * p0, p1 - p0, b->d_fld + 4 * p0);
                    cudaMemcpyAsync(b->sink + 4 * p0, b->d_fld + 4 * p0, sizeof(double) * 4 * (p1 - p0),
                                    cudaMemcpyDeviceToHost, b->copy_st);
                    ++L;
                }
            }
        }
        if (chunked) {
            cudaEventRecord(b->ev_copy, b->copy_st);
            cudaStreamWaitEvent(st, b->ev_copy, 0);
        }
    }
    mark(8);
    check("far field");
    b->launches = L;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess)
        return fail(ctx, FNEC_ERR_CUDA, std::string(failed ? failed : "run") + ": " + cudaGetErrorString(e) +
                                            (detail.empty() ? "" : " [" + detail + "]"));
    return FNEC_OK;
}

// Capture the pipeline from the batch stream into a graph.  Capture may be
// refused (a launch form the driver does not record); the batch then keeps
// launching eagerly and says why.
static void capture_pipeline(fnec_batch *b) {
    fnec_ctx *ctx = b->ctx;
    const std::string saved = ctx->err;
    cudaStream_t st = b->st;
    cudaError_t e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) {
        (void)cudaGetLastError();
        b->graph_state = FNEC_GRAPH_FAILED;
        b->graph_why = std::string("begin capture: ") + cudaGetErrorString(e);
        return;
    }
    int rc = run_pipeline(b);
    cudaGraph_t g = nullptr;
    e = cudaStreamEndCapture(st, &g);
    cudaGraphExec_t ex = nullptr;
    std::string why;
    if (rc != FNEC_OK) why = "capture: " + ctx->err;
    else if (e != cudaSuccess || !g) why = std::string("end capture: ") + cudaGetErrorString(e);
    else if ((e = cudaGraphInstantiateWithFlags(&ex, g, 0)) != cudaSuccess)
        why = std::string("instantiate: ") + cudaGetErrorString(e);
    if (g) cudaGraphDestroy(g);
    if (!why.empty() || !ex) {
        (void)cudaGetLastError();
        if (ex) cudaGraphExecDestroy(ex);
        ctx->err = saved;
        b->graph_state = FNEC_GRAPH_FAILED;
        b->graph_why = why;
        return;
    }
    b->gexec = ex;
    b->graph_state = FNEC_GRAPH_READY;
    b->graph_launches = b->launches;
}

static void drop_graph(fnec_batch *b) {
    if (b->gexec) cudaGraphExecDestroy(b->gexec);
    b->gexec = nullptr;
    b->graph_state = FNEC_GRAPH_NONE;
    b->graph_why.clear();
}

int fnec_batch_run(fnec_batch *b) {
    if (!b) return FNEC_ERR_BAD_ARG;
    fnec_ctx *ctx = b->ctx;
    cudaSetDevice(ctx->device);
    if (b->units.empty()) return FNEC_OK;
    const bool graph = b->sched.graph != 0 && !b->profile && b->graph_state != FNEC_GRAPH_FAILED &&
                       (b->sched.graph == 2 || b->n_runs >= 1);
    ++b->n_runs;
    if (!graph) return run_pipeline(b);
    if (!b->gexec) {
        cudaError_t pre = cudaGetLastError();
        if (pre != cudaSuccess)
            return fail(ctx, FNEC_ERR_CUDA, std::string("an earlier call left an error: ") + cudaGetErrorString(pre));
        capture_pipeline(b);
        if (!b->gexec) return run_pipeline(b);
    }
    CUDA_TRY(ctx, cudaGraphLaunch(b->gexec, b->st));
    b->launches = b->graph_launches;
    return FNEC_OK;
}

// ---- resident systems: new voltage sources on the stored factorisation ----

// The voltage sources of one antenna of a batch that has run: resolved on
// the host against the antenna's own segments (excitation.rs:119-187, the
// same resolution as at planning) and written into the batch's source and
// feed tables, host and device.  The new cards must give every right-hand
// side the planned numbers of resolved sources and feed rows.
int fnec_batch_set_sources(fnec_batch *b, uint32_t antenna, const fnec_source *sources, uint32_t n_sources) {
    if (!b || (!sources && n_sources)) return FNEC_ERR_BAD_ARG;
    fnec_ctx *ctx = b->ctx;
    if (antenna >= b->ants.size()) return fail(ctx, FNEC_ERR_BAD_ARG, "set_sources: no such antenna");
    const AntDesc &a = b->ants[antenna];
    if (a.hom2) return fail(ctx, FNEC_ERR_BAD_ARG, "set_sources: a receiving (plane-wave) antenna has no sources");
    if (b->rhs_given_flag || !b->from_wires)
        return fail(ctx, FNEC_ERR_BAD_ARG, "set_sources: the batch was planned from segments and given right-hand sides");
    // the antenna's GW cards, as planned
    std::vector<fnec_wire> wires;
    for (const DevWire &d : b->wires)
        if (d.seg_off >= a.seg_off && d.seg_off < a.seg_off + a.n) {
            fnec_wire w{};
            w.tag = d.tag;
            w.segments = d.nseg;
            for (int c = 0; c < 3; ++c) {
                w.start[c] = d.start[c];
                w.end[c] = d.end[c];
            }
            w.radius = d.radius;
            wires.push_back(w);
        }
    const double f1 = 1.0e6;
    fnec_antenna A{};
    A.wires = wires.data();
    A.n_wires = (uint32_t)wires.size();
    A.sources = sources;
    A.n_sources = n_sources;
    A.ground = a.ground;
    A.n_freqs = 1;
    A.freqs_hz = &f1;
    A.separate_sources = a.n_rhs > 1 ? 1u : 0u;
    HostAnt h;
    std::string why;
    int st = antenna_from_cards(A, h, why);
    if (st != FNEC_OK) return fail(ctx, st, "set_sources: " + why);
    if (h.rhs_srcs.empty()) {
        h.rhs_srcs.assign(1, {});
        h.rhs_feeds.assign(1, {});
    }
    if ((int)h.rhs_srcs.size() != a.n_rhs)
        return fail(ctx, FNEC_ERR_BAD_ARG, "set_sources: the planned antenna has " + std::to_string(a.n_rhs) +
                                                " right-hand sides, the new sources give " +
                                                std::to_string(h.rhs_srcs.size()));
    const int32_t *sptr = b->ibuf.data() + a.sptr_off, *fptr = b->ibuf.data() + a.fptr_off;
    for (int r = 0; r < a.n_rhs; ++r)
        if ((int)h.rhs_srcs[r].size() != sptr[r + 1] - sptr[r] || (int)h.rhs_feeds[r].size() != fptr[r + 1] - fptr[r])
            return fail(ctx, FNEC_ERR_BAD_ARG,
                        "set_sources: right-hand side " + std::to_string(r) +
                            " needs the planned numbers of resolved sources and feed rows (EX cards)");
    for (int r = 0; r < a.n_rhs; ++r) {
        std::copy(h.rhs_srcs[r].begin(), h.rhs_srcs[r].end(), b->srcs.begin() + a.src_off + sptr[r]);
        std::copy(h.rhs_feeds[r].begin(), h.rhs_feeds[r].end(), b->feeds.begin() + a.feed_off + fptr[r]);
    }
    // the packed input arena mirrors the tables: keep both copies current
    cudaSetDevice(ctx->device);
    const size_t so = (size_t)((unsigned char *)(b->d_srcs + a.src_off) - b->d_in);
    const size_t fo = (size_t)((unsigned char *)(b->d_feeds + a.feed_off) - b->d_in);
    const size_t sb = sizeof(DevSource) * (size_t)a.n_src, fb = sizeof(DevFeed) * (size_t)a.n_feed;
    if (sb) std::memcpy(b->h_in + so, b->srcs.data() + a.src_off, sb);
    if (fb) std::memcpy(b->h_in + fo, b->feeds.data() + a.feed_off, fb);
    if (sb) CUDA_TRY(ctx, cudaMemcpyAsync(b->d_in + so, b->h_in + so, sb, cudaMemcpyHostToDevice, b->st));
    if (fb) CUDA_TRY(ctx, cudaMemcpyAsync(b->d_in + fo, b->h_in + fo, fb, cudaMemcpyHostToDevice, b->st));
    return FNEC_OK;
}

// Every solve of the batch again on the factorisations of its last run:
// the right-hand sides of the current sources, then the plain form's
// substitution on the stored factor (the elimination replayed for each
// right-hand side, bit-identical to a fresh solve) or the mixed form's
// refinement on the stored preconditioner, the feedpoints and the pattern.
// Fill, normal equations and factorisation do not run.
int fnec_batch_resolve(fnec_batch *b) {
    if (!b) return FNEC_ERR_BAD_ARG;
    fnec_ctx *ctx = b->ctx;
    cudaSetDevice(ctx->device);
    if (b->units.empty()) return FNEC_OK;
    if (b->n_runs == 0) return fail(ctx, FNEC_ERR_BAD_ARG, "resolve: the batch has not run (no factorisation yet)");
    if (b->has_wave || b->rhs_given_flag)
        return fail(ctx, FNEC_ERR_BAD_ARG, "resolve: receiving antennas and given right-hand sides are not re-solved");
    {
        cudaError_t pre = cudaGetLastError();
        if (pre != cudaSuccess)
            return fail(ctx, FNEC_ERR_CUDA, std::string("an earlier call left an error: ") + cudaGetErrorString(pre));
    }
    cudaStream_t st = b->st;
    const int nu = (int)b->units.size(), ns = (int)b->solves.size();
    uint64_t L = 0;
    const double MU0 = 4.0 * PI * 1e-7;
    const double ETA0 = MU0 * C0;
    // the factor's status words stay: a singular system stays flagged
    CUDA_TRY(ctx, cudaMemsetAsync(b->d_total, 0, sizeof(double) * ns, st));
    launch_hallen_rhs(b->d_solves, ns, b->d_ants, b->d_segs, b->d_ibuf, b->d_srcs, b->d_pts, b->d_rhs, b->d_cos,
                      2.0 * PI / ETA0, st);
    ++L;
    if (b->precision == FNEC_PRECISION_MIXED) {
        MixedMarks mm{nullptr};
        L += refine_mixed(b->mixed, b->d_units, nu, b->d_solves, ns, b->d_ants, b->d_ibuf, b->d_crows, b->d_z,
                          b->d_rhs, b->d_cos, b->d_x, b->d_piv, b->d_status, b->max_s, mm, st, false);
    } else {
        launch_extra_rhs_exact(b->d_solves, ns, b->max_s, b->d_ants, b->d_ibuf, b->d_z, b->d_rhs, b->d_cos, b->d_a,
                               b->d_piv, b->d_x, b->d_status, st, nullptr, 0, 0);
        L += 2;
    }
    launch_feedpoints(b->d_solves, ns, b->d_ants, b->d_segs, b->d_ibuf, b->d_feeds, b->d_x, b->d_status,
                      b->d_feed_out, b->d_feed_row_off, st);
    ++L;
    if (b->ff_blocks > 0) {
        launch_farfield(b->d_solves, ns, b->d_ants, b->d_runs, b->d_rps, b->d_pts, b->d_ibuf, b->d_x, b->d_status,
                        b->d_fld, b->d_partials, b->ff_blocks, b->ff_smem, b->d_pat, b->d_total, st);
        L += 2;
    }
    b->launches = L;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(ctx, FNEC_ERR_CUDA, std::string("resolve: ") + cudaGetErrorString(e));
    return FNEC_OK;
}

int fnec_batch_set_profiling(fnec_batch *b, int on) {
    if (!b) return FNEC_ERR_BAD_ARG;
    cudaSetDevice(b->ctx->device);
    if (on && !b->ev_made) {
        for (auto &e : b->ev) CUDA_TRY(b->ctx, cudaEventCreate(&e));
        b->ev_made = true;
    }
    b->profile = on != 0;
    return FNEC_OK;
}

int fnec_batch_phase_ms(fnec_batch *b, double *ms) {
    if (!b || !ms) return FNEC_ERR_BAD_ARG;
    if (!b->ev_made) return fail(b->ctx, FNEC_ERR_BAD_ARG, "profiling was never enabled");
    cudaSetDevice(b->ctx->device);
    CUDA_TRY(b->ctx, cudaEventSynchronize(b->ev[FNEC_N_PHASES]));
    for (int k = 0; k < FNEC_N_PHASES; ++k) {
        float f = 0.f;
        CUDA_TRY(b->ctx, cudaEventElapsedTime(&f, b->ev[k], b->ev[k + 1]));
        ms[k] = (double)f;
    }
    return FNEC_OK;
}

int fnec_batch_sync(fnec_batch *b) {
    if (!b) return FNEC_ERR_BAD_ARG;
    cudaSetDevice(b->ctx->device);
    CUDA_TRY(b->ctx, cudaStreamSynchronize(b->st));
    return FNEC_OK;
}

// ---------------------------------------------------------------------------
// schedules, the autotuner and its cache
// ---------------------------------------------------------------------------

static bool schedule_valid(const fnec_schedule &s) {
    auto bit = [](int32_t v) { return v == 0 || v == 1; };
    return bit(s.grid_panels) && (s.class_shift == 1 || s.class_shift == 2) && bit(s.gram_tensor) &&
           (s.gmres_cluster == 1 || s.gmres_cluster == 2 || s.gmres_cluster == 4 || s.gmres_cluster == 8) &&
           bit(s.grid_gmres) && s.graph >= 0 && s.graph <= 2 &&
           (s.factor_streams == 1 || s.factor_streams == 2 || s.factor_streams == 4) && s.unit_factor >= 0 &&
           s.unit_factor <= 3 &&
           bit(s.block_inverse) && s.tensor_trailing >= 0 && s.tensor_trailing <= 2 &&
           (s.gmres_ctas_per_sm == 3 || s.gmres_ctas_per_sm == 4) && bit(s.factor_pivoting);
}

// Make the batch launch as s says (s valid); drops a captured graph when
// anything the pipeline's launches depend on changes.
static void apply_schedule(fnec_batch *b, const fnec_schedule &s) {
    fnec_schedule t = s;
    if (t.gmres_cluster > b->mixed.cluster_max) t.gmres_cluster = b->mixed.cluster_max;
    const bool same_launches = t.grid_panels == b->sched.grid_panels && t.class_shift == b->sched.class_shift &&
                               t.gram_tensor == b->sched.gram_tensor && t.gmres_cluster == b->sched.gmres_cluster &&
                               t.grid_gmres == b->sched.grid_gmres && t.factor_streams == b->sched.factor_streams &&
                               t.unit_factor == b->sched.unit_factor && t.block_inverse == b->sched.block_inverse &&
                               t.tensor_trailing == b->sched.tensor_trailing &&
                               t.gmres_ctas_per_sm == b->sched.gmres_ctas_per_sm &&
                               t.factor_pivoting == b->sched.factor_pivoting;
    if (!same_launches || (t.graph == 0) != (b->sched.graph == 0)) drop_graph(b);
    b->sched = t;
    b->grid.grid_on = t.grid_panels != 0;
    b->grid.class_shift = t.class_shift;
    b->mixed.use_tc = t.gram_tensor != 0;
    b->mixed.cluster_c = t.gmres_cluster < 1 ? 1 : t.gmres_cluster;
    b->mixed.grid_on = t.grid_gmres != 0;
    b->grid.factor_streams = t.factor_streams;
    b->grid.unit_factor = t.unit_factor;
    b->mixed.use_binv = t.block_inverse != 0;
    b->mixed.use_tc_trail = t.tensor_trailing == 1;
    b->mixed.two_step = t.tensor_trailing == 2;
    b->mixed.gmres_minb = t.gmres_ctas_per_sm;
    b->mixed.pivoting = t.factor_pivoting != 0;
}

static int ceil_log2(int64_t v) {
    int k = 0;
    while (((int64_t)1 << k) < v) ++k;
    return k;
}

// Batches whose launch structure is alike share a key: precision, SM count,
// solve count, largest and mean system size (log2 buckets) and which
// optional kernels the plan holds.
static std::string tune_key(const fnec_batch *b) {
    int64_t ssum = 0;
    for (const UnitDesc &u : b->units) ssum += u.s;
    const int64_t nu = (int64_t)b->units.size();
    char k[96];
    std::snprintf(k, sizeof(k), "p%d.sm%d.ns%d.nu%d.smax%d.smean%d.gp%d.gg%d.tc%d.cm%d", b->precision, b->grid.sms,
                  ceil_log2((int64_t)b->solves.size()), ceil_log2(nu), ceil_log2(b->max_s),
                  ceil_log2(nu ? ssum / nu : 0), b->grid.d_xchg ? 1 : 0, b->mixed.grid_solves.empty() ? 0 : 1,
                  b->mixed.tc ? 1 : 0, b->mixed.cluster_max);
    return k;
}

static std::mutex g_tune_mu;
static std::map<std::string, fnec_schedule> g_tune_cache;

static void schedule_from_cache(fnec_batch *b) {
    fnec_schedule s;
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        auto it = g_tune_cache.find(tune_key(b));
        if (it == g_tune_cache.end()) return;
        s = it->second;
    }
    apply_schedule(b, s);
}

int fnec_batch_get_schedule(const fnec_batch *b, fnec_schedule *out) {
    if (!b || !out) return FNEC_ERR_BAD_ARG;
    *out = b->sched;
    return FNEC_OK;
}

int fnec_batch_set_schedule(fnec_batch *b, const fnec_schedule *s) {
    if (!b || !s) return FNEC_ERR_BAD_ARG;
    if (!schedule_valid(*s)) return fail(b->ctx, FNEC_ERR_BAD_ARG, "schedule field out of range");
    cudaSetDevice(b->ctx->device);
    apply_schedule(b, *s);
    return FNEC_OK;
}

int fnec_batch_graph_state(const fnec_batch *b, int32_t *state, uint64_t *nodes) {
    if (!b) return FNEC_ERR_BAD_ARG;
    if (state) *state = b->graph_state;
    if (nodes) *nodes = b->graph_state == FNEC_GRAPH_READY ? b->graph_launches : 0;
    return FNEC_OK;
}

// Median device time (ms) of reps runs under s after one warm-up run, or
// a negative value if a run failed.
static double time_schedule(fnec_batch *b, const fnec_schedule &s, uint32_t reps, cudaEvent_t *ev) {
    apply_schedule(b, s);
    if (fnec_batch_run(b) != FNEC_OK || cudaStreamSynchronize(b->st) != cudaSuccess) return -1.0;
    std::vector<float> ms(reps);
    for (uint32_t r = 0; r < reps; ++r) {
        cudaEventRecord(ev[0], b->st);
        if (fnec_batch_run(b) != FNEC_OK) return -1.0;
        cudaEventRecord(ev[1], b->st);
        if (cudaEventSynchronize(ev[1]) != cudaSuccess) return -1.0;
        cudaEventElapsedTime(&ms[r], ev[0], ev[1]);
    }
    std::sort(ms.begin(), ms.end());
    return (double)ms[reps / 2];
}

int fnec_batch_tune(fnec_batch *b, uint32_t reps, fnec_tune_report *out) {
    if (!b) return FNEC_ERR_BAD_ARG;
    fnec_ctx *ctx = b->ctx;
    cudaSetDevice(ctx->device);
    const std::string key = tune_key(b);
    fnec_tune_report rep = {};
    std::snprintf(rep.key, sizeof(rep.key), "%s", key.c_str());
    fnec_schedule start = b->sched;
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        auto it = g_tune_cache.find(key);
        if (it != g_tune_cache.end()) {
            start = it->second;
            rep.from_cache = 1;
        }
    }
    if (reps == 0 || b->units.empty()) {
        apply_schedule(b, start);
        rep.best = b->sched;
        if (out) *out = rep;
        return FNEC_OK;
    }
    CUDA_TRY(ctx, cudaStreamSynchronize(b->st));
    cudaEvent_t ev[2];
    CUDA_TRY(ctx, cudaEventCreate(&ev[0]));
    if (cudaEventCreate(&ev[1]) != cudaSuccess) {
        cudaEventDestroy(ev[0]);
        return fail(ctx, FNEC_ERR_CUDA, "tune: event creation failed");
    }
    const bool prof = b->profile;
    b->profile = false;
    // graph capture first (the other fields are then timed as they will run)
    fnec_schedule best = start;
    best.graph = 2;
    double best_ms = time_schedule(b, best, reps, ev);
    if (b->graph_state != FNEC_GRAPH_READY || best_ms < 0) {
        best.graph = 0;
        best_ms = time_schedule(b, best, reps, ev);
    } else {
        fnec_schedule eager = best;
        eager.graph = 0;
        double t = time_schedule(b, eager, reps, ev);
        ++rep.candidates;
        if (t >= 0 && t < 0.98 * best_ms) {
            best = eager;
            best_ms = t;
        }
    }
    ++rep.candidates;
    if (best_ms < 0) {
        cudaEventDestroy(ev[0]);
        cudaEventDestroy(ev[1]);
        b->profile = prof;
        apply_schedule(b, start);
        return fail(ctx, FNEC_ERR_CUDA, "tune: the starting schedule failed to run: " + ctx->err);
    }
    rep.default_ms = best_ms;
    // coordinate descent over the launch-shape fields that can matter here
    struct Knob {
        int32_t fnec_schedule::*f;
        std::vector<int32_t> v;
    };
    std::vector<Knob> knobs;
    const bool mixed = b->precision == FNEC_PRECISION_MIXED;
    if (mixed) knobs.push_back(b->mixed.trail ? Knob{&fnec_schedule::tensor_trailing, {0, 1, 2}}
                                              : Knob{&fnec_schedule::tensor_trailing, {0, 2}});
    if (mixed && b->mixed.tc) knobs.push_back({&fnec_schedule::gram_tensor, {1, 0}});
    if (mixed && b->mixed.cluster_max > 1) {
        std::vector<int32_t> c;
        for (int v = 1; v <= b->mixed.cluster_max; v *= 2) c.push_back(v);
        knobs.push_back({&fnec_schedule::gmres_cluster, c});
    }
    if (mixed && !b->mixed.grid_solves.empty()) knobs.push_back({&fnec_schedule::grid_gmres, {1, 0}});
    if (b->grid.d_xchg) knobs.push_back({&fnec_schedule::grid_panels, {1, 0}});
    if (b->units.size() > 1) knobs.push_back({&fnec_schedule::class_shift, {1, 2}});
    if (mixed && !b->grid.s_desc.empty() && b->grid.s_desc.back() <= 512)
        knobs.push_back({&fnec_schedule::unit_factor, {1, 0, 2, 3}});
    if (mixed && b->mixed.fmade) knobs.push_back({&fnec_schedule::factor_streams, {1, 2, 4}});
    if (mixed) knobs.push_back({&fnec_schedule::block_inverse, {1, 0}});
    if (mixed) knobs.push_back({&fnec_schedule::gmres_ctas_per_sm, {3, 4}});
    if (mixed) knobs.push_back({&fnec_schedule::factor_pivoting, {0, 1}});
    // two passes of coordinate descent: a field's best value can depend on
    // fields tuned after it
    for (int pass = 0; pass < 2; ++pass)
    for (const Knob &k : knobs) {
        for (int32_t v : k.v) {
            if (best.*(k.f) == v) continue;
            fnec_schedule c = best;
            c.*(k.f) = v;
            double t = time_schedule(b, c, reps, ev);
            ++rep.candidates;
            if (t >= 0 && t < 0.98 * best_ms) {  // 2 % margin against timing noise
                best = c;
                best_ms = t;
            }
        }
    }
    cudaEventDestroy(ev[0]);
    cudaEventDestroy(ev[1]);
    b->profile = prof;
    (void)cudaGetLastError();  // a refused candidate's launch error
    if (best.graph) best.graph = 1;
    apply_schedule(b, best);
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        g_tune_cache[key] = b->sched;
    }
    rep.best = b->sched;
    rep.best_ms = best_ms;
    if (out) *out = rep;
    return FNEC_OK;
}

constexpr int N_SCHED_FIELDS = 12;
static const char *const SCHED_FIELDS[N_SCHED_FIELDS] = {"grid_panels",    "class_shift",   "gram_tensor",
                                                         "gmres_cluster",  "grid_gmres",    "graph",
                                                         "factor_streams", "unit_factor",   "block_inverse",
                                                         "tensor_trailing", "gmres_ctas_per_sm", "factor_pivoting"};
static int32_t *sched_field(fnec_schedule &s, int i) {
    int32_t *f[N_SCHED_FIELDS] = {&s.grid_panels,    &s.class_shift, &s.gram_tensor,   &s.gmres_cluster,
                                  &s.grid_gmres,     &s.graph,       &s.factor_streams, &s.unit_factor,
                                  &s.block_inverse,  &s.tensor_trailing, &s.gmres_ctas_per_sm, &s.factor_pivoting};
    return f[i];
}

int fnec_tune_cache_save(const char *path) {
    if (!path) return FNEC_ERR_BAD_ARG;
    std::FILE *f = std::fopen(path, "w");
    if (!f) return FNEC_ERR_BAD_ARG;
    std::lock_guard<std::mutex> lk(g_tune_mu);
    for (auto &kv : g_tune_cache) {
        fnec_schedule s = kv.second;
        std::fprintf(f, "%s", kv.first.c_str());
        for (int i = 0; i < N_SCHED_FIELDS; ++i) std::fprintf(f, " %s=%d", SCHED_FIELDS[i], (int)*sched_field(s, i));
        std::fprintf(f, "\n");
    }
    return std::fclose(f) == 0 ? FNEC_OK : FNEC_ERR_BAD_ARG;
}

int fnec_tune_cache_load(const char *path) {
    if (!path) return FNEC_ERR_BAD_ARG;
    std::FILE *f = std::fopen(path, "r");
    if (!f) return FNEC_ERR_BAD_ARG;
    std::map<std::string, fnec_schedule> got;
    char line[512];
    int rc = FNEC_OK;
    while (std::fgets(line, sizeof(line), f)) {
        char *save = nullptr;
        char *tok = strtok_r(line, " \t\r\n", &save);
        if (!tok || tok[0] == '#') continue;
        std::string key = tok;
        fnec_schedule s = {1, 1, 1, 1, 1, 1, 1, 1, 1, 0, 3, 0};
        int seen = 0;
        while ((tok = strtok_r(nullptr, " \t\r\n", &save))) {
            char *eq = std::strchr(tok, '=');
            if (!eq) {
                rc = FNEC_ERR_BAD_ARG;
                break;
            }
            *eq = 0;
            int i = 0;
            while (i < N_SCHED_FIELDS && std::strcmp(tok, SCHED_FIELDS[i]) != 0) ++i;
            if (i == N_SCHED_FIELDS) {
                rc = FNEC_ERR_BAD_ARG;
                break;
            }
            *sched_field(s, i) = (int32_t)std::atoi(eq + 1);
            seen |= 1 << i;
        }
        if (rc != FNEC_OK || seen != (1 << N_SCHED_FIELDS) - 1 || !schedule_valid(s)) {
            rc = FNEC_ERR_BAD_ARG;
            break;
        }
        got[key] = s;
    }
    std::fclose(f);
    if (rc != FNEC_OK) return rc;  // a malformed file changes nothing
    std::lock_guard<std::mutex> lk(g_tune_mu);
    for (auto &kv : got) g_tune_cache[kv.first] = kv.second;
    return FNEC_OK;
}

int fnec_tune_cache_clear(void) {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune_cache.clear();
    return FNEC_OK;
}

int fnec_tune_cache_size(uint32_t *n) {
    if (!n) return FNEC_ERR_BAD_ARG;
    std::lock_guard<std::mutex> lk(g_tune_mu);
    *n = (uint32_t)g_tune_cache.size();
    return FNEC_OK;
}

namespace fnec {
// currents of every solve, compacted (the c_hom tail of each x dropped)
__global__ void k_gather_currents(const UnitDesc *__restrict__ solves, const int64_t *__restrict__ cur_off,
                                  const cx *__restrict__ x, cx *cur) {
    const UnitDesc u = solves[blockIdx.x];
    for (int i = threadIdx.x; i < u.n; i += blockDim.x) cur[cur_off[blockIdx.x] + i] = x[u.x_off + i];
}
}  // namespace fnec

// Page-locked host memory (cudaMallocHost or registered): copies into it
// need no staging.
static bool is_pinned(const void *p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        (void)cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

extern "C" int fnec_host_alloc(uint64_t bytes, void **out) {
    if (!out) return FNEC_ERR_BAD_ARG;
    *out = nullptr;
    if (pin_alloc(out, (size_t)bytes) != cudaSuccess) {
        (void)cudaGetLastError();
        return FNEC_ERR_OUT_OF_MEMORY;
    }
    return FNEC_OK;
}

extern "C" int fnec_host_free(void *p) {
    if (!p) return FNEC_OK;
    if (pin_free(p)) return FNEC_OK;
    return cudaFreeHost(p) == cudaSuccess ? FNEC_OK : FNEC_ERR_CUDA;  // not one of the cache's blocks
}

extern "C" int fnec_host_cache_release(uint64_t *released) {
    std::multimap<size_t, void *> blocks;
    {
        std::lock_guard<std::mutex> lk(g_pin_mu);
        blocks.swap(g_pin_free);
        if (released) *released = g_pin_cached;
        g_pin_cached = 0;
    }
    for (auto &kv : blocks) cudaFreeHost(kv.second);
    return FNEC_OK;
}

int fnec_batch_read(fnec_batch *b, double *currents, double *feeds, double *pattern, int32_t *status,
                    double *total_radiated) {
    if (!b) return FNEC_ERR_BAD_ARG;
    fnec_ctx *ctx = b->ctx;
    cudaSetDevice(ctx->device);
    cudaStream_t st = b->st;
    int nu = (int)b->units.size(), ns = (int)b->solves.size();
    // device -> pinned staging -> caller arrays
    unsigned char *hx = b->h_out;
    unsigned char *hf = hx + sizeof(cx) * (size_t)b->x_el;
    unsigned char *hp = hf + sizeof(double) * 7 * (size_t)b->feed_rows;
    unsigned char *hs = hp + sizeof(double) * PAT_STRIDE * (size_t)b->pat_el;
    unsigned char *ht = hs + sizeof(int32_t) * (size_t)nu;
    size_t fb = sizeof(double) * 7 * (size_t)b->feed_rows, pb = sizeof(double) * PAT_STRIDE * (size_t)b->pat_el;
    const int64_t tc = b->uinfo.empty() ? 0 : b->uinfo.back().cur_off + b->uinfo.back().n;
    // caller arrays in page-locked memory are written directly; others
    // through the pinned staging buffer
    const bool pc = currents && is_pinned(currents), pf = feeds && fb && is_pinned(feeds),
               pp = pattern && pb && is_pinned(pattern), pt = total_radiated && is_pinned(total_radiated);
    if (currents && pc && tc > 0) {
        k_gather_currents<<<ns, 128, 0, st>>>(b->d_solves, b->d_cur_off, b->d_x, b->d_cur);
        CUDA_TRY(ctx, cudaMemcpyAsync(currents, b->d_cur, sizeof(cx) * tc, cudaMemcpyDeviceToHost, st));
    } else if (currents) {
        CUDA_TRY(ctx, cudaMemcpyAsync(hx, b->d_x, sizeof(cx) * b->x_el, cudaMemcpyDeviceToHost, st));
    }
    if (feeds && fb)
        CUDA_TRY(ctx, cudaMemcpyAsync(pf ? (void *)feeds : (void *)hf, b->d_feed_out, fb, cudaMemcpyDeviceToHost, st));
    if (pattern && pb)
        CUDA_TRY(ctx, cudaMemcpyAsync(pp ? (void *)pattern : (void *)hp, b->d_pat, pb, cudaMemcpyDeviceToHost, st));
    if (status) CUDA_TRY(ctx, cudaMemcpyAsync(hs, b->d_status, sizeof(int32_t) * nu, cudaMemcpyDeviceToHost, st));
    if (total_radiated)
        CUDA_TRY(ctx, cudaMemcpyAsync(pt ? (void *)total_radiated : (void *)ht, b->d_total, sizeof(double) * ns,
                                      cudaMemcpyDeviceToHost, st));
    CUDA_TRY(ctx, cudaStreamSynchronize(st));
    if (currents && !pc) {
        const cx *x = (const cx *)hx;
        for (int u = 0; u < ns; ++u)
            std::memcpy(currents + 2 * b->uinfo[u].cur_off, &x[b->solves[u].x_off], sizeof(cx) * b->solves[u].n);
    }
    if (feeds && fb && !pf) std::memcpy(feeds, hf, fb);
    if (pattern && pb && !pp) std::memcpy(pattern, hp, pb);
    if (status) {  // per solve: the status of its system
        const int32_t *sst = (const int32_t *)hs;
        std::vector<int32_t> tmp(sst, sst + nu);
        for (int u = 0; u < ns; ++u) status[u] = tmp[b->solves[u].sys];
    }
    if (total_radiated && !pt) std::memcpy(total_radiated, ht, sizeof(double) * ns);
    return FNEC_OK;
}

int fnec_batch_run_report(fnec_batch *b, double *pattern4) {
    if (!b || !pattern4) return FNEC_ERR_BAD_ARG;
    if (!is_pinned(pattern4)) return fail(b->ctx, FNEC_ERR_BAD_ARG, "run_report: pattern4 must be page-locked");
    cudaSetDevice(b->ctx->device);
    b->sink = pattern4;
    const int st = run_pipeline(b);  // eager: the sink's copies are not part of the batch's graph
    b->sink = nullptr;
    ++b->n_runs;
    return st;
}

int fnec_batch_read_report(fnec_batch *b, double *currents, double *feeds, double *pattern4, int32_t *status) {
    if (!b) return FNEC_ERR_BAD_ARG;
    fnec_ctx *ctx = b->ctx;
    cudaSetDevice(ctx->device);
    cudaStream_t st = b->st;
    const int64_t np = b->pat_el;
    if (pattern4 && np > 0) {
        if (!is_pinned(pattern4)) return fail(ctx, FNEC_ERR_BAD_ARG, "read_report: pattern4 must be page-locked");
        // the far-field field buffer (4 doubles per point) is free after the run
        const int blocks = (int)std::min<int64_t>((4 * np + 255) / 256, 148 * 16);
        k_pack_report<<<blocks, 256, 0, st>>>(b->d_pat, np, b->d_fld);
        CUDA_TRY(ctx, cudaMemcpyAsync(pattern4, b->d_fld, sizeof(double) * 4 * np, cudaMemcpyDeviceToHost, st));
    }
    return fnec_batch_read(b, currents, feeds, nullptr, status, nullptr);
}

int fnec_batch_read_receive(fnec_batch *b, double *out) {
    if (!b || !out) return FNEC_ERR_BAD_ARG;
    const size_t ns = b->solves.size();
    std::vector<double> peak(ns, std::nan(""));
    if (b->has_wave && ns > 0) {
        cudaError_t e = cudaMemcpyAsync(peak.data(), b->d_peak, sizeof(double) * ns, cudaMemcpyDeviceToHost, b->st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(b->st);
        if (e != cudaSuccess) return fail(b->ctx, FNEC_ERR_CUDA, cudaGetErrorString(e));
    }
    // solve_session.rs:356-374: each system's responses relative to its
    // largest peak (f64::max folds from 0 and passes over NaN)
    std::vector<double> top(b->units.size(), 0.0);
    for (size_t q = 0; q < ns; ++q)
        if (!std::isnan(peak[q])) top[b->solves[q].sys] = std::max(top[b->solves[q].sys], peak[q]);
    for (size_t q = 0; q < ns; ++q) {
        out[3 * q] = b->recv_dirs[2 * q];
        out[3 * q + 1] = b->recv_dirs[2 * q + 1];
        const double pk = peak[q], mx = top[b->solves[q].sys];
        if (std::isnan(b->recv_dirs[2 * q]) || std::isnan(pk)) out[3 * q + 2] = std::nan("");
        else out[3 * q + 2] = (pk > 0.0 && mx > 0.0) ? 20.0 * std::log10(pk / mx) : -999.99;
    }
    return FNEC_OK;
}

int fnec_batch_read_unit(fnec_batch *b, uint32_t unit, double *x, int32_t *pivots) {
    if (!b || unit >= b->solves.size()) return FNEC_ERR_BAD_ARG;
    fnec_ctx *ctx = b->ctx;
    cudaSetDevice(ctx->device);
    const UnitDesc &u = b->solves[unit];
    if (x)
        CUDA_TRY(ctx, cudaMemcpyAsync(x, b->d_x + u.x_off, sizeof(cx) * u.s, cudaMemcpyDeviceToHost,
                                      b->st));
    if (pivots)
        CUDA_TRY(ctx, cudaMemcpyAsync(pivots, b->d_piv + u.piv_off, sizeof(int32_t) * u.s,
                                      cudaMemcpyDeviceToHost, b->st));
    CUDA_TRY(ctx, cudaStreamSynchronize(b->st));
    return FNEC_OK;
}

int fnec_batch_read_refinement(fnec_batch *b, int32_t *iters, double *resid) {
    if (!b) return FNEC_ERR_BAD_ARG;
    if (b->precision != FNEC_PRECISION_MIXED) return fail(b->ctx, FNEC_ERR_BAD_ARG, "not a mixed-precision batch");
    cudaSetDevice(b->ctx->device);
    CUDA_TRY(b->ctx, read_mixed_stats(b->mixed, iters, resid, b->st));
    return FNEC_OK;
}

int fnec_batch_read_z(fnec_batch *b, uint32_t unit, double *z) {
    if (!b || !z || unit >= b->solves.size()) return FNEC_ERR_BAD_ARG;
    fnec_ctx *ctx = b->ctx;
    cudaSetDevice(ctx->device);
    const UnitDesc &u = b->units[b->solves[unit].sys];
    CUDA_TRY(ctx, cudaMemcpyAsync(z, b->d_z + u.z_off, sizeof(cx) * (size_t)u.n * u.n,
                                  cudaMemcpyDeviceToHost, b->st));
    CUDA_TRY(ctx, cudaStreamSynchronize(b->st));
    return FNEC_OK;
}

// ---- reference nec_accel entry points ---------------------------------------

int fnec_fill_zmatrix(fnec_ctx *ctx, const fnec_zsegment *segments, uint64_t n, double freq_hz,
                      int32_t ground, double *z_out) {
    if (!ctx || (!segments && n) || (!z_out && n)) return FNEC_ERR_BAD_ARG;
    if (ground != FNEC_GROUND_FREE && ground != FNEC_GROUND_PEC) return FNEC_ERR_BAD_ARG;
    if (n == 0) return FNEC_OK;
    cudaSetDevice(ctx->device);
    std::vector<DevSeg> hs(n);
    for (uint64_t i = 0; i < n; ++i) {
        DevSeg s{};
        for (int c = 0; c < 3; ++c) {
            s.mid[c] = segments[i].midpoint[c];
            s.dir[c] = segments[i].direction[c];
        }
        s.len = segments[i].length;
        s.rad = segments[i].radius;
        s.self_log = self_log_term(s.len, s.rad);
        hs[i] = s;
    }
    DevSeg *d_s = nullptr;
    cx *d_z = nullptr;
    CUDA_TRY(ctx, cudaMalloc(&d_s, sizeof(DevSeg) * n));
    cudaError_t e = cudaMalloc(&d_z, sizeof(cx) * n * n);
    if (e != cudaSuccess) {
        cudaFree(d_s);
        return fail(ctx, FNEC_ERR_OUT_OF_MEMORY, "fill_zmatrix: Z allocation");
    }
    e = cudaMemcpyAsync(d_s, hs.data(), sizeof(DevSeg) * n, cudaMemcpyHostToDevice, ctx->stream);
    double k = 2.0 * PI * freq_hz / C0;
    if (e == cudaSuccess) {
        launch_fill_exact_flat(d_s, (int)n, k, ground, d_z, ctx->stream);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(z_out, d_z, sizeof(cx) * n * n, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    cudaFree(d_s);
    cudaFree(d_z);
    if (e != cudaSuccess) return fail(ctx, FNEC_ERR_CUDA, cudaGetErrorString(e));
    return FNEC_OK;
}

static int solve_common(fnec_ctx *ctx, const fnec_zsegment *segments, const double *zin, uint64_t n,
                        const double *rhs, const double *cos_vec, const uint64_t *wire_endpoints, uint64_t w,
                        const fnec_junction *junctions, uint64_t nj, double freq_hz, int32_t ground,
                        int32_t precision, double *x_out, int32_t *pivots_out) {
    if (!ctx || n == 0 || (!segments && !zin) || !rhs || !cos_vec || !x_out) return FNEC_ERR_BAD_ARG;
    if (ground != FNEC_GROUND_FREE && ground != FNEC_GROUND_PEC) return FNEC_ERR_BAD_ARG;
    if (w && !wire_endpoints) return FNEC_ERR_BAD_ARG;
    if (precision == FNEC_PRECISION_MIXED && !mixed_available())
        return fail(ctx, FNEC_ERR_UNSUPPORTED, "mixed precision path not built");
    if (nj && !junctions) return FNEC_ERR_BAD_ARG;
    cudaSetDevice(ctx->device);
    std::vector<HostAnt> hs(1);
    HostAnt &h = hs[0];
    h.ground = ground;
    for (uint64_t i = 0; i < n; ++i) {
        DevSeg s{};
        if (segments) {
            for (int c = 0; c < 3; ++c) {
                s.mid[c] = segments[i].midpoint[c];
                s.dir[c] = segments[i].direction[c];
            }
            s.len = segments[i].length;
            s.rad = segments[i].radius;
            s.self_log = self_log_term(s.len, s.rad);
        }
        h.segs.push_back(s);
    }
    if (zin) h.z.assign(zin, zin + 2 * n * n);
    // linear.rs:689-696: an empty endpoint list means one wire (0, n-1)
    if (w == 0) {
        h.ep.push_back({0, (int64_t)n - 1});
    } else {
        for (uint64_t q = 0; q < w; ++q) {
            uint64_t f = wire_endpoints[2 * q], l = wire_endpoints[2 * q + 1];
            if (f > l || l >= n) return fail(ctx, FNEC_ERR_BAD_ARG, "wire endpoint out of range");
            h.ep.push_back({(int64_t)f, (int64_t)l});
        }
    }
    for (uint64_t t = 0; t < nj; ++t) {
        if (junctions[t].seg_a >= n || junctions[t].seg_b >= n)
            return fail(ctx, FNEC_ERR_BAD_ARG, "junction segment out of range");
        h.ja.push_back((int64_t)junctions[t].seg_a);
        h.jb.push_back((int64_t)junctions[t].seg_b);
        h.js.push_back(junctions[t].sign);
    }
    h.rhs_given = true;
    h.rhs.assign(rhs, rhs + 2 * n);
    h.cosv.assign(cos_vec, cos_vec + n);
    h.comp.assign(2 * n, 0);
    h.rp.pts_off = -1;
    h.rp.skip_integral = 1;
    h.freqs.push_back(freq_hz);
    fnec_batch *b = nullptr;
    int st = build_batch(ctx, hs, precision, &b);
    if (st != FNEC_OK) return st;
    st = fnec_batch_run(b);
    if (st == FNEC_OK) st = fnec_batch_sync(b);
    int32_t ust = 0;
    if (st == FNEC_OK) st = fnec_batch_read(b, nullptr, nullptr, nullptr, &ust, nullptr);
    if (st == FNEC_OK) st = fnec_batch_read_unit(b, 0, x_out, pivots_out);
    fnec_batch_destroy(b);
    if (st != FNEC_OK) return st;
    if (ust != 0) return fail(ctx, FNEC_ERR_SINGULAR, "singular pivot at column " + std::to_string(-ust - 1));
    return FNEC_OK;
}

int fnec_solve_hallen_resident(fnec_ctx *ctx, const fnec_zsegment *segments, uint64_t n,
                               const double *rhs, const double *cos_vec, const uint64_t *wire_endpoints,
                               uint64_t w, const fnec_junction *junctions, uint64_t nj, double freq_hz,
                               int32_t ground, int32_t precision, double *x_out, int32_t *pivots_out) {
    if (!segments) return FNEC_ERR_BAD_ARG;
    return solve_common(ctx, segments, nullptr, n, rhs, cos_vec, wire_endpoints, w, junctions, nj, freq_hz,
                        ground, precision, x_out, pivots_out);
}

int fnec_solve_hallen(fnec_ctx *ctx, const double *z, uint64_t n, const double *rhs, const double *cos_vec,
                      const uint64_t *wire_endpoints, uint64_t w, const fnec_junction *junctions, uint64_t nj,
                      int32_t precision, double *x_out, int32_t *pivots_out) {
    if (!z) return FNEC_ERR_BAD_ARG;
    return solve_common(ctx, nullptr, z, n, rhs, cos_vec, wire_endpoints, w, junctions, nj, 1.0,
                        FNEC_GROUND_FREE, precision, x_out, pivots_out);
}

static int pattern_common(fnec_ctx *ctx, const fnec_gpu_segment *segments, uint64_t n,
                          const double *currents, double k_rp, int32_t ground, const double *points,
                          uint64_t p, bool skip_integral, double total_given, std::vector<double> &pat,
                          double &total) {
    if (!ctx || n == 0 || !segments || !currents) return FNEC_ERR_BAD_ARG;
    if (p && !points) return FNEC_ERR_BAD_ARG;
    cudaSetDevice(ctx->device);
    std::vector<HostAnt> hs(1);
    HostAnt &h = hs[0];
    h.ground = ground;
    for (uint64_t i = 0; i < n; ++i) {
        DevSeg s{};
        for (int c = 0; c < 3; ++c) {
            s.mid[c] = segments[i].midpoint[c];
            s.dir[c] = segments[i].direction[c];
        }
        s.len = segments[i].length;
        s.tag = 1;
        h.segs.push_back(s);
    }
    h.ep.push_back({0, (int64_t)n - 1});
    h.comp.assign(2 * n, 0);
    build_runs(h);
    h.rp.pts_off = -1;
    if (p) h.pts.assign(points, points + 2 * p);
    h.rp.skip_integral = skip_integral ? 1 : 0;
    h.rp.total_given = total_given;
    h.freqs.push_back(1.0);  // placeholder; k is set below
    fnec_batch *b = nullptr;
    int st = build_batch(ctx, hs, FNEC_PRECISION_FP64, &b, false);
    if (st != FNEC_OK) return st;
    b->units[0].k_rp = k_rp;
    b->solves[0].k_rp = k_rp;
    cudaStream_t s = ctx->stream;
    cudaStreamSynchronize(s);
    cudaError_t e = cudaMemcpyAsync(b->d_units, b->units.data(), sizeof(UnitDesc), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(b->d_solves, b->solves.data(), sizeof(UnitDesc), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(b->d_status, 0, sizeof(int32_t), s);
    if (e == cudaSuccess) e = cudaMemsetAsync(b->d_total, 0, sizeof(double), s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(b->d_x, currents, sizeof(cx) * n, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) {
        launch_farfield(b->d_solves, 1, b->d_ants, b->d_runs, b->d_rps, b->d_pts, b->d_ibuf, b->d_x, b->d_status, b->d_fld,
                        b->d_partials, b->ff_blocks, b->ff_smem, b->d_pat, b->d_total, s);
        e = cudaGetLastError();
    }
    pat.assign(PAT_STRIDE * (p ? p : 1), 0.0);
    if (e == cudaSuccess && p)
        e = cudaMemcpyAsync(pat.data(), b->d_pat, sizeof(double) * PAT_STRIDE * p, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&total, b->d_total, sizeof(double), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    fnec_batch_destroy(b);
    if (e != cudaSuccess) return fail(ctx, FNEC_ERR_CUDA, cudaGetErrorString(e));
    return FNEC_OK;
}

int fnec_rp_farfield_batch(fnec_ctx *ctx, const fnec_gpu_segment *segments, uint64_t n,
                           const double *currents, double k, double total_radiated, const double *points,
                           uint64_t p, fnec_rp_result *out) {
    if (p == 0) return FNEC_OK;
    if (!out) return FNEC_ERR_BAD_ARG;
    std::vector<double> pat;
    double total = 0;
    int st = pattern_common(ctx, segments, n, currents, k, FNEC_GROUND_FREE, points, p, true, total_radiated,
                            pat, total);
    if (st != FNEC_OK) return st;
    for (uint64_t q = 0; q < p; ++q) {
        const double *o = &pat[PAT_STRIDE * q];
        out[q].gain_total_dbi = o[0];
        out[q].gain_theta_dbi = o[1];
        out[q].gain_phi_dbi = o[2];
        out[q].axial_ratio = o[3];
        out[q].u_theta = o[4];
        out[q].u_phi = o[5];
        out[q].theta_deg = points[2 * q];
        out[q].phi_deg = points[2 * q + 1];
    }
    return FNEC_OK;
}

int fnec_radiation_pattern(fnec_ctx *ctx, const fnec_gpu_segment *segments, uint64_t n,
                           const double *currents, double freq_hz, int32_t ground, const double *points,
                           uint64_t p, double *out, double *total_out) {
    if (p && !out) return FNEC_ERR_BAD_ARG;
    std::vector<double> pat;
    double total = 0;
    int st = pattern_common(ctx, segments, n, currents, 2.0 * PI / (C0 / freq_hz), ground, points, p, false,
                            0.0, pat, total);
    if (st != FNEC_OK) return st;
    for (uint64_t q = 0; q < p; ++q)
        for (int c = 0; c < 4; ++c) out[4 * q + c] = pat[PAT_STRIDE * q + c];
    if (total_out) *total_out = total;
    return FNEC_OK;
}

int fnec_integrate_radiated_power(fnec_ctx *ctx, const fnec_gpu_segment *segments, uint64_t n,
                                  const double *currents, double freq_hz, int32_t pec_ground, double *out) {
    if (!out) return FNEC_ERR_BAD_ARG;
    std::vector<double> pat;
    double total = 0;
    int st = pattern_common(ctx, segments, n, currents, 2.0 * PI / (C0 / freq_hz),
                            pec_ground ? FNEC_GROUND_PEC : FNEC_GROUND_FREE, nullptr, 0, false, 0.0, pat, total);
    if (st != FNEC_OK) return st;
    *out = total;
    return FNEC_OK;
}

int fnec_build_geometry(const fnec_wire *wires, uint32_t n_wires, fnec_zsegment *out, uint64_t cap,
                        uint64_t *n_out) {
    if (!n_out || (n_wires && !wires)) return FNEC_ERR_BAD_ARG;
    uint64_t n = 0;
    for (uint32_t w = 0; w < n_wires; ++w) {
        const fnec_wire &gw = wires[w];
        const double dx = gw.end[0] - gw.start[0], dy = gw.end[1] - gw.start[1], dz = gw.end[2] - gw.start[2];
        if (gw.segments == 0 || std::sqrt(dx * dx + dy * dy + dz * dz) == 0.0) return FNEC_ERR_BAD_ARG;
        n += gw.segments;
    }
    *n_out = n;
    if (!out || cap < n) return FNEC_OK;
    uint64_t q = 0;
    for (uint32_t w = 0; w < n_wires; ++w)
        for (uint32_t i = 0; i < wires[w].segments; ++i, ++q) {
            const DevSeg d = host_seg(wires[w], i);
            for (int c = 0; c < 3; ++c) {
                out[q].midpoint[c] = d.mid[c];
                out[q].direction[c] = d.dir[c];
            }
            out[q].length = d.len;
            out[q].radius = d.rad;
        }
    return FNEC_OK;
}

static_assert(sizeof(fnec_gpu_segment) == 7 * sizeof(double), "fnec_gpu_segment is 7 packed doubles");

int fnec_near_field(fnec_ctx *ctx, const fnec_gpu_segment *segments, uint64_t n, const double *currents,
                    double freq_hz, const double *points, uint64_t p, double *e_out, double *h_out) {
    if (!ctx) return FNEC_ERR_BAD_ARG;
    if (p == 0) return FNEC_OK;
    if (!points || (!e_out && !h_out) || (n && (!segments || !currents)))
        return fail(ctx, FNEC_ERR_BAD_ARG, "near field: null argument");
    if (!(freq_hz > 0.0) || !std::isfinite(freq_hz)) return fail(ctx, FNEC_ERR_BAD_ARG, "near field: bad frequency");
    if (p > (uint64_t)INT32_MAX * 128 || n > (uint64_t)INT32_MAX)
        return fail(ctx, FNEC_ERR_BAD_ARG, "near field: too many points or segments");
    // farfield.rs:160-161, :224-225 (host code built without contraction)
    const double k = 2.0 * PI * freq_hz / C0;
    const double eta0 = 4.0 * PI * 1e-7 * C0;
    const double coeff_e = eta0 / (4.0 * PI), coeff_h = 1.0 / (4.0 * PI);
    cudaSetDevice(ctx->device);
    const size_t n_seg = 7 * n, n_cur = 2 * n, n_pts = 3 * p, n_fld = 6 * p;
    const size_t total = n_seg + n_cur + n_pts + (e_out ? n_fld : 0) + (h_out ? n_fld : 0);
    double *d = nullptr;
    CUDA_TRY(ctx, cudaMalloc(&d, sizeof(double) * total));
    double *d_seg = d, *d_cur = d_seg + n_seg, *d_pts = d_cur + n_cur, *d_e = d_pts + n_pts;
    double *d_h = d_e + (e_out ? n_fld : 0);
    cudaStream_t s = ctx->stream;
    cudaError_t e = cudaSuccess;
    if (n) e = cudaMemcpyAsync(d_seg, segments, sizeof(double) * n_seg, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess && n) e = cudaMemcpyAsync(d_cur, currents, sizeof(double) * n_cur, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_pts, points, sizeof(double) * n_pts, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) {
        launch_near_field(d_seg, (int64_t)n, reinterpret_cast<const cx *>(d_cur), k, coeff_e, coeff_h, d_pts,
                          (int64_t)p, e_out ? reinterpret_cast<cx *>(d_e) : nullptr,
                          h_out ? reinterpret_cast<cx *>(d_h) : nullptr, s);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess && e_out) e = cudaMemcpyAsync(e_out, d_e, sizeof(double) * n_fld, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess && h_out) e = cudaMemcpyAsync(h_out, d_h, sizeof(double) * n_fld, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    cudaFree(d);
    if (e != cudaSuccess) return fail(ctx, FNEC_ERR_CUDA, cudaGetErrorString(e));
    return FNEC_OK;
}

int fnec_microbench_zmatrix_dispatch(int device, uint64_t n_segments, uint32_t n_dispatches,
                                     uint64_t *device_init_us, uint64_t *dispatch_min_us,
                                     uint64_t *dispatch_median_us) {
    using clk = std::chrono::steady_clock;
    if (n_segments == 0 || n_dispatches == 0) return FNEC_ERR_BAD_ARG;
    auto t0 = clk::now();
    fnec_ctx *ctx = nullptr;
    int st = fnec_ctx_create(device, &ctx);
    if (st != FNEC_OK) return st;
    std::vector<fnec_zsegment> segs(n_segments);
    double L = 10.0, dl = L / (double)n_segments;
    for (uint64_t i = 0; i < n_segments; ++i) {
        fnec_zsegment s{};
        s.midpoint[2] = -L / 2 + dl * ((double)i + 0.5);
        s.direction[2] = 1.0;
        s.length = dl;
        s.radius = 1e-3;
        segs[i] = s;
    }
    std::vector<double> z(2 * n_segments * n_segments);
    st = fnec_fill_zmatrix(ctx, segs.data(), n_segments, 14.2e6, FNEC_GROUND_FREE, z.data());
    auto t1 = clk::now();
    std::vector<uint64_t> us;
    for (uint32_t d = 0; d < n_dispatches && st == FNEC_OK; ++d) {
        auto a = clk::now();
        st = fnec_fill_zmatrix(ctx, segs.data(), n_segments, 14.2e6, FNEC_GROUND_FREE, z.data());
        us.push_back((uint64_t)std::chrono::duration_cast<std::chrono::microseconds>(clk::now() - a).count());
    }
    fnec_ctx_destroy(ctx);
    if (st != FNEC_OK) return st;
    std::sort(us.begin(), us.end());
    if (device_init_us)
        *device_init_us = (uint64_t)std::chrono::duration_cast<std::chrono::microseconds>(t1 - t0).count();
    if (dispatch_min_us) *dispatch_min_us = us.front();
    if (dispatch_median_us) *dispatch_median_us = us[us.size() / 2];
    return FNEC_OK;
}

int fnec_enumerate_devices(int *count, int index, char *name, uint64_t cap) {
    int c = 0;
    if (cudaGetDeviceCount(&c) != cudaSuccess) c = 0;
    if (count) *count = c;
    if (name && cap > 0) {
        name[0] = 0;
        if (index >= 0 && index < c) {
            cudaDeviceProp p;
            if (cudaGetDeviceProperties(&p, index) == cudaSuccess) {
                std::snprintf(name, (size_t)cap, "%s (sm_%d%d)", p.name, p.major, p.minor);
            }
        }
    }
    return FNEC_OK;
}

int fnec_dispatch_frequency_point(int request_kind, double freq_hz) {
    (void)request_kind;
    (void)freq_hz;
    int c = 0;
    if (cudaGetDeviceCount(&c) != cudaSuccess) return 0;
    return c > 0 ? 1 : 0;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Serving: requests (one antenna deck each) batched continuously over lanes.
//
// Each lane is a CUDA stream driven by its own host thread.  A lane that is
// free takes queued requests in arrival order while the device bytes of the
// batches in flight stay within the HBM budget, plans them as one batch
// (stream-ordered pool allocations), enqueues upload + solve + result copies
// on its stream, sleeps on the completion event, and delivers the results.
// Requests that arrive while other batches run are taken by the next free
// lane; the lanes' planning, kernels and copies overlap.  A request's systems
// keep Z and the factor on the device for all of its right-hand sides (one
// per source position) and its pattern.  Results land in a page-locked slab
// of the server: requests submitted with output arrays get a copy, the others
// read the slab in place until they are released.
// ---------------------------------------------------------------------------
#include <condition_variable>
#include <deque>
#include <mutex>
#include <thread>
#include <unordered_map>

namespace {

using Clock = std::chrono::steady_clock;

struct Slab {  // page-locked results of one batch, shared by its requests
    PinnedArena mem;
    int refs = 0;
};

struct ServerReq {
    uint64_t ticket = 0;
    HostAnt host;
    fnec_request_out out{};
    bool copy_out = false;
    int64_t bytes = 0;
    uint32_t n_solves = 0, n = 0, s = 0, n_points = 0, n_feed_rows = 0;
    Clock::time_point t_submit, t_done;
    int32_t state = FNEC_REQ_QUEUED;
    // results in place (no output arrays): offsets into the slab
    Slab *slab = nullptr;
    size_t x_off = 0, feed_row = 0, pat_row = 0;  // complex / feed rows / pattern rows
    size_t hf_off = 0, hp_off = 0;                // byte offsets of the feed and pattern blocks
    std::vector<int32_t> status;
};

struct Lane {
    cudaStream_t st = nullptr;
    cudaEvent_t done = nullptr;
    PinnedArena in, aux;
    std::thread worker;
};

// Upper bound of the device bytes one request's batch needs (Z, the
// factor, solution and work vectors, Gram operand stacks, pattern buffers).
int64_t request_bytes(const HostAnt &h, int precision) {
    const int64_t n = (int64_t)h.segs.size(), w = h.cols(), s = n + w;
    const int64_t f = (int64_t)h.freqs.size(), r = (int64_t)std::max<size_t>(h.rhs_srcs.size(), 1);
    const int64_t rows = n + 2 * w + (int64_t)h.ja.size();
    const int64_t pts = h.rp.pts_off >= 0 ? (int64_t)h.pts.size() / 2 : (int64_t)h.rp.n_theta * h.rp.n_phi;
    const int64_t n_int = h.rp.skip_integral ? 0 : (h.ground == 1 ? 91 : 181) * 360;
    int64_t b = 0;
    b += 16 * n * n * f;                                   // Z
    b += 160 * n + 256 * w + 64 * rows + 4 * n_int;        // geometry, tables, coverage maps
    b += n * n / 16 + 64 * ((n + 63) / 64) * ((n + 64) / 64);  // fill and Gram tile lists
    b += 16 * n * f * r;                                   // compact currents for pinned reads
    b += (16 * s + 16 * n + 8 * n + 64) * f * r;           // x, rhs, cos, feeds
    if (h.planewave) b += 8 * n * f + 8 * f * r + 80 * r + 16 * n + 8 * n * n * f;  // sin column, peaks,
                                                                                   // waves, arc, sin(k|ds|) table
    b += (48 + 32) * pts * f * r + 8 * 1024 * f * r;      // pattern, fields, partials
    if (precision == FNEC_PRECISION_MIXED) {
        int64_t kb = (n + 31) / 32, rp = ((2 * n + 127) / 128) * 128;
        b += 8 * s * s * f;                                // FP32 factor
        b += 2 * 128 * kb * rp * f + 64 * kb * kb * f;     // Gram operand stacks (hi, lo), tiles
        b += 16 * (25 * s + 6 * s + 2 * rows) * f * r;     // GMRES basis and work vectors
        b += (16 * (((n + 31) / 32) * n + 2 * s + 512) + 4) * f * r;  // cluster GMRES scratch, launch order
        b += 16 * 2048 * ((s + 31) / 32) * f;              // diagonal block inverses of the factor
        if (s - 32 >= 192) {                               // tensor-core trailing stacks and step lists
            const int64_t m0 = s - 32, pa = (m0 + 127) / 128 * 128, pb = (2 * m0 + 127) / 128 * 128;
            b += (256 * (2 * pa + 2 * pb) + 32 * ((s + 31) / 32)) * f;
        }
    } else {
        b += 16 * s * (s + 1) * f + 4 * s * f;             // FP64 factor, pivots
    }
    if (s > 380) b += (int64_t)grid_xchg_bytes() + (int64_t)grid_sync_bytes((int)((s + 31) / 32));  // grid panels
    if (precision == FNEC_PRECISION_MIXED && s >= 1536)   // grid-wide GMRES scratch
        b += 16 * n * ((n + 255) / 256) + 64 * s + 16 * 2 * 296 * 25 + 4096;
    return b + (1 << 20);
}

bool finished(const ServerReq *r) { return r->state == FNEC_REQ_DONE || r->state < 0; }

constexpr size_t SERVER_IN_ARENA = 128ull << 20;  // packed inputs of one batch
constexpr size_t SERVER_AUX_ARENA = 64ull << 20;  // its other uploads
constexpr size_t SERVER_SLAB = 512ull << 20;      // results of one batch (grows for larger ones)

}  // namespace

struct fnec_server {
    int device = 0;
    fnec_server_config cfg{};
    std::mutex mu;
    std::condition_variable work_cv;  // wakes lanes: a request queued, memory freed, stop
    std::condition_variable done_cv;  // wakes waiters
    std::deque<ServerReq *> queue;
    std::deque<uint64_t> done_q;  // finished tickets, in completion order
    std::unordered_map<uint64_t, ServerReq *> live;
    std::vector<Lane> lanes;
    std::vector<Slab *> slabs_free, slabs_all;
    size_t max_slabs = 0;  // page-locked result slabs, at most (lanes and unreleased requests share them)
    int64_t in_flight = 0;
    uint64_t next_ticket = 1;
    bool stop = false;
    // statistics since the last reset
    std::vector<double> lat_ms;
    uint64_t submitted = 0, completed = 0, failed = 0, solves = 0, batches = 0, launches = 0, h2d = 0, d2h = 0;
    int64_t peak_bytes = 0;
    uint64_t max_batch_seen = 0;
    double plan_ms = 0, launch_ms = 0, collect_ms = 0;  // host time of the lanes' three jobs
    double alloc_ms = 0;                                // of plan_ms: allocation
    double t_dev = 0, t_copy = 0, t_pinned = 0, t_mixed = 0;
    std::string last_err;  // the most recent failure, for fnec_server_last_error
    std::string err_copy;
};

namespace {

void slab_unref(fnec_server *S, Slab *sl) {  // S->mu held
    if (sl && --sl->refs == 0) S->slabs_free.push_back(sl);
}

// Takes the next batch (arrival order, within budget and max_batch); S->mu held.
std::vector<ServerReq *> admit(fnec_server *S, int64_t &bytes) {
    std::vector<ServerReq *> take;
    bytes = 0;
    while (!S->queue.empty() && take.size() < S->cfg.max_batch) {
        ServerReq *r = S->queue.front();
        if (S->in_flight + bytes + r->bytes > (int64_t)S->cfg.hbm_budget_bytes) break;
        bytes += r->bytes;
        take.push_back(r);
        S->queue.pop_front();
    }
    return take;
}

// Distribute a finished batch's results (in the slab b->h_out) to its requests.
void deliver(fnec_batch *b, const std::vector<ServerReq *> &take, Slab *slab, bool ok) {
    const unsigned char *hx = b->h_out;
    const size_t f_off = sizeof(cx) * (size_t)b->x_el;
    const size_t p_off = f_off + sizeof(double) * 7 * (size_t)b->feed_rows;
    const int32_t *hst = (const int32_t *)(hx + p_off + sizeof(double) * PAT_STRIDE * (size_t)b->pat_el);
    const cx *x = (const cx *)hx;
    struct Next {
        uint32_t k = 0;    // next solve of the request
        size_t row = 0;    // its next feed row
    };
    std::vector<Next> next(take.size());
    for (size_t u = 0; u < b->solves.size(); ++u) {
        const fnec_unit_info &ui = b->uinfo[u];
        ServerReq *r = take[ui.antenna];
        const uint32_t k = next[ui.antenna].k++;
        const size_t row0 = next[ui.antenna].row;
        next[ui.antenna].row += ui.n_feed;
        r->status[k] = ok ? hst[b->solves[u].sys] : FNEC_ERR_CUDA;
        if (k == 0) {  // a request's solves are consecutive: its first solve locates its blocks
            r->slab = slab;
            r->x_off = (size_t)b->solves[u].x_off;
            r->feed_row = (size_t)ui.feed_off;
            r->pat_row = (size_t)ui.pat_off;
            r->hf_off = f_off;
            r->hp_off = p_off;
        }
        if (!ok || !r->copy_out) continue;
        if (r->out.status) r->out.status[k] = r->status[k];
        if (r->out.currents)
            std::memcpy(r->out.currents + 2 * (size_t)k * r->n, &x[b->solves[u].x_off], sizeof(cx) * ui.n);
        if (r->out.feeds && ui.n_feed)
            std::memcpy(r->out.feeds + 7 * row0, hx + f_off + sizeof(double) * 7 * ui.feed_off,
                        sizeof(double) * 7 * ui.n_feed);
        if (r->out.pattern && ui.n_points)
            std::memcpy(r->out.pattern + (size_t)PAT_STRIDE * k * r->n_points,
                        hx + p_off + sizeof(double) * PAT_STRIDE * ui.pat_off,
                        sizeof(double) * PAT_STRIDE * ui.n_points);
    }
    if (!ok)
        for (ServerReq *r : take)
            if (r->out.status)
                for (uint32_t k = 0; k < r->n_solves; ++k) r->out.status[k] = FNEC_ERR_CUDA;
}

// Enqueue the device -> slab copies of every result of a batch.
cudaError_t enqueue_results(fnec_batch *b) {
    unsigned char *hx = b->h_out;
    unsigned char *hf = hx + sizeof(cx) * (size_t)b->x_el;
    unsigned char *hp = hf + sizeof(double) * 7 * (size_t)b->feed_rows;
    unsigned char *hs = hp + sizeof(double) * PAT_STRIDE * (size_t)b->pat_el;
    size_t fb = sizeof(double) * 7 * (size_t)b->feed_rows, pb = sizeof(double) * PAT_STRIDE * (size_t)b->pat_el;
    cudaError_t e = cudaMemcpyAsync(hx, b->d_x, sizeof(cx) * b->x_el, cudaMemcpyDeviceToHost, b->st);
    if (e == cudaSuccess && fb) e = cudaMemcpyAsync(hf, b->d_feed_out, fb, cudaMemcpyDeviceToHost, b->st);
    if (e == cudaSuccess && pb) e = cudaMemcpyAsync(hp, b->d_pat, pb, cudaMemcpyDeviceToHost, b->st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(hs, b->d_status, sizeof(int32_t) * b->units.size(), cudaMemcpyDeviceToHost, b->st);
    return e;
}

void lane_worker(fnec_server *S, Lane *L) {
    cudaSetDevice(S->device);
    fnec_ctx own;  // this lane's private context: its own error string
    own.device = S->device;
    own.stream = L->st;
    for (;;) {
        std::vector<ServerReq *> take;
        int64_t bytes = 0;
        Slab *slab = nullptr;
        {
            std::unique_lock<std::mutex> lk(S->mu);
            for (;;) {
                // a result slab must be free (or creatable) before requests are taken:
                // allocating page-locked memory while other lanes run stalls them all
                const bool slab_ok = !S->slabs_free.empty() || S->slabs_all.size() < S->max_slabs;
                if (slab_ok) {
                    take = admit(S, bytes);
                    if (!take.empty()) break;
                }
                if (S->stop && S->queue.empty()) return;
                S->work_cv.wait(lk);
            }
            for (ServerReq *r : take) r->state = FNEC_REQ_RUNNING;
            S->in_flight += bytes;
            S->peak_bytes = std::max(S->peak_bytes, S->in_flight);
            if (!S->slabs_free.empty()) {
                slab = S->slabs_free.back();
                S->slabs_free.pop_back();
            } else {
                slab = new Slab();
                S->slabs_all.push_back(slab);
            }
        }
        std::vector<HostAnt> hs;
        hs.reserve(take.size());
        for (ServerReq *r : take) hs.push_back(r->host);
        BatchPlace place;
        place.st = L->st;
        place.pooled = true;
        place.allow_grid = S->lanes.size() == 1;  // cooperative kernels need the whole device
        place.in = &L->in;
        place.out = &slab->mem;
        place.aux = &L->aux;
        fnec_batch *b = nullptr;
        const auto t0 = Clock::now();
        int st = build_batch(&own, hs, S->cfg.precision, &b, true, place);
        const auto t1 = Clock::now();
        cudaError_t e = cudaSuccess;
        if (st == FNEC_OK) st = fnec_batch_run(b);
        if (st == FNEC_OK) e = enqueue_results(b);
        if (st == FNEC_OK && e == cudaSuccess) e = cudaEventRecord(L->done, L->st);
        const auto t2 = Clock::now();
        if (st == FNEC_OK && e == cudaSuccess) e = cudaEventSynchronize(L->done);  // the thread sleeps
        const bool ok = st == FNEC_OK && e == cudaSuccess;
        const auto t3 = Clock::now();
        if (b) deliver(b, take, slab, ok);
        const auto t4 = Clock::now();
        uint64_t launches = 0, h2d = 0, d2h = 0;
        double alloc_ms = 0, t_dev = 0, t_copy = 0, t_pinned = 0, t_mixed = 0;
        if (b) {
            alloc_ms = b->alloc_ms;
            t_dev = b->t_dev;
            t_copy = b->t_copy;
            t_pinned = b->t_pinned;
            t_mixed = b->t_mixed;
            launches = b->launches;
            h2d = b->in_bytes;
            d2h = sizeof(cx) * (size_t)b->x_el + sizeof(double) * 7 * (size_t)b->feed_rows +
                  sizeof(double) * PAT_STRIDE * (size_t)b->pat_el + sizeof(int32_t) * b->units.size();
            if (!ok) cudaStreamSynchronize(L->st);
            free_batch(b);  // pooled: the frees are ordered on the lane's stream
            delete b;
        }
        {
            std::lock_guard<std::mutex> lk(S->mu);
            S->plan_ms += std::chrono::duration<double, std::milli>(t1 - t0).count();
            S->alloc_ms += alloc_ms;
            S->t_dev += t_dev;
            S->t_copy += t_copy;
            S->t_pinned += t_pinned;
            S->t_mixed += t_mixed;
            S->launch_ms += std::chrono::duration<double, std::milli>(t2 - t1).count();
            S->collect_ms += std::chrono::duration<double, std::milli>(t4 - t3).count();
            if (!ok) {
                if (st != FNEC_OK) S->last_err = "batch of " + std::to_string(take.size()) + " requests: " + own.err;
                else S->last_err = std::string("lane batch: ") + cudaGetErrorString(e);
            }
            S->in_flight -= bytes;
            ++S->batches;
            S->max_batch_seen = std::max<uint64_t>(S->max_batch_seen, take.size());
            S->launches += launches;
            S->h2d += h2d;
            S->d2h += d2h;
            const auto now = Clock::now();
            for (ServerReq *r : take) {
                r->t_done = now;
                r->state = ok ? FNEC_REQ_DONE : (st != FNEC_OK ? st : FNEC_ERR_CUDA);
                if (ok) {
                    S->lat_ms.push_back(std::chrono::duration<double, std::milli>(r->t_done - r->t_submit).count());
                    ++S->completed;
                    S->solves += r->n_solves;
                    if (!r->copy_out) ++slab->refs;  // read in place until released
                } else {
                    ++S->failed;
                }
                if (r->copy_out || !ok) r->slab = nullptr;
                S->done_q.push_back(r->ticket);
            }
            if (slab->refs == 0) S->slabs_free.push_back(slab);
        }
        S->done_cv.notify_all();
        S->work_cv.notify_all();  // memory freed: the queue head may fit now
    }
}

}  // namespace

int fnec_server_create(fnec_ctx *ctx, const fnec_server_config *cfg, fnec_server **out) {
    if (!ctx || !cfg || !out) return FNEC_ERR_BAD_ARG;
    *out = nullptr;
    if (cfg->precision != FNEC_PRECISION_FP64 && cfg->precision != FNEC_PRECISION_MIXED)
        return fail(ctx, FNEC_ERR_BAD_ARG, "precision must be FP64 or MIXED");
    if (cfg->lanes < 1 || cfg->lanes > 16 || cfg->max_batch < 1 || cfg->hbm_budget_bytes == 0)
        return fail(ctx, FNEC_ERR_BAD_ARG, "lanes 1..16, max_batch >= 1 and a nonzero HBM budget");
    cudaSetDevice(ctx->device);
    fnec_server *S = new fnec_server();
    S->device = ctx->device;
    S->cfg = *cfg;
    if (S->cfg.queue_cap == 0) S->cfg.queue_cap = 1u << 20;
    S->lanes.resize(cfg->lanes);
    for (Lane &L : S->lanes) {
        if (cudaStreamCreateWithFlags(&L.st, cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&L.done, cudaEventDisableTiming | cudaEventBlockingSync) != cudaSuccess) {
            for (Lane &M : S->lanes) {
                if (M.done) cudaEventDestroy(M.done);
                if (M.st) cudaStreamDestroy(M.st);
            }
            delete S;
            return fail(ctx, FNEC_ERR_CUDA, "lane stream creation failed");
        }
    }
    // keep pool memory freed by finished batches cached for the next ones,
    // and map the HBM budget into the pool now (less what it holds already;
    // at most the device's free memory less 2 GiB): a lane admitting a large
    // batch under load then suballocates instead of waiting for the driver
    // to map gigabytes (about a second for 8 GiB)
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, ctx->device) == cudaSuccess) {
        uint64_t keep = UINT64_MAX;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        uint64_t held = 0;
        size_t fr = 0, tot = 0;
        cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &held);
        if (cudaMemGetInfo(&fr, &tot) == cudaSuccess) {
            const uint64_t margin = (uint64_t)2 << 30;
            uint64_t want = S->cfg.hbm_budget_bytes > held ? S->cfg.hbm_budget_bytes - held : 0;
            want = std::min<uint64_t>(want, fr > margin ? fr - margin : 0);
            void *p = nullptr;
            if (want >= ((uint64_t)64 << 20)) {
                if (cudaMallocAsync(&p, want, S->lanes[0].st) == cudaSuccess) {
                    cudaFreeAsync(p, S->lanes[0].st);
                    cudaStreamSynchronize(S->lanes[0].st);
                } else {
                    (void)cudaGetLastError();  // the pool grows on demand instead
                }
            }
        } else {
            (void)cudaGetLastError();
        }
    }
    // page-locked arenas sized for typical batches up front: growing one later
    // frees the old arena, which waits for the whole device
    for (Lane &L : S->lanes) {
        L.in.ensure((size_t)SERVER_IN_ARENA);
        L.aux.ensure((size_t)SERVER_AUX_ARENA);
    }
    S->max_slabs = (size_t)cfg->lanes + 4;
    for (size_t i = 0; i < S->max_slabs; ++i) {
        Slab *sl = new Slab();
        sl->mem.ensure((size_t)SERVER_SLAB);
        S->slabs_all.push_back(sl);
        S->slabs_free.push_back(sl);
    }
    for (Lane &L : S->lanes) L.worker = std::thread(lane_worker, S, &L);
    *out = S;
    return FNEC_OK;
}

int fnec_server_destroy(fnec_server *S) {
    if (!S) return FNEC_ERR_BAD_ARG;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        S->stop = true;
    }
    S->work_cv.notify_all();
    for (Lane &L : S->lanes)
        if (L.worker.joinable()) L.worker.join();
    cudaSetDevice(S->device);
    for (Lane &L : S->lanes) {
        cudaStreamSynchronize(L.st);
        L.in.release();
        L.aux.release();
        cudaEventDestroy(L.done);
        cudaStreamDestroy(L.st);
    }
    for (auto &kv : S->live) delete kv.second;
    for (Slab *sl : S->slabs_all) {
        sl->mem.release();
        delete sl;
    }
    delete S;
    return FNEC_OK;
}

int fnec_request_shape(fnec_ctx *ctx, const fnec_antenna *req, int32_t precision, fnec_request_info *out) {
    if (!ctx || !req || !out) return FNEC_ERR_BAD_ARG;
    HostAnt h;
    std::string why;
    int st = antenna_from_cards(*req, h, why);
    if (st != FNEC_OK) return fail(ctx, st, why);
    out->n_segments = (uint32_t)h.segs.size();
    out->n_rhs = (uint32_t)std::max<size_t>(h.rhs_srcs.size(), 1);
    out->n_solves = out->n_rhs * (uint32_t)h.freqs.size();
    uint32_t fr = 0;
    for (auto &v : h.rhs_feeds) fr += (uint32_t)v.size();
    out->n_feed_rows = fr * (uint32_t)h.freqs.size();
    out->n_points = h.rp.pts_off >= 0 ? (uint32_t)(h.pts.size() / 2) : (uint32_t)(h.rp.n_theta * h.rp.n_phi);
    out->pad = 0;
    out->device_bytes = (uint64_t)request_bytes(h, precision);
    return FNEC_OK;
}

int fnec_server_submit(fnec_server *S, const fnec_antenna *req, const fnec_request_out *out, uint64_t *ticket,
                       fnec_request_info *info) {
    if (!S || !req || !ticket) return FNEC_ERR_BAD_ARG;
    ServerReq *r = new ServerReq();
    std::string why;
    int st = antenna_from_cards(*req, r->host, why);
    if (st != FNEC_OK) {
        delete r;
        return st;
    }
    if (out) {
        r->out = *out;
        r->copy_out = true;
    }
    const HostAnt &h = r->host;
    r->n = (uint32_t)h.segs.size();
    r->s = r->n + (uint32_t)h.cols();
    r->n_solves = (uint32_t)(std::max<size_t>(h.rhs_srcs.size(), 1) * h.freqs.size());
    r->n_points = h.rp.pts_off >= 0 ? (uint32_t)(h.pts.size() / 2) : (uint32_t)(h.rp.n_theta * h.rp.n_phi);
    uint32_t fr = 0;
    for (auto &v : h.rhs_feeds) fr += (uint32_t)v.size();
    r->n_feed_rows = fr * (uint32_t)h.freqs.size();
    r->status.assign(r->n_solves, 0);
    r->bytes = request_bytes(h, S->cfg.precision);
    if (info) {
        info->n_segments = r->n;
        info->n_rhs = (uint32_t)std::max<size_t>(h.rhs_srcs.size(), 1);
        info->n_solves = r->n_solves;
        info->n_feed_rows = r->n_feed_rows;
        info->n_points = r->n_points;
        info->pad = 0;
        info->device_bytes = (uint64_t)r->bytes;
    }
    if (r->bytes > (int64_t)S->cfg.hbm_budget_bytes) {
        delete r;
        return FNEC_ERR_TOO_LARGE;
    }
    {
        std::lock_guard<std::mutex> lk(S->mu);
        if (S->queue.size() >= S->cfg.queue_cap) {
            delete r;
            return FNEC_ERR_BUSY;
        }
        r->ticket = S->next_ticket++;
        r->t_submit = Clock::now();
        S->queue.push_back(r);
        S->live[r->ticket] = r;
        ++S->submitted;
        *ticket = r->ticket;
    }
    S->work_cv.notify_one();
    return FNEC_OK;
}

int fnec_server_poll(fnec_server *S, uint64_t ticket, int32_t *state, double *latency_ms) {
    if (!S || !state) return FNEC_ERR_BAD_ARG;
    std::lock_guard<std::mutex> lk(S->mu);
    auto it = S->live.find(ticket);
    if (it == S->live.end()) return FNEC_ERR_BAD_ARG;
    ServerReq *r = it->second;
    *state = r->state;
    if (finished(r) && latency_ms)
        *latency_ms = std::chrono::duration<double, std::milli>(r->t_done - r->t_submit).count();
    return FNEC_OK;
}

int fnec_server_wait(fnec_server *S, uint64_t ticket, double timeout_ms, int32_t *state, double *latency_ms) {
    if (!S || !state) return FNEC_ERR_BAD_ARG;
    std::unique_lock<std::mutex> lk(S->mu);
    auto it = S->live.find(ticket);
    if (it == S->live.end()) return FNEC_ERR_BAD_ARG;
    ServerReq *r = it->second;
    const auto until = Clock::now() + std::chrono::microseconds((int64_t)(timeout_ms * 1000.0));
    while (!finished(r)) {
        if (S->done_cv.wait_until(lk, until) == std::cv_status::timeout && !finished(r)) {
            *state = r->state;
            return FNEC_ERR_TIMEOUT;
        }
    }
    *state = r->state;
    if (latency_ms) *latency_ms = std::chrono::duration<double, std::milli>(r->t_done - r->t_submit).count();
    return FNEC_OK;
}

int fnec_server_next_done(fnec_server *S, double timeout_ms, uint64_t *ticket) {
    if (!S || !ticket) return FNEC_ERR_BAD_ARG;
    std::unique_lock<std::mutex> lk(S->mu);
    const auto until = Clock::now() + std::chrono::microseconds((int64_t)(timeout_ms * 1000.0));
    for (;;) {
        while (!S->done_q.empty() && !S->live.count(S->done_q.front())) S->done_q.pop_front();  // released
        if (!S->done_q.empty()) break;
        if (S->done_cv.wait_until(lk, until) == std::cv_status::timeout) {
            while (!S->done_q.empty() && !S->live.count(S->done_q.front())) S->done_q.pop_front();
            if (S->done_q.empty()) return FNEC_ERR_TIMEOUT;
            break;
        }
    }
    *ticket = S->done_q.front();
    S->done_q.pop_front();
    return FNEC_OK;
}

int fnec_server_result(fnec_server *S, uint64_t ticket, fnec_request_result *out) {
    if (!S || !out) return FNEC_ERR_BAD_ARG;
    std::lock_guard<std::mutex> lk(S->mu);
    auto it = S->live.find(ticket);
    if (it == S->live.end()) return FNEC_ERR_BAD_ARG;
    ServerReq *r = it->second;
    if (!finished(r)) return FNEC_ERR_BUSY;
    std::memset(out, 0, sizeof(*out));
    out->n_solves = r->n_solves;
    out->n_segments = r->n;
    out->n_feed_rows = r->n_feed_rows;
    out->n_points = r->n_points;
    out->status = r->status.data();
    if (r->slab && r->state == FNEC_REQ_DONE) {
        const unsigned char *base = r->slab->mem.p;
        out->currents = (const double *)(base + sizeof(cx) * r->x_off);
        out->cur_stride = r->s;
        out->feeds = (const double *)(base + r->hf_off + sizeof(double) * 7 * r->feed_row);
        out->pattern = r->n_points ? (const double *)(base + r->hp_off + sizeof(double) * PAT_STRIDE * r->pat_row)
                                   : nullptr;
    }
    return FNEC_OK;
}

int fnec_server_release(fnec_server *S, uint64_t ticket) {
    if (!S) return FNEC_ERR_BAD_ARG;
    std::lock_guard<std::mutex> lk(S->mu);
    auto it = S->live.find(ticket);
    if (it == S->live.end()) return FNEC_ERR_BAD_ARG;
    ServerReq *r = it->second;
    if (!finished(r)) return FNEC_ERR_BUSY;
    const bool freed = r->slab && r->slab->refs == 1;
    slab_unref(S, r->slab);
    S->live.erase(it);
    delete r;
    if (freed) S->work_cv.notify_all();  // a lane may be waiting for a slab
    return FNEC_OK;
}

int fnec_server_stats(fnec_server *S, fnec_server_stats_t *out, int32_t reset) {
    if (!S || !out) return FNEC_ERR_BAD_ARG;
    std::lock_guard<std::mutex> lk(S->mu);
    std::vector<double> v = S->lat_ms;
    std::sort(v.begin(), v.end());
    auto pct = [&](double q) {
        if (v.empty()) return 0.0;
        double i = std::ceil(q * (double)v.size()) - 1.0;
        return v[(size_t)std::min<double>((double)v.size() - 1, std::max(0.0, i))];
    };
    out->submitted = S->submitted;
    out->completed = S->completed;
    out->failed = S->failed;
    out->solves = S->solves;
    out->batches = S->batches;
    out->queued = S->queue.size();
    out->in_flight_bytes = (uint64_t)std::max<int64_t>(S->in_flight, 0);
    out->peak_in_flight_bytes = (uint64_t)S->peak_bytes;
    out->max_batch = S->max_batch_seen;
    out->kernel_launches = S->launches;
    out->h2d_bytes = S->h2d;
    out->d2h_bytes = S->d2h;
    out->plan_ms = S->plan_ms;
    out->launch_ms = S->launch_ms;
    out->collect_ms = S->collect_ms;
    out->alloc_ms = S->alloc_ms;
    out->alloc_device_ms = S->t_dev;
    out->alloc_upload_ms = S->t_copy;
    out->alloc_pinned_ms = S->t_pinned;
    out->alloc_mixed_ms = S->t_mixed;
    out->p50_ms = pct(0.50);
    out->p99_ms = pct(0.99);
    out->max_ms = v.empty() ? 0.0 : v.back();
    double sum = 0;
    for (double x : v) sum += x;
    out->mean_ms = v.empty() ? 0.0 : sum / (double)v.size();
    if (reset) {
        S->lat_ms.clear();
        S->submitted = S->completed = S->failed = S->solves = S->batches = S->launches = S->h2d = S->d2h = 0;
        S->peak_bytes = S->in_flight;
        S->max_batch_seen = 0;
        S->plan_ms = S->launch_ms = S->collect_ms = S->alloc_ms = 0;
        S->t_dev = S->t_copy = S->t_pinned = S->t_mixed = 0;
    }
    return FNEC_OK;
}

const char *fnec_server_last_error(fnec_server *S) {
    if (!S) return "";
    std::lock_guard<std::mutex> lk(S->mu);
    S->err_copy = S->last_err;
    return S->err_copy.c_str();
}

// ---- self-tests of the failure paths (no counterpart in the reference) -----

extern "C" int fnec_selftest_wait_timeout(int32_t device, int32_t which, uint64_t wait_ns, int32_t *unit_status,
                                          double *elapsed_ms) {
    if (!unit_status || wait_ns == 0 || wait_ns > 2000000000ull) return FNEC_ERR_BAD_ARG;
    *unit_status = 0;
    if (elapsed_ms) *elapsed_ms = 0.0;
    switch (which) {
    case 0: return fnec::selftest_grid_timeout(device, 8, 3, wait_ns, unit_status, elapsed_ms);
    case 1: return fnec::selftest_grid_timeout(device, 8, -1, wait_ns, unit_status, elapsed_ms);
    case 2: {
        if (cudaSetDevice(device) != cudaSuccess) return FNEC_ERR_NO_DEVICE;
        const auto t0 = std::chrono::steady_clock::now();
        int rc = fnec::selftest_tc_timeout(device, wait_ns, unit_status);
        if (elapsed_ms)
            *elapsed_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        return rc;
    }
    default: return FNEC_ERR_BAD_ARG;
    }
}

extern "C" int fnec_test_fail_device_allocation(int32_t after) {
    if (after < -1) return FNEC_ERR_BAD_ARG;
    g_fail_alloc_after.store(after);
    return FNEC_OK;
}

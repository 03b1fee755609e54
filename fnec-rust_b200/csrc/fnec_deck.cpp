// fnec_deck.cpp -- the deck reader and the report contract v1 writer: a NEC
// deck's text in, the CLI's per-frequency text report out, with every solve
// on the device through the library's own C ABI.
//
//   fnec_deck_parse   nec_parser::parse (crates/nec_parser/src/lib.rs:78-418):
//                     CM CE GW GE GM GR GN EX FR RP NE NH LD TL NT PT EN; other
//                     mnemonics are counted as warnings and skipped, a bad or
//                     missing field is the first fatal error ("line N: ...").
//   fnec_deck_solve   the deck -> fnec_antenna mapping of the CLI
//                     (geometry.rs:71-110 ground, solve_session.rs:984-1011 FR,
//                     main.rs:292-304 RP points, solve_session.rs:645-688
//                     NE/NH points), one batch over all FR frequencies, then
//                     nec_report::render_text_report (crates/nec_report/src/
//                     lib.rs:307-484) per frequency, the reports separated by a
//                     blank line as main.rs:356-360 prints them.
//
// Host code built without FMA contraction: the few values formed here (FR
// frequencies, RP / NE points, the normalised pattern, the average power
// gain) take the reference's operations in its order.  Numbers are printed
// as Rust's {:.N} and {:.Ne} print them: %.Nf / %.Ne digits (both exact
// decimal expansions with ties to even), Rust's exponent form (e-3, e2),
// NaN / inf / -inf.
#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <stdexcept>
#include <string>
#include <vector>

#include "fnec_cuda.h"

namespace {

constexpr double PI_D = 3.14159265358979323846;

struct ExCard {
    uint32_t type, tag, seg, i4;
    double vr, vi, f3, f4, f5, f6;
};
struct FrCard {
    uint32_t step_type, steps;
    double f_mhz, step_mhz;
};
struct RpCard {
    uint32_t mode, n_theta, n_phi;
    double theta0, phi0, d_theta, d_phi;
    bool normalize, avg_power_gain;
};
struct NeCard {
    bool magnetic;
    uint32_t coord, nx, ny, nz;
    double x0, y0, z0, dx, dy, dz;
};
struct GnCard {
    int32_t type;
};

// ---- field grammar (nec_parser/src/lib.rs:424-485) ------------------------

// Rust's f64::from_str: an optional sign, decimal digits with an optional
// point and exponent, or inf / infinity / nan; nothing else (no hex, no
// surrounding blanks).
bool parse_f64(const std::string &t, double &v) {
    if (t.empty()) return false;
    size_t i = (t[0] == '+' || t[0] == '-') ? 1 : 0;
    std::string body = t.substr(i);
    std::string low;
    for (char c : body) low += (char)std::tolower((unsigned char)c);
    if (low == "inf" || low == "infinity" || low == "nan") {
        v = low == "nan" ? std::nan("") : (t[0] == '-' ? -INFINITY : INFINITY);
        return true;
    }
    bool digits = false, point = false, exp = false;
    for (size_t k = i; k < t.size(); ++k) {
        const char c = t[k];
        if (std::isdigit((unsigned char)c)) {
            digits = true;
        } else if (c == '.' && !point && !exp) {
            point = true;
        } else if ((c == 'e' || c == 'E') && digits && !exp) {
            exp = true;
            if (k + 1 < t.size() && (t[k + 1] == '+' || t[k + 1] == '-')) ++k;
            if (k + 1 >= t.size() || !std::isdigit((unsigned char)t[k + 1])) return false;
        } else {
            return false;
        }
    }
    if (!digits) return false;
    char *end = nullptr;
    v = std::strtod(t.c_str(), &end);
    return end && *end == '\0';
}

// `v as u32` / `as i32` / `as i64`: truncation, NaN -> 0, saturation.
uint32_t sat_u32(double v) {
    if (std::isnan(v) || v <= 0.0) return 0;
    if (v >= 4294967295.0) return 4294967295u;
    return (uint32_t)v;
}
int32_t sat_i32(double v) {
    if (std::isnan(v)) return 0;
    if (v <= -2147483648.0) return INT32_MIN;
    if (v >= 2147483647.0) return INT32_MAX;
    return (int32_t)v;
}
int64_t sat_i64(double v) {
    if (std::isnan(v)) return 0;
    if (v <= -9223372036854775808.0) return INT64_MIN;
    if (v >= 9223372036854775807.0) return INT64_MAX;
    return (int64_t)v;
}
// u32::from_str: an optional '+', decimal digits, no overflow.
bool parse_u32_int(const std::string &t, uint32_t &v) {
    size_t i = (!t.empty() && t[0] == '+') ? 1 : 0;
    if (i >= t.size()) return false;
    uint64_t acc = 0;
    for (size_t k = i; k < t.size(); ++k) {
        if (!std::isdigit((unsigned char)t[k])) return false;
        acc = acc * 10 + (uint64_t)(t[k] - '0');
        if (acc > 4294967295ull) return false;
    }
    v = (uint32_t)acc;
    return true;
}

std::vector<std::string> split_ws(const std::string &s) {
    std::vector<std::string> out;
    size_t i = 0;
    while (i < s.size()) {
        while (i < s.size() && std::isspace((unsigned char)s[i])) ++i;
        size_t j = i;
        while (j < s.size() && !std::isspace((unsigned char)s[j])) ++j;
        if (j > i) out.push_back(s.substr(i, j - i));
        i = j;
    }
    return out;
}

// ---- Rust float formatting -------------------------------------------------
std::string rfix(double v, int prec) {
    if (std::isnan(v)) return "NaN";
    if (std::isinf(v)) return v > 0 ? "inf" : "-inf";
    std::vector<char> b(400);
    std::snprintf(b.data(), b.size(), "%.*f", prec, v);
    return std::string(b.data());
}
std::string rexp(double v, int prec) {
    if (std::isnan(v)) return "NaN";
    if (std::isinf(v)) return v > 0 ? "inf" : "-inf";
    char b[64];
    std::snprintf(b, sizeof b, "%.*e", prec, v);
    std::string s(b);
    const size_t e = s.find('e');
    return s.substr(0, e) + "e" + std::to_string(std::atoi(s.c_str() + e + 1));
}

// compiler-rt __powidf2 (binary exponentiation), which Rust's f64::powi
// lowers to: the FR multiplicative steps (solve_session.rs:1003)
double powi(double a, int b) {
    const bool recip = b < 0;
    double r = 1.0;
    for (;;) {
        if (b & 1) r *= a;
        b /= 2;
        if (b == 0) break;
        a *= a;
    }
    return recip ? 1.0 / r : r;
}

}  // namespace

struct fnec_deck {
    // cards in deck order
    std::vector<fnec_wire> wires;
    std::vector<GnCard> gn;
    std::vector<int32_t> ge;
    bool transforms = false;  // GM / GR
    std::vector<ExCard> ex;
    std::vector<FrCard> fr;
    std::vector<RpCard> rp;
    std::vector<NeCard> ne;
    std::vector<fnec_load> loads;
    std::vector<fnec_tl> tls;
    std::vector<std::vector<std::string>> nt_raw, pt_raw;
    uint32_t warnings = 0;
    std::string first_warning;
    // the antenna view (views into these vectors)
    std::vector<fnec_source> sources;
    std::vector<fnec_nt> nts;
    std::vector<double> freqs, rp_pts;
    fnec_rp_card rp1{};
    fnec_plane_wave pw{};
    bool has_pw = false;
    int32_t ground = FNEC_GROUND_FREE;
    std::string unsupported;  // why the device path cannot run this deck ("" if it can)
    std::string report;
};

namespace {

std::string upper(std::string s) {
    for (auto &c : s) c = (char)std::toupper((unsigned char)c);
    return s;
}

// fatal field errors, in the reference's wording
struct Fatal {
    std::string msg;
};

// A deck whose expanded grids exceed the built maxima (FNEC_DECK_MAX_*).
struct TooLarge {
    std::string msg;
};

void need(size_t line, const char *card, const std::vector<std::string> &f, size_t n) {
    if (f.size() < n)
        throw Fatal{"line " + std::to_string(line) + ": " + card + " needs " + std::to_string(n) + " fields, got " +
                    std::to_string(f.size())};
}
double fld(size_t line, const char *card, size_t field, const std::string &raw) {
    double v;
    if (!parse_f64(raw, v))
        throw Fatal{"line " + std::to_string(line) + ": " + card + " field " + std::to_string(field) +
                    ": cannot parse '" + raw + "'"};
    return v;
}

void parse_text(fnec_deck &d, const char *text) {
    // str::lines: '\n' separated, a trailing '\r' dropped
    std::vector<std::string> lines;
    {
        const char *p = text;
        while (*p) {
            const char *q = std::strchr(p, '\n');
            std::string ln = q ? std::string(p, q - p) : std::string(p);
            if (!ln.empty() && ln.back() == '\r') ln.pop_back();
            lines.push_back(ln);
            if (!q) break;
            p = q + 1;
        }
    }
    for (size_t idx = 0; idx < lines.size(); ++idx) {
        const size_t no = idx + 1;
        const std::vector<std::string> tok = split_ws(lines[idx]);
        if (tok.empty()) continue;
        const std::string m = upper(tok[0]);
        const std::vector<std::string> f(tok.begin() + 1, tok.end());
        const char *c = m.c_str();
        if (m == "CM" || m == "CE") continue;
        if (m == "GW") {
            need(no, c, f, 9);
            fnec_wire w{};
            w.tag = sat_u32(fld(no, c, 1, f[0]));
            w.segments = sat_u32(fld(no, c, 2, f[1]));
            for (int k = 0; k < 3; ++k) {
                w.start[k] = fld(no, c, 3 + k, f[2 + k]);
                w.end[k] = fld(no, c, 6 + k, f[5 + k]);
            }
            w.radius = fld(no, c, 9, f[8]);
            d.wires.push_back(w);
        } else if (m == "GE") {
            d.ge.push_back(f.empty() ? 0 : sat_i32(fld(no, c, 1, f[0])));
        } else if (m == "GM") {
            need(no, c, f, 9);
            for (size_t k = 0; k < 9; ++k) fld(no, c, k + 1, f[k]);
            d.transforms = true;
        } else if (m == "GR") {
            need(no, c, f, 3);
            for (size_t k = 0; k < 3; ++k) fld(no, c, k + 1, f[k]);
            d.transforms = true;
        } else if (m == "GN") {
            need(no, c, f, 1);
            if (f.size() > 4) fld(no, c, 5, f[4]);
            if (f.size() > 5) fld(no, c, 6, f[5]);
            d.gn.push_back({sat_i32(fld(no, c, 1, f[0]))});
        } else if (m == "EX") {
            need(no, c, f, 4);
            ExCard e{};
            const double vr = f.size() > 4 ? fld(no, c, 5, f[4]) : 0.0;
            const double vi = f.size() > 5 ? fld(no, c, 6, f[5]) : 0.0;
            const double f3 = f.size() > 6 ? fld(no, c, 7, f[6]) : 0.0;
            const double f4 = f.size() > 7 ? fld(no, c, 8, f[7]) : 0.0;
            const double f5 = f.size() > 8 ? fld(no, c, 9, f[8]) : 0.0;
            const double f6 = f.size() > 9 ? fld(no, c, 10, f[9]) : 0.0;
            e.type = sat_u32(fld(no, c, 1, f[0]));
            e.tag = sat_u32(fld(no, c, 2, f[1]));
            e.seg = sat_u32(fld(no, c, 3, f[2]));
            e.i4 = sat_u32(fld(no, c, 4, f[3]));
            e.vr = vr, e.vi = vi, e.f3 = f3, e.f4 = f4, e.f5 = f5, e.f6 = f6;
            d.ex.push_back(e);
        } else if (m == "NE" || m == "NH") {
            need(no, c, f, 4);
            auto g = [&](size_t i) { return f.size() > i ? fld(no, c, i + 1, f[i]) : 0.0; };
            NeCard n{};
            n.magnetic = m == "NH";
            n.coord = sat_u32(fld(no, c, 1, f[0]));
            n.nx = sat_u32(fld(no, c, 2, f[1]));
            n.ny = sat_u32(fld(no, c, 3, f[2]));
            n.nz = sat_u32(fld(no, c, 4, f[3]));
            n.x0 = g(4), n.y0 = g(5), n.z0 = g(6), n.dx = g(7), n.dy = g(8), n.dz = g(9);
            d.ne.push_back(n);
        } else if (m == "FR") {
            need(no, c, f, 4);
            const size_t fi = f.size() >= 6 ? 4 : 2, si = f.size() >= 6 ? 5 : 3;
            FrCard r{};
            r.step_type = sat_u32(fld(no, c, 1, f[0]));
            r.steps = sat_u32(fld(no, c, 2, f[1]));
            r.f_mhz = fld(no, c, fi + 1, f[fi]);
            r.step_mhz = fld(no, c, si + 1, f[si]);
            d.fr.push_back(r);
        } else if (m == "RP") {
            need(no, c, f, 7);
            const size_t a = f.size() >= 8 ? 4 : 3;
            RpCard r{};
            if (f.size() >= 8) {
                const uint32_t xnda = sat_u32(fld(no, c, 4, f[3]));
                r.normalize = (xnda / 1000) % 10 != 0;
                r.avg_power_gain = xnda % 10 != 0;
            }
            r.mode = sat_u32(fld(no, c, 1, f[0]));
            r.n_theta = sat_u32(fld(no, c, 2, f[1]));
            r.n_phi = sat_u32(fld(no, c, 3, f[2]));
            r.theta0 = fld(no, c, a + 1, f[a]);
            r.phi0 = fld(no, c, a + 2, f[a + 1]);
            r.d_theta = fld(no, c, a + 3, f[a + 2]);
            r.d_phi = fld(no, c, a + 4, f[a + 3]);
            d.rp.push_back(r);
        } else if (m == "LD") {
            need(no, c, f, 4);
            fnec_load l{};
            l.f1 = f.size() > 4 ? fld(no, c, 5, f[4]) : 0.0;
            l.f2 = f.size() > 5 ? fld(no, c, 6, f[5]) : 0.0;
            l.f3 = f.size() > 6 ? fld(no, c, 7, f[6]) : 0.0;
            l.load_type = sat_i32(fld(no, c, 1, f[0]));
            l.tag = sat_u32(fld(no, c, 2, f[1]));
            l.seg_first = sat_u32(fld(no, c, 3, f[2]));
            l.seg_last = sat_u32(fld(no, c, 4, f[3]));
            d.loads.push_back(l);
        } else if (m == "TL") {
            need(no, c, f, 8);
            fnec_tl t{};
            t.f3 = f.size() > 8 ? fld(no, c, 9, f[8]) : 1.0;
            t.tag1 = sat_u32(fld(no, c, 1, f[0]));
            t.seg1 = sat_u32(fld(no, c, 2, f[1]));
            t.tag2 = sat_u32(fld(no, c, 3, f[2]));
            t.seg2 = sat_u32(fld(no, c, 4, f[3]));
            t.num_segments = sat_u32(fld(no, c, 5, f[4]));
            t.tl_type = sat_u32(fld(no, c, 6, f[5]));
            t.z0 = fld(no, c, 7, f[6]);
            t.length = fld(no, c, 8, f[7]);
            d.tls.push_back(t);
        } else if (m == "NT") {
            d.nt_raw.push_back(f);
        } else if (m == "PT") {
            d.pt_raw.push_back(f);
        } else if (m == "EN") {
            break;
        } else {
            if (d.warnings == 0) d.first_warning = "line " + std::to_string(no) + ": unknown card '" + tok[0] + "'";
            ++d.warnings;
        }
    }
}

// The deck as one antenna of the device path; `unsupported` says why not.
void build_view(fnec_deck &d) {
    d.unsupported.clear();
    auto refuse = [&](const std::string &why) {
        if (d.unsupported.empty()) d.unsupported = why;
    };
    if (d.wires.empty()) refuse("deck contains no GW (wire) cards");
    if (d.transforms) refuse("GM / GR geometry transforms are not built");
    // geometry.rs:71-110: the first GN card, else a GE flag of 1
    if (!d.gn.empty()) {
        const int32_t t = d.gn[0].type;
        if (t == -1) d.ground = FNEC_GROUND_FREE;
        else if (t == 1) d.ground = FNEC_GROUND_PEC;
        else refuse("GN " + std::to_string(t) + ": only free space (GN -1) and PEC (GN 1) grounds are built");
    } else {
        d.ground = FNEC_GROUND_FREE;
        for (int32_t g : d.ge)
            if (g == 1) d.ground = FNEC_GROUND_PEC;
    }
    d.sources.clear();
    d.has_pw = false;
    for (const ExCard &e : d.ex) {
        if (e.type == 0 || e.type == 5) {
            d.sources.push_back({e.tag, e.seg, e.vr, e.vi});
        } else if (e.type >= 1 && e.type <= 3) {
            if (!d.has_pw) {  // the first plane-wave card (planewave.rs:167-174)
                d.pw = fnec_plane_wave{};
                d.pw.ex_type = e.type;
                d.pw.n_theta = std::max<uint32_t>(e.tag, 1);
                d.pw.n_phi = std::max<uint32_t>(e.seg, 1);
                d.pw.theta0 = e.vr;
                d.pw.phi0 = e.vi;
                d.pw.eta = e.f3;
                d.pw.d_theta = e.f4;
                d.pw.d_phi = e.f5;
                d.pw.axial_ratio = e.f6;
                d.has_pw = true;
            }
        } else if (e.type == 4) {
            refuse("EX 4 current sources are not built");
        } else {
            refuse("EX type " + std::to_string(e.type) + " is not an excitation the device path builds");
        }
    }
    if (d.has_pw && !d.sources.empty()) refuse("a deck with both voltage and plane-wave EX cards is not built");
    // solve_session.rs:984-1011 (the first FR card)
    d.freqs.clear();
    if (!d.fr.empty()) {
        const FrCard &r = d.fr[0];
        const uint32_t steps = std::max<uint32_t>(r.steps, 1);
        if (steps > FNEC_DECK_MAX_FREQS && r.step_type <= 1)
            throw TooLarge{"FR card asks for " + std::to_string(steps) + " frequencies; at most " +
                           std::to_string(FNEC_DECK_MAX_FREQS) + " are built"};
        for (uint32_t i = 0; i < steps; ++i) {
            if (r.step_type == 0) d.freqs.push_back((r.f_mhz + (double)i * r.step_mhz) * 1e6);
            else if (r.step_type == 1) d.freqs.push_back(r.f_mhz * powi(r.step_mhz, (int)i) * 1e6);
            else {
                d.freqs.push_back(r.f_mhz * 1e6);
                break;
            }
        }
    }
    if (d.freqs.empty()) refuse("deck has no FR card");
    // main.rs:292-304: every RP card's grid, phi outer, theta inner (farfield.rs:677-699)
    d.rp_pts.clear();
    uint64_t rp_total = 0;
    for (const RpCard &r : d.rp)
        rp_total += (uint64_t)std::max<uint32_t>(r.n_theta, 1) * std::max<uint32_t>(r.n_phi, 1);
    if (rp_total > FNEC_DECK_MAX_POINTS)
        throw TooLarge{"RP cards ask for " + std::to_string(rp_total) + " pattern points; at most " +
                       std::to_string(FNEC_DECK_MAX_POINTS) + " are built"};
    uint64_t ne_total = 0;
    for (const NeCard &c : d.ne)
        ne_total += (uint64_t)std::max<uint32_t>(c.nx, 1) * std::max<uint32_t>(c.ny, 1) * std::max<uint32_t>(c.nz, 1);
    if (ne_total > FNEC_DECK_MAX_POINTS)
        throw TooLarge{"NE/NH cards ask for " + std::to_string(ne_total) + " field points; at most " +
                       std::to_string(FNEC_DECK_MAX_POINTS) + " are built"};
    for (const RpCard &r : d.rp) {
        const uint32_t nt = std::max<uint32_t>(r.n_theta, 1), np = std::max<uint32_t>(r.n_phi, 1);
        for (uint32_t ip = 0; ip < np; ++ip) {
            const double phi = r.phi0 + (double)ip * r.d_phi;
            for (uint32_t it = 0; it < nt; ++it) {
                d.rp_pts.push_back(r.theta0 + (double)it * r.d_theta);
                d.rp_pts.push_back(phi);
            }
        }
    }
    if (d.rp.size() == 1) {
        d.rp1 = {d.rp[0].n_theta, d.rp[0].n_phi, d.rp[0].theta0, d.rp[0].phi0, d.rp[0].d_theta, d.rp[0].d_phi};
    }
    // network.rs:59-90: NT cards with all ten fields, integer ends
    d.nts.clear();
    for (const auto &f : d.nt_raw) {
        if (f.size() < 10) continue;
        fnec_nt n{};
        double y[6];
        bool ok = parse_u32_int(f[0], n.tag1) && parse_u32_int(f[1], n.seg1) && parse_u32_int(f[2], n.tag2) &&
                  parse_u32_int(f[3], n.seg2);
        for (int k = 0; k < 6 && ok; ++k) ok = parse_f64(f[4 + k], y[k]);
        if (!ok) continue;
        n.y11_re = y[0], n.y11_im = y[1], n.y12_re = y[2], n.y12_im = y[3], n.y22_re = y[4], n.y22_im = y[5];
        d.nts.push_back(n);
    }
}

void antenna_of(const fnec_deck &d, fnec_antenna &a) {
    std::memset(&a, 0, sizeof a);
    a.wires = d.wires.data();
    a.n_wires = (uint32_t)d.wires.size();
    a.sources = d.sources.empty() ? nullptr : d.sources.data();
    a.n_sources = (uint32_t)d.sources.size();
    a.ground = d.ground;
    a.n_freqs = (uint32_t)d.freqs.size();
    a.freqs_hz = d.freqs.data();
    if (d.rp.size() == 1) {
        a.rp = &d.rp1;
    } else if (!d.rp_pts.empty()) {
        a.rp_points = d.rp_pts.data();
        a.n_rp_points = (uint32_t)(d.rp_pts.size() / 2);
    }
    a.loads = d.loads.empty() ? nullptr : d.loads.data();
    a.n_loads = (uint32_t)d.loads.size();
    a.tls = d.tls.empty() ? nullptr : d.tls.data();
    a.n_tls = (uint32_t)d.tls.size();
    a.nts = d.nts.empty() ? nullptr : d.nts.data();
    a.n_nts = (uint32_t)d.nts.size();
    a.plane_wave = d.has_pw ? &d.pw : nullptr;
}

// solve_session.rs:645-688
void ne_points(const NeCard &n, std::vector<double> &out) {
    const double rad = PI_D / 180.0;
    if (n.coord == 0) {
        for (uint32_t ix = 0; ix < std::max<uint32_t>(n.nx, 1); ++ix)
            for (uint32_t iy = 0; iy < std::max<uint32_t>(n.ny, 1); ++iy)
                for (uint32_t iz = 0; iz < std::max<uint32_t>(n.nz, 1); ++iz) {
                    out.push_back(n.x0 + (double)ix * n.dx);
                    out.push_back(n.y0 + (double)iy * n.dy);
                    out.push_back(n.z0 + (double)iz * n.dz);
                }
    } else {
        for (uint32_t it = 0; it < std::max<uint32_t>(n.nz, 1); ++it) {
            const double th = (n.z0 + (double)it * n.dz) * rad;
            for (uint32_t ip = 0; ip < std::max<uint32_t>(n.ny, 1); ++ip) {
                const double ph = (n.y0 + (double)ip * n.dy) * rad;
                for (uint32_t ir = 0; ir < std::max<uint32_t>(n.nx, 1); ++ir) {
                    const double r = n.x0 + (double)ir * n.dx;
                    out.push_back(r * std::sin(th) * std::cos(ph));
                    out.push_back(r * std::sin(th) * std::sin(ph));
                    out.push_back(r * std::cos(th));
                }
            }
        }
    }
}

}  // namespace

extern "C" {

uint32_t fnec_abi_struct_sizes(uint64_t *out, uint32_t cap) {
    const uint64_t sz[] = {sizeof(fnec_wire),          sizeof(fnec_source),         sizeof(fnec_rp_card),
                           sizeof(fnec_plane_wave),    sizeof(fnec_load),           sizeof(fnec_tl),
                           sizeof(fnec_nt),            sizeof(fnec_antenna),        sizeof(fnec_unit_info),
                           sizeof(fnec_batch_info),    sizeof(fnec_deck_info),      sizeof(fnec_server_config),
                           sizeof(fnec_request_out),   sizeof(fnec_request_info),   sizeof(fnec_request_result),
                           sizeof(fnec_server_stats_t), sizeof(fnec_schedule),      sizeof(fnec_tune_report),
                           sizeof(fnec_zsegment),      sizeof(fnec_gpu_segment),    sizeof(fnec_rp_result),
                           sizeof(fnec_junction)};
    const uint32_t n = (uint32_t)(sizeof sz / sizeof sz[0]);
    for (uint32_t i = 0; i < n && i < cap && out; ++i) out[i] = sz[i];
    return n;
}

int fnec_deck_parse(const char *text, fnec_deck **out, char *err, uint64_t err_cap) {
    if (!text || !out) return FNEC_ERR_BAD_ARG;
    *out = nullptr;
    fnec_deck *d = new (std::nothrow) fnec_deck();
    if (!d) return FNEC_ERR_OUT_OF_MEMORY;
    auto fail = [&](int code, const std::string &msg) {
        if (err && err_cap) {
            std::strncpy(err, msg.c_str(), err_cap - 1);
            err[err_cap - 1] = '\0';
        }
        delete d;
        return code;
    };
    // no C++ exception crosses the C boundary
    try {
        parse_text(*d, text);
        build_view(*d);
    } catch (const Fatal &e) {
        return fail(FNEC_ERR_BAD_ARG, e.msg);
    } catch (const TooLarge &e) {
        return fail(FNEC_ERR_TOO_LARGE, e.msg);
    } catch (const std::bad_alloc &) {
        return fail(FNEC_ERR_OUT_OF_MEMORY, "host memory exhausted while expanding the deck");
    } catch (const std::exception &e) {
        return fail(FNEC_ERR_BAD_ARG, e.what());
    }
    *out = d;
    return FNEC_OK;
}

int fnec_deck_destroy(fnec_deck *d) {
    delete d;
    return FNEC_OK;
}

int fnec_deck_get_info(const fnec_deck *d, fnec_deck_info *out) {
    if (!d || !out) return FNEC_ERR_BAD_ARG;
    std::memset(out, 0, sizeof *out);
    out->n_wires = (uint32_t)d->wires.size();
    out->n_sources = (uint32_t)d->sources.size();
    out->n_ex = (uint32_t)d->ex.size();
    out->n_loads = (uint32_t)d->loads.size();
    out->n_tls = (uint32_t)d->tls.size();
    out->n_nts = (uint32_t)d->nts.size();
    out->n_freqs = (uint32_t)d->freqs.size();
    out->n_rp_cards = (uint32_t)d->rp.size();
    out->n_points = (uint32_t)(d->rp_pts.size() / 2);
    out->n_ne_cards = (uint32_t)d->ne.size();
    out->ground = d->ground;
    out->plane_wave = d->has_pw ? 1 : 0;
    out->warnings = d->warnings;
    out->runnable = d->unsupported.empty() ? 1 : 0;
    std::strncpy(out->why, d->unsupported.empty() ? d->first_warning.c_str() : d->unsupported.c_str(),
                 sizeof out->why - 1);
    return FNEC_OK;
}

int fnec_deck_get_antenna(const fnec_deck *d, fnec_antenna *out, double *freqs) {
    if (!d || !out) return FNEC_ERR_BAD_ARG;
    antenna_of(*d, *out);
    if (freqs)
        for (size_t i = 0; i < d->freqs.size(); ++i) freqs[i] = d->freqs[i];
    return FNEC_OK;
}

static int deck_solve(fnec_ctx *ctx, fnec_deck *d, int32_t precision, const char **report, uint64_t *len);

int fnec_deck_solve(fnec_ctx *ctx, fnec_deck *d, int32_t precision, const char **report, uint64_t *len) {
    // no C++ exception crosses the C boundary
    try {
        return deck_solve(ctx, d, precision, report, len);
    } catch (const std::bad_alloc &) {
        return FNEC_ERR_OUT_OF_MEMORY;
    } catch (const std::exception &) {
        return FNEC_ERR_BAD_ARG;
    }
}

static int deck_solve(fnec_ctx *ctx, fnec_deck *d, int32_t precision, const char **report, uint64_t *len) {
    if (!ctx || !d || !report) return FNEC_ERR_BAD_ARG;
    *report = nullptr;
    if (!d->unsupported.empty()) return FNEC_ERR_UNSUPPORTED;
    fnec_antenna ant;
    antenna_of(*d, ant);
    fnec_batch *b = nullptr;
    int st = fnec_batch_create(ctx, &ant, 1, precision, &b);
    if (st != FNEC_OK) return st;
    auto done = [&](int code) {
        fnec_batch_destroy(b);
        return code;
    };
    st = fnec_batch_run(b);
    if (st == FNEC_OK) st = fnec_batch_sync(b);
    if (st != FNEC_OK) return done(st);
    fnec_batch_info bi{};
    fnec_batch_get_info(b, &bi);
    std::vector<fnec_unit_info> ui(bi.n_units);
    for (uint32_t u = 0; u < bi.n_units; ++u) fnec_batch_get_unit_info(b, u, &ui[u]);
    std::vector<double> cur(2 * std::max<uint64_t>(bi.total_currents, 1)), feeds(7 * std::max<uint64_t>(bi.total_feeds, 1)),
        pat(6 * std::max<uint64_t>(bi.total_points, 1)), recv(3 * (size_t)bi.n_units);
    std::vector<int32_t> status(bi.n_units);
    st = fnec_batch_read(b, cur.data(), feeds.data(), pat.data(), status.data(), nullptr);
    if (st == FNEC_OK && d->has_pw) st = fnec_batch_read_receive(b, recv.data());
    if (st != FNEC_OK) return done(st);
    for (uint32_t u = 0; u < bi.n_units; ++u)
        if (status[u] != 0) return done(FNEC_ERR_SINGULAR);
    // segments (tags, and the near-field geometry)
    uint64_t n = 0;
    fnec_build_geometry(d->wires.data(), (uint32_t)d->wires.size(), nullptr, 0, &n);
    std::vector<fnec_zsegment> zs(n);
    fnec_build_geometry(d->wires.data(), (uint32_t)d->wires.size(), zs.data(), n, &n);
    std::vector<fnec_gpu_segment> gs(n);
    std::vector<uint32_t> seg_tag(n), seg_idx(n);
    {
        uint64_t q = 0;
        for (const fnec_wire &w : d->wires)
            for (uint32_t i = 0; i < w.segments; ++i, ++q) {
                seg_tag[q] = w.tag;
                seg_idx[q] = i + 1;
            }
        for (uint64_t i = 0; i < n; ++i) {
            for (int c = 0; c < 3; ++c) {
                gs[i].midpoint[c] = zs[i].midpoint[c];
                gs[i].direction[c] = zs[i].direction[c];
            }
            gs[i].length = zs[i].length;
        }
    }
    std::vector<double> ne_e, nh_e;
    for (const NeCard &c : d->ne) ne_points(c, c.magnetic ? nh_e : ne_e);
    // solve_session.rs:781-826: the last PT card filters the current table
    int64_t pt_mode = 0, pt_tag = 0, pt_first = 0, pt_last = 0;
    if (!d->pt_raw.empty()) {
        const auto &f = d->pt_raw.back();
        auto g = [&](size_t i) -> int64_t {
            double v;
            return (i < f.size() && parse_f64(f[i], v)) ? sat_i64(v) : 0;
        };
        pt_mode = g(0), pt_tag = g(1), pt_first = g(2), pt_last = g(3);
    }
    const bool normalize = std::any_of(d->rp.begin(), d->rp.end(), [](const RpCard &r) { return r.normalize; });
    const bool avg = std::any_of(d->rp.begin(), d->rp.end(), [](const RpCard &r) { return r.avg_power_gain; });
    const uint32_t per_freq = d->has_pw ? d->pw.n_theta * d->pw.n_phi : 1;
    std::string out;
    for (size_t fi = 0; fi < d->freqs.size(); ++fi) {
        const uint32_t u = (uint32_t)(fi * per_freq);  // the deck's own solve of this frequency
        const fnec_unit_info &x = ui[u];
        const double *I = &cur[2 * x.cur_off];
        std::string r;
        r += "FNEC FEEDPOINT REPORT\nFORMAT_VERSION 1\n";
        r += "FREQ_MHZ " + rfix(x.freq_hz / 1e6, 6) + "\n";
        r += std::string("SOLVER_MODE ") + (d->has_pw ? "hallen-planewave" : "hallen") + "\n";
        r += "PULSE_RHS Nec2\n\nFEEDPOINTS\nTAG SEG V_RE V_IM I_RE I_IM Z_RE Z_IM\n";
        for (uint32_t k = 0; k < x.n_feed; ++k) {
            const double *o = &feeds[7 * (x.feed_off + k)];
            const uint64_t sg = (uint64_t)o[0];
            r += std::to_string(seg_tag[sg]) + " " + std::to_string(seg_idx[sg]);
            for (int c = 1; c < 7; ++c) r += " " + rfix(o[c], 6);
            r += "\n";
        }
        if (!d->ex.empty()) {
            r += "\nSOURCES\nN_SOURCES " + std::to_string(d->ex.size()) + "\nTYPE TAG SEG I4 V_RE V_IM\n";
            for (const ExCard &e : d->ex)
                r += std::to_string(e.type) + " " + std::to_string(e.tag) + " " + std::to_string(e.seg) + " " +
                     std::to_string(e.i4) + " " + rfix(e.vr, 6) + " " + rfix(e.vi, 6) + "\n";
        }
        if (!d->loads.empty()) {
            r += "\nLOADS\nN_LOADS " + std::to_string(d->loads.size()) + "\nTYPE TAG SEG_FIRST SEG_LAST F1 F2 F3\n";
            for (const fnec_load &l : d->loads)
                r += std::to_string(l.load_type) + " " + std::to_string(l.tag) + " " + std::to_string(l.seg_first) +
                     " " + std::to_string(l.seg_last) + " " + rfix(l.f1, 6) + " " + rfix(l.f2, 6) + " " +
                     rfix(l.f3, 6) + "\n";
        }
        std::string rows;
        size_t n_rows = 0;
        if (pt_mode > -1)
            for (uint64_t i = 0; i < n; ++i) {
                if (pt_mode != 0) {
                    const bool tag_ok = pt_tag == 0 || (int64_t)seg_tag[i] == pt_tag;
                    const bool seg_ok = pt_first == 0 || ((int64_t)seg_idx[i] >= pt_first &&
                                                          (pt_last == 0 || (int64_t)seg_idx[i] <= pt_last));
                    if (!(tag_ok && seg_ok)) continue;
                }
                const double re = I[2 * i], im = I[2 * i + 1];
                rows += std::to_string(seg_tag[i]) + " " + std::to_string(seg_idx[i]) + " " + rexp(re, 6) + " " +
                        rexp(im, 6) + " " + rexp(std::hypot(re, im), 6) + " " +
                        rfix(std::atan2(im, re) * (180.0 / PI_D), 4) + "\n";
                ++n_rows;
            }
        if (n_rows) r += "\nCURRENTS\nTAG SEG I_RE I_IM I_MAG I_PHASE\n" + rows;
        const uint32_t np = x.n_points;
        if (np) {
            r += "\nRADIATION_PATTERN\nN_POINTS " + std::to_string(np) + "\nTHETA PHI GAIN_DB GAIN_V_DB GAIN_H_DB AXIAL_RATIO\n";
            for (uint32_t k = 0; k < np; ++k) {
                const double *o = &pat[6 * (x.pat_off + k)];
                r += rfix(d->rp_pts[2 * k], 4) + " " + rfix(d->rp_pts[2 * k + 1], 4) + " " + rfix(o[0], 4) + " " +
                     rfix(o[1], 4) + " " + rfix(o[2], 4) + " " + rfix(o[3], 4) + "\n";
            }
        }
        if (d->has_pw && per_freq > 1) {
            r += "\nRECEIVE_PATTERN\nN_POINTS " + std::to_string(per_freq) + "\nTHETA PHI RESPONSE_DB\n";
            for (uint32_t k = 0; k < per_freq; ++k) {
                const double *o = &recv[3 * (u + k)];
                r += rfix(o[0], 4) + " " + rfix(o[1], 4) + " " + rfix(o[2], 4) + "\n";
            }
        }
        for (int pass = 0; pass < 2; ++pass) {
            const std::vector<double> &pts = pass == 0 ? ne_e : nh_e;
            const uint64_t p = pts.size() / 3;
            if (!p) continue;
            std::vector<double> f(6 * p);
            st = fnec_near_field(ctx, gs.data(), n, I, x.freq_hz, pts.data(), p, pass == 0 ? f.data() : nullptr,
                                 pass == 1 ? f.data() : nullptr);
            if (st != FNEC_OK) return done(st);
            r += pass == 0 ? "\nNEAR_FIELD\nN_POINTS " + std::to_string(p) + "\nX Y Z EX_RE EX_IM EY_RE EY_IM EZ_RE EZ_IM\n"
                           : "\nNEAR_H_FIELD\nN_POINTS " + std::to_string(p) + "\nX Y Z HX_RE HX_IM HY_RE HY_IM HZ_RE HZ_IM\n";
            for (uint64_t k = 0; k < p; ++k) {
                r += rfix(pts[3 * k], 4) + " " + rfix(pts[3 * k + 1], 4) + " " + rfix(pts[3 * k + 2], 4);
                for (int c = 0; c < 6; ++c) r += " " + rexp(f[6 * k + c], 6);
                r += "\n";
            }
        }
        if (normalize && np) {
            double peak = -INFINITY;  // fold(NEG_INFINITY, f64::max): NaN passes over
            for (uint32_t k = 0; k < np; ++k) peak = std::fmax(peak, pat[6 * (x.pat_off + k)]);
            r += "\nNORMALIZED_PATTERN\nN_POINTS " + std::to_string(np) + "\nTHETA PHI GAIN_NORM_DB\n";
            for (uint32_t k = 0; k < np; ++k) {
                const double g = pat[6 * (x.pat_off + k)];
                r += rfix(d->rp_pts[2 * k], 4) + " " + rfix(d->rp_pts[2 * k + 1], 4) + " " +
                     rfix(g > -900.0 ? g - peak : g, 4) + "\n";
            }
        }
        if (avg && np) {  // solve_session.rs:1702-1719
            double num = 0.0, den = 0.0;
            for (uint32_t k = 0; k < np; ++k) {
                const double g = pat[6 * (x.pat_off + k)];
                if (g <= -900.0) continue;
                const double w = std::sin(d->rp_pts[2 * k] * (PI_D / 180.0));
                num += std::pow(10.0, g / 10.0) * w;
                den += w;
            }
            if (den > 0.0) r += "\nAVERAGE_POWER_GAIN " + rfix(num / den, 4) + "\n";
        }
        if (fi > 0) out += "\n";
        out += r;
    }
    fnec_batch_destroy(b);
    d->report = out;
    *report = d->report.c_str();
    if (len) *len = d->report.size();
    return FNEC_OK;
}

}  // extern "C"

/*
 * fnec_oracle.c -- CPU oracle (test infrastructure) for the Hallen MoM path.
 *
 * Restates the reference CPU algorithm of dc0sk/fnec-rust v0.11.0 operation
 * by operation; each function cites the reference file:line it follows.
 * Only the test suite, smoke() and bench.py's CPU arms use this file.
 * Build: see oracle/Makefile (-O2 -ffp-contract=off, glibc libm, pthreads).
 */
#include "fnec_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------- */
/* Constants (matrix.rs:31-33, excitation.rs:19-21, farfield.rs:27-31)       */
/* ------------------------------------------------------------------------- */
#define OR_PI 3.14159265358979323846
static const double C0 = 299792458.0;
static const double RADS_PER_DEG = OR_PI / 180.0; /* Rust f64::to_radians */

/* Gauss-Legendre tables exactly as written in matrix.rs:39-72 (15 digits). */
static const double GL_N4[4] = {-0.861136311594953, -0.339981043584856, 0.339981043584856,
                                0.861136311594953};
static const double GL_W4[4] = {0.347854845137454, 0.652145154862626, 0.652145154862626,
                                0.347854845137454};
static const double GL_N8[8] = {-0.960289856497536, -0.796666477413627, -0.525532409916329,
                                -0.183434642495650, 0.183434642495650,  0.525532409916329,
                                0.796666477413627,  0.960289856497536};
static const double GL_W8[8] = {0.101228536290376, 0.222381034453374, 0.313706645877887,
                                0.362683783378362, 0.362683783378362, 0.313706645877887,
                                0.222381034453374, 0.101228536290376};

/* ------------------------------------------------------------------------- */
/* num-complex 0.4.6 arithmetic                                              */
/* ------------------------------------------------------------------------- */
typedef struct {
    double re, im;
} c64;
static inline c64 cmk(double re, double im) {
    c64 c = {re, im};
    return c;
}
static inline c64 cadd(c64 a, c64 b) { return cmk(a.re + b.re, a.im + b.im); }
static inline c64 csub(c64 a, c64 b) { return cmk(a.re - b.re, a.im - b.im); }
static inline c64 cmul(c64 a, c64 b) {
    return cmk(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re);
}
static inline c64 cdiv(c64 a, c64 b) {
    double ns = b.re * b.re + b.im * b.im;
    double re = a.re * b.re + a.im * b.im;
    double im = a.im * b.re - a.re * b.im;
    return cmk(re / ns, im / ns);
}
static inline c64 cconj(c64 a) { return cmk(a.re, -a.im); }
static inline double cnorm(c64 a) { return hypot(a.re, a.im); }
static inline double cnorm_sqr(c64 a) { return a.re * a.re + a.im * a.im; }
static inline c64 crs(double s, c64 a) { return cmk(s * a.re, s * a.im); }
static inline c64 cdivr(c64 a, double s) { return cmk(a.re / s, a.im / s); }
static inline c64 cld(const double *p) { return cmk(p[0], p[1]); }
static inline void cst(double *p, c64 v) {
    p[0] = v.re;
    p[1] = v.im;
}

static inline double dot3(const double *a, const double *b) {
    return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}

/* ------------------------------------------------------------------------- */
/* Geometry                                                                   */
/* ------------------------------------------------------------------------- */

/* geometry.rs:710-754 expand_wire + :676-704 build_geometry (GW only). */
int64_t or_build_geometry(const or_wire *wires, int64_t nw, or_seg *out, int64_t cap) {
    int64_t n = 0;
    for (int64_t w = 0; w < nw; ++w) {
        const or_wire *gw = &wires[w];
        if (gw->segments == 0) return OR_ERR_ZERO_SEGMENTS;
        double x1 = gw->start[0], y1 = gw->start[1], z1 = gw->start[2];
        double x2 = gw->end[0], y2 = gw->end[1], z2 = gw->end[2];
        double dx = x2 - x1, dy = y2 - y1, dz = z2 - z1;
        double wl = sqrt(dx * dx + dy * dy + dz * dz);
        if (wl == 0.0) return OR_ERR_ZERO_LENGTH;
        double dir[3] = {dx / wl, dy / wl, dz / wl};
        double nn = (double)gw->segments;
        double seg_len = wl / nn;
        for (uint32_t i = 0; i < gw->segments; ++i) {
            if (n >= cap) return OR_ERR_CAPACITY;
            double t0 = (double)i / nn;
            double t1 = ((double)i + 1.0) / nn;
            double tm = (t0 + t1) * 0.5;
            or_seg *s = &out[n++];
            s->tag = gw->tag;
            s->tag_index = i + 1;
            s->start[0] = x1 + dx * t0;
            s->start[1] = y1 + dy * t0;
            s->start[2] = z1 + dz * t0;
            s->end[0] = x1 + dx * t1;
            s->end[1] = y1 + dy * t1;
            s->end[2] = z1 + dz * t1;
            s->mid[0] = x1 + dx * tm;
            s->mid[1] = y1 + dy * tm;
            s->mid[2] = z1 + dz * tm;
            memcpy(s->dir, dir, sizeof dir);
            s->length = seg_len;
            s->radius = gw->radius;
        }
    }
    if (n == 0) return OR_ERR_NO_WIRES;
    return n;
}

/* geometry.rs:168-185 wire_endpoints_from_segs. */
int64_t or_wire_endpoints(const or_seg *segs, int64_t n, int64_t *out, int64_t cap) {
    int64_t cnt = 0;
    uint32_t cur = UINT32_MAX;
    int64_t first = 0;
    for (int64_t i = 0; i < n; ++i) {
        if (segs[i].tag != cur) {
            if (cur != UINT32_MAX) {
                if (cnt < cap) {
                    out[2 * cnt] = first;
                    out[2 * cnt + 1] = i - 1;
                }
                cnt++;
            }
            cur = segs[i].tag;
            first = i;
        }
    }
    if (cur != UINT32_MAX) {
        if (cnt < cap) {
            out[2 * cnt] = first;
            out[2 * cnt + 1] = n - 1;
        }
        cnt++;
    }
    return cnt;
}

static double dist2(const double *a, const double *b) {
    double d0 = a[0] - b[0], d1 = a[1] - b[1], d2 = a[2] - b[2];
    return d0 * d0 + d1 * d1 + d2 * d2;
}

/* geometry.rs:227-236 dir_aligned. */
static int dir_aligned(const double *a, const double *b, double tol) {
    double cr[3] = {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2],
                    a[0] * b[1] - a[1] * b[0]};
    double zero[3] = {0.0, 0.0, 0.0};
    double dot = a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
    return dist2(cr, zero) < tol * tol && dot > 0.0;
}

/* geometry.rs:200-225 merge_collinear_wire_endpoints. */
int64_t or_merge_collinear(const or_seg *segs, int64_t n, int64_t *out, int64_t cap) {
    int64_t nb = or_wire_endpoints(segs, n, NULL, 0);
    int64_t *base = (int64_t *)malloc(sizeof(int64_t) * 2 * (nb > 0 ? nb : 1));
    or_wire_endpoints(segs, n, base, nb);
    int64_t cnt = 0;
    if (nb < 2) {
        for (int64_t i = 0; i < nb; ++i) {
            if (cnt < cap) {
                out[2 * cnt] = base[2 * i];
                out[2 * cnt + 1] = base[2 * i + 1];
            }
            cnt++;
        }
        free(base);
        return cnt;
    }
    const double POS_TOL = 1e-6, DIR_TOL = 1e-6;
    int64_t c0 = base[0], c1 = base[1];
    for (int64_t k = 1; k < nb; ++k) {
        int64_t n0 = base[2 * k], n1 = base[2 * k + 1];
        const or_seg *a = &segs[c1];
        const or_seg *b = &segs[n0];
        int contiguous = (c1 + 1 == n0);
        int connects = dist2(a->end, b->start) < POS_TOL * POS_TOL;
        int collinear = dir_aligned(a->dir, b->dir, DIR_TOL);
        int same_radius = fabs(a->radius - b->radius) < POS_TOL;
        if (contiguous && connects && collinear && same_radius) {
            c1 = n1;
        } else {
            if (cnt < cap) {
                out[2 * cnt] = c0;
                out[2 * cnt + 1] = c1;
            }
            cnt++;
            c0 = n0;
            c1 = n1;
        }
    }
    if (cnt < cap) {
        out[2 * cnt] = c0;
        out[2 * cnt + 1] = c1;
    }
    cnt++;
    free(base);
    return cnt;
}

/* geometry.rs:274-339 detect_wire_junctions. */
int64_t or_detect_junctions(const or_seg *segs, const int64_t *ep, int64_t w, double tol,
                            int64_t *ja, int64_t *jb, double *jsign, int64_t cap) {
    int64_t nn = 2 * w;
    int64_t cnt = 0;
    for (int64_t i = 0; i < nn; ++i) {
        int64_t si = ep[i];
        int starti = (i % 2) == 0;
        const double *pi = starti ? segs[si].start : segs[si].end;
        for (int64_t j = i + 1; j < nn; ++j) {
            int64_t sj = ep[j];
            if (si == sj) continue;
            int startj = (j % 2) == 0;
            const double *pj = startj ? segs[sj].start : segs[sj].end;
            double dx = pi[0] - pj[0], dy = pi[1] - pj[1], dz = pi[2] - pj[2];
            if (sqrt(dx * dx + dy * dy + dz * dz) > tol) continue;
            double sign = (starti == startj) ? 1.0 : -1.0;
            if (cnt < cap) {
                ja[cnt] = si;
                jb[cnt] = sj;
                jsign[cnt] = sign;
            }
            cnt++;
        }
    }
    return cnt;
}

/* solve_session.rs:1386-1400: junctions over merged endpoints, keeping only
 * pairs whose segments lie in different merged components. */
int64_t or_cli_junctions(const or_seg *segs, int64_t n, const int64_t *merged, int64_t w,
                         int64_t *ja, int64_t *jb, double *jsign, int64_t cap) {
    int64_t total = or_detect_junctions(segs, merged, w, 1e-6, NULL, NULL, NULL, 0);
    int64_t *a = (int64_t *)malloc(sizeof(int64_t) * (total + 1));
    int64_t *b = (int64_t *)malloc(sizeof(int64_t) * (total + 1));
    double *s = (double *)malloc(sizeof(double) * (total + 1));
    or_detect_junctions(segs, merged, w, 1e-6, a, b, s, total);
    int64_t *comp = (int64_t *)calloc((size_t)(n > 0 ? n : 1), sizeof(int64_t));
    for (int64_t ci = 0; ci < w; ++ci)
        for (int64_t m = merged[2 * ci]; m <= merged[2 * ci + 1]; ++m) comp[m] = ci;
    int64_t cnt = 0;
    for (int64_t t = 0; t < total; ++t) {
        if (comp[a[t]] == comp[b[t]]) continue;
        if (cnt < cap) {
            ja[cnt] = a[t];
            jb[cnt] = b[t];
            jsign[cnt] = s[t];
        }
        cnt++;
    }
    free(a);
    free(b);
    free(s);
    free(comp);
    return cnt;
}

/* ------------------------------------------------------------------------- */
/* Excitation                                                                 */
/* ------------------------------------------------------------------------- */

static int64_t find_seg(const or_seg *segs, int64_t n, uint32_t tag, uint32_t idx) {
    for (int64_t i = 0; i < n; ++i)
        if (segs[i].tag == tag && segs[i].tag_index == idx) return i;
    return -1;
}

/* excitation.rs:78-90 build_excitation / :450-482 apply_ex. */
int or_excitation(const or_seg *segs, int64_t n, const or_source *src, int64_t ns, double *v) {
    for (int64_t i = 0; i < 2 * n; ++i) v[i] = 0.0;
    for (int64_t e = 0; e < ns; ++e) {
        int64_t idx = find_seg(segs, n, src[e].tag, src[e].segment);
        if (idx < 0) return OR_ERR_SEGMENT_NOT_FOUND;
        c64 add = cdivr(cmk(src[e].v_re, src[e].v_im), segs[idx].length);
        cst(&v[2 * idx], cadd(cld(&v[2 * idx]), add));
    }
    return OR_OK;
}

/* excitation.rs:119-244 build_hallen_rhs. */
int or_hallen_rhs(const or_seg *segs, int64_t n, double freq_hz, const or_source *src,
                  int64_t ns, double *rhs, double *cosv) {
    for (int64_t i = 0; i < n; ++i) {
        rhs[2 * i] = 0.0;
        rhs[2 * i + 1] = 0.0;
        cosv[i] = 0.0;
    }
    if (ns == 0) return OR_OK;
    int64_t feed = find_seg(segs, n, src[0].tag, src[0].segment);
    if (feed < 0) return OR_ERR_SEGMENT_NOT_FOUND;
    const double MU0 = 4.0 * OR_PI * 1e-7;
    const double ETA0 = MU0 * C0;
    double k = 2.0 * OR_PI * freq_hz / C0;
    double scale = 2.0 * OR_PI / ETA0;
    uint32_t driven_tag = segs[feed].tag;

    /* source_by_tag: BTreeMap<tag, (idx, V)>; the driven tag keeps the first
     * source, other tags keep the last one found (insert overwrites). */
    int64_t *s_idx = (int64_t *)malloc(sizeof(int64_t) * (size_t)ns);
    uint32_t *s_tag = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)ns);
    c64 *s_v = (c64 *)malloc(sizeof(c64) * (size_t)ns);
    int64_t nm = 0;
    s_idx[0] = feed;
    s_tag[0] = driven_tag;
    s_v[0] = cmk(src[0].v_re, src[0].v_im);
    nm = 1;
    for (int64_t e = 0; e < ns; ++e) {
        if (src[e].tag == driven_tag) continue;
        int64_t idx = find_seg(segs, n, src[e].tag, src[e].segment);
        if (idx < 0) continue;
        int64_t slot = -1;
        for (int64_t q = 0; q < nm; ++q)
            if (s_tag[q] == src[e].tag) slot = q;
        if (slot < 0) slot = nm++;
        s_tag[slot] = src[e].tag;
        s_idx[slot] = idx;
        s_v[slot] = cmk(src[e].v_re, src[e].v_im);
    }
    /* iterate in ascending tag order (BTreeMap) */
    for (int64_t a = 0; a < nm; ++a)
        for (int64_t b = a + 1; b < nm; ++b)
            if (s_tag[b] < s_tag[a]) {
                uint32_t tt = s_tag[a];
                s_tag[a] = s_tag[b];
                s_tag[b] = tt;
                int64_t ti = s_idx[a];
                s_idx[a] = s_idx[b];
                s_idx[b] = ti;
                c64 tv = s_v[a];
                s_v[a] = s_v[b];
                s_v[b] = tv;
            }

    int64_t ncomp = or_merge_collinear(segs, n, NULL, 0);
    int64_t *comp = (int64_t *)malloc(sizeof(int64_t) * 2 * (size_t)ncomp);
    or_merge_collinear(segs, n, comp, ncomp);
    int64_t *comp_of = (int64_t *)calloc((size_t)n, sizeof(int64_t));
    for (int64_t ci = 0; ci < ncomp; ++ci)
        for (int64_t m = comp[2 * ci]; m <= comp[2 * ci + 1]; ++m) comp_of[m] = ci;

    for (int64_t m = 0; m < n; ++m) {
        int64_t first = comp[2 * comp_of[m]], last = comp[2 * comp_of[m] + 1];
        const double *wd = segs[first].dir;
        double wm[3] = {(segs[first].mid[0] + segs[last].mid[0]) / 2.0,
                        (segs[first].mid[1] + segs[last].mid[1]) / 2.0,
                        (segs[first].mid[2] + segs[last].mid[2]) / 2.0};
        double dl[3] = {segs[m].mid[0] - wm[0], segs[m].mid[1] - wm[1], segs[m].mid[2] - wm[2]};
        double s_local = dl[0] * wd[0] + dl[1] * wd[1] + dl[2] * wd[2];
        cosv[m] = cos(k * s_local);
    }
    for (int64_t q = 0; q < nm; ++q) {
        int64_t fi = s_idx[q];
        c64 vsrc = s_v[q];
        int64_t cf = comp[2 * comp_of[fi]], cl = comp[2 * comp_of[fi] + 1];
        const double *sm = segs[fi].mid;
        const double *sd = segs[fi].dir;
        for (int64_t m = cf; m <= cl; ++m) {
            double d[3] = {segs[m].mid[0] - sm[0], segs[m].mid[1] - sm[1], segs[m].mid[2] - sm[2]};
            double s = d[0] * sd[0] + d[1] * sd[1] + d[2] * sd[2];
            c64 t = cmul(cmk(0.0, -scale * sin(k * fabs(s))), vsrc);
            cst(&rhs[2 * m], cadd(cld(&rhs[2 * m]), t));
        }
    }
    free(s_idx);
    free(s_tag);
    free(s_v);
    free(comp);
    free(comp_of);
    return OR_OK;
}

/* geometry.rs:404-584 build_conductor_paths: wires (per-tag runs) joined
 * through degree-2 endpoint nodes into open chains.  Outputs per segment
 * its path (in path order), traversal sign and signed arc length of its
 * midpoint from the path centre; free_ends holds each path's (first,
 * last) traversed segment.  Returns the number of paths, or -1 where the
 * reference returns None (a node of degree >= 3, a wire closed on itself,
 * a chain without exactly two free ends).  *nontrivial = 1 if some path
 * is not a forward run of ascending segments (ConductorPath::is_trivial). */
static int64_t uf_find(int64_t *parent, int64_t x) {
    int64_t r = x;
    while (parent[r] != r) r = parent[r];
    while (parent[x] != x) {
        int64_t nx = parent[x];
        parent[x] = r;
        x = nx;
    }
    return r;
}

int64_t or_conductor_paths(const or_seg *segs, int64_t n, int64_t *path_of, double *sign,
                           double *s_mid, int64_t *free_ends, int *nontrivial) {
    int64_t w = or_wire_endpoints(segs, n, NULL, 0);
    *nontrivial = 0;
    if (w <= 0) return 0;
    int64_t *ep = (int64_t *)malloc(sizeof(int64_t) * 2 * (size_t)w);
    or_wire_endpoints(segs, n, ep, w);
    const double TOL = 1e-6;
    /* endpoint id = 2 wi + end (0 start of its first segment, 1 end of its last) */
    int64_t ne = 2 * w;
    int64_t *node_of = (int64_t *)malloc(sizeof(int64_t) * (size_t)ne);
    int64_t *node_cnt = (int64_t *)calloc((size_t)ne, sizeof(int64_t));
    int64_t *node_mem = (int64_t *)malloc(sizeof(int64_t) * 2 * (size_t)ne); /* first two members */
    for (int64_t i = 0; i < ne; ++i) node_of[i] = -1;
    int64_t nodes = 0;
    int64_t ret = 0;
#define EP_POINT(id) ((id) % 2 == 0 ? segs[ep[2 * ((id) / 2)]].start : segs[ep[2 * ((id) / 2) + 1]].end)
    for (int64_t id = 0; id < ne; ++id) {
        if (node_of[id] >= 0) continue;
        int64_t nd = nodes++;
        node_of[id] = nd;
        node_mem[2 * nd] = id;
        node_cnt[nd] = 1;
        const double *p = EP_POINT(id);
        for (int64_t j = 0; j < ne; ++j) {
            if (node_of[j] >= 0) continue;
            if (dist2(p, EP_POINT(j)) < TOL * TOL) {
                node_of[j] = nd;
                if (node_cnt[nd] < 2) node_mem[2 * nd + node_cnt[nd]] = j;
                node_cnt[nd]++;
            }
        }
    }
#undef EP_POINT
    int64_t *parent = (int64_t *)malloc(sizeof(int64_t) * (size_t)w);
    int64_t *root = (int64_t *)malloc(sizeof(int64_t) * (size_t)w);
    char *visited = (char *)calloc((size_t)w, 1);
    for (int64_t nd = 0; nd < nodes; ++nd)
        if (node_cnt[nd] >= 3) {
            ret = -1;
            goto done;
        }
    for (int64_t i = 0; i < w; ++i) parent[i] = i;
    for (int64_t nd = 0; nd < nodes; ++nd) {
        if (node_cnt[nd] != 2) continue;
        int64_t a = node_mem[2 * nd] / 2, b = node_mem[2 * nd + 1] / 2;
        if (a == b) {
            ret = -1;
            goto done;
        }
        int64_t ra = uf_find(parent, a), rb = uf_find(parent, b);
        parent[ra] = rb;
    }
    for (int64_t i = 0; i < w; ++i) root[i] = uf_find(parent, i);
    /* components in ascending root order (BTreeMap), wires ascending within */
    for (int64_t r = 0; r < w; ++r) {
        int64_t fe[2], nfe = 0, any = 0;
        for (int64_t wi = 0; wi < w; ++wi) {
            if (root[wi] != r) continue;
            any = 1;
            for (int e = 0; e < 2; ++e)
                if (node_cnt[node_of[2 * wi + e]] == 1) {
                    if (nfe < 2) fe[nfe] = 2 * wi + e;
                    nfe++;
                }
        }
        if (!any) continue;
        if (nfe != 2) {
            ret = -1;
            goto done;
        }
        int64_t pi = ret++;
        int64_t cur = fe[0] / 2, enter = fe[0] % 2;
        double arc = 0.0;
        int64_t first_seg = -1, last_seg = -1, prev = -1, cnt = 0;
        int64_t *walked = (int64_t *)malloc(sizeof(int64_t) * (size_t)(n > 0 ? n : 1));
        for (;;) {
            visited[cur] = 1;
            int64_t f = ep[2 * cur], l = ep[2 * cur + 1];
            double sg = enter == 0 ? 1.0 : -1.0;
            for (int64_t t = 0; t <= l - f; ++t) {
                int64_t m = enter == 0 ? f + t : l - t;
                double half = segs[m].length * 0.5;
                s_mid[m] = arc + half; /* arc length from the path start, re-centred below */
                arc += segs[m].length;
                path_of[m] = pi;
                sign[m] = sg;
                if (sg != 1.0 || (prev >= 0 && m != prev + 1)) *nontrivial = 1;
                if (first_seg < 0) first_seg = m;
                last_seg = m;
                prev = m;
                walked[cnt++] = m;
            }
            int64_t exit_id = 2 * cur + (1 - enter);
            int64_t nd = node_of[exit_id];
            if (node_cnt[nd] == 1) break;
            int64_t nxt = -1;
            for (int q = 0; q < 2; ++q) {
                int64_t mid = node_mem[2 * nd + q];
                if (mid / 2 != cur && !visited[mid / 2]) nxt = mid;
            }
            if (nxt < 0) break;
            cur = nxt / 2;
            enter = nxt % 2;
        }
        for (int64_t t = 0; t < cnt; ++t) s_mid[walked[t]] = s_mid[walked[t]] - arc * 0.5;
        free(walked);
        free_ends[2 * pi] = first_seg;
        free_ends[2 * pi + 1] = last_seg;
    }
done:
    free(ep);
    free(node_of);
    free(node_cnt);
    free(node_mem);
    free(parent);
    free(root);
    free(visited);
    return ret;
}

/* excitation.rs:264-341 build_hallen_rhs_paths: cos(k s) along each path
 * with the traversal sign; every voltage EX card, in deck order, drives
 * its whole path with the sign of its feed segment. */
int or_hallen_rhs_paths(const or_seg *segs, int64_t n, double freq_hz, const or_source *src,
                        int64_t ns, const int64_t *path_of, const double *sign, const double *s_mid,
                        double *rhs, double *cosv) {
    const double MU0 = 4.0 * OR_PI * 1e-7;
    const double ETA0 = MU0 * C0;
    double k = 2.0 * OR_PI * freq_hz / C0;
    double scale = 2.0 * OR_PI / ETA0;
    for (int64_t m = 0; m < n; ++m) {
        cosv[m] = sign[m] * cos(k * s_mid[m]);
        rhs[2 * m] = 0.0;
        rhs[2 * m + 1] = 0.0;
    }
    for (int64_t e = 0; e < ns; ++e) {
        int64_t fi = find_seg(segs, n, src[e].tag, src[e].segment);
        if (fi < 0) return OR_ERR_SEGMENT_NOT_FOUND;
        c64 vsrc = cmk(src[e].v_re, src[e].v_im);
        double feed_sign = sign[fi];
        for (int64_t m = 0; m < n; ++m) {
            if (path_of[m] != path_of[fi]) continue;
            double ds = fabs(s_mid[m] - s_mid[fi]);
            c64 t = crs(sign[m] * feed_sign, cmul(cmk(0.0, -scale * sin(k * ds)), vsrc));
            cst(&rhs[2 * m], cadd(cld(&rhs[2 * m]), t));
        }
    }
    return OR_OK;
}

/* loads.rs:34-57 i0_over_i1: I0(z)/I1(z) by the power series for |z| <= 15,
 * the asymptotic expansion beyond. */
/* planewave.rs:86-105 r_hat / pol_hat: the arrival direction and the
 * complex polarisation vector e = u_maj + j sense AR u_min. */
static void pw_vectors(const or_wave *w, double *r_hat, c64 *pol) {
    double t = w->theta_deg * RADS_PER_DEG, p = w->phi_deg * RADS_PER_DEG;
    r_hat[0] = sin(t) * cos(p);
    r_hat[1] = sin(t) * sin(p);
    r_hat[2] = cos(t);
    double eta = w->eta_deg * RADS_PER_DEG;
    double th[3] = {cos(t) * cos(p), cos(t) * sin(p), -sin(t)};
    double ph[3] = {-sin(p), cos(p), 0.0};
    double ce = cos(eta), se = sin(eta);
    double ar = 0.0, sense = 0.0; /* planewave.rs:62-67 */
    if (w->ex_type == 2) {
        ar = w->axial_ratio;
        sense = 1.0;
    } else if (w->ex_type == 3) {
        ar = w->axial_ratio;
        sense = -1.0;
    }
    c64 jminor = cmk(0.0, sense * ar);
    for (int i = 0; i < 3; ++i) {
        double major = ce * th[i] + se * ph[i];
        double minor = -se * th[i] + ce * ph[i];
        pol[i] = cadd(cmk(major, 0.0), crs(minor, jminor));
    }
}

int or_planewave_rhs(const or_seg *segs, int64_t n, double freq_hz, const or_wave *wave, const int64_t *path_of,
                     const double *sign, const double *s_mid, double *rhs, double *cosv, double *sinv) {
    const double C0 = 299792458.0;
    const double ETA0 = 4.0 * OR_PI * 1e-7 * C0;
    double k = 2.0 * OR_PI * freq_hz / C0;
    double scale = 2.0 * OR_PI / ETA0;
    double r_hat[3];
    c64 pol[3];
    pw_vectors(wave, r_hat, pol);
    int64_t *grp = (int64_t *)malloc(sizeof(int64_t) * (size_t)(n > 0 ? n : 1));
    double *sc = (double *)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
    double *sg = (double *)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
    c64 *e = (c64 *)malloc(sizeof(c64) * (size_t)(n > 0 ? n : 1));
    int st = OR_OK;
    if (!path_of) {
        /* :176-209 per-tag wires, rejected when junctioned; s from the wire's
         * geometric midpoint along the direction of its first segment */
        int64_t w = or_wire_endpoints(segs, n, NULL, 0);
        int64_t *ep = (int64_t *)malloc(sizeof(int64_t) * 2 * (size_t)(w > 0 ? w : 1));
        or_wire_endpoints(segs, n, ep, w);
        if (or_detect_junctions(segs, ep, w, 1e-6, NULL, NULL, NULL, 0) > 0) st = OR_ERR_JUNCTION;
        for (int64_t q = 0; q < w && st == OR_OK; ++q) {
            const double *a = segs[ep[2 * q]].mid, *b = segs[ep[2 * q + 1]].mid;
            const double *dir = segs[ep[2 * q]].dir;
            double wm[3] = {(a[0] + b[0]) / 2.0, (a[1] + b[1]) / 2.0, (a[2] + b[2]) / 2.0};
            for (int64_t i = ep[2 * q]; i <= ep[2 * q + 1]; ++i) {
                double d[3] = {segs[i].mid[0] - wm[0], segs[i].mid[1] - wm[1], segs[i].mid[2] - wm[2]};
                grp[i] = q;
                sc[i] = dot3(d, dir);
                sg[i] = 1.0;
                c64 coup = cmk(0.0, 0.0);
                for (int c = 0; c < 3; ++c) coup = cadd(coup, crs(dir[c], pol[c]));
                double phase = k * dot3(r_hat, segs[i].mid);
                e[i] = cmul(coup, cmk(1.0 * cos(phase), 1.0 * sin(phase))); /* from_polar(1, phase) */
            }
        }
        free(ep);
    } else {
        /* :291-315 the path's signed arc length and traversal sign */
        for (int64_t i = 0; i < n; ++i) {
            grp[i] = path_of[i];
            sc[i] = s_mid[i];
            sg[i] = sign[i];
            c64 coup = cmk(0.0, 0.0);
            for (int c = 0; c < 3; ++c) coup = cadd(coup, crs(segs[i].dir[c], pol[c]));
            double phase = k * dot3(r_hat, segs[i].mid);
            e[i] = crs(sg[i], cmul(coup, cmk(1.0 * cos(phase), 1.0 * sin(phase))));
        }
    }
    if (st == OR_OK)
        for (int64_t m = 0; m < n; ++m) {
            c64 acc = cmk(0.0, 0.0);
            for (int64_t p = 0; p < n; ++p) {
                if (grp[p] != grp[m]) continue;
                double kern = sin(k * fabs(sc[m] - sc[p]));
                acc = cadd(acc, crs(segs[p].length, crs(kern, e[p])));
            }
            c64 r = cmul(cmk(0.0, -scale), acc);
            if (path_of) r = crs(sg[m], r);
            cst(&rhs[2 * m], r);
            cosv[m] = sg[m] * cos(k * sc[m]);
            sinv[m] = sg[m] * sin(k * sc[m]);
        }
    free(grp);
    free(sc);
    free(sg);
    free(e);
    return st;
}

static c64 i0_over_i1(c64 z) {
    if (cnorm(z) > 15.0) {
        c64 inv = cdiv(cmk(1.0, 0.0), z);
        return cadd(cadd(cmk(1.0, 0.0), cmk(inv.re * 0.5, inv.im * 0.5)),
                    (c64){cmul(inv, inv).re * 0.375, cmul(inv, inv).im * 0.375});
    }
    c64 half = cmk(z.re * 0.5, z.im * 0.5);
    c64 half_sq = cmul(half, half);
    c64 i0 = cmk(1.0, 0.0), term0 = cmk(1.0, 0.0);
    c64 i1 = half, term1 = half;
    for (int k = 1; k < 300; ++k) {
        double kf = (double)k;
        term0 = cmul(term0, cdivr(half_sq, kf * kf));
        i0 = cadd(i0, term0);
        term1 = cmul(term1, cdivr(half_sq, kf * (kf + 1.0)));
        i1 = cadd(i1, term1);
        if (cnorm(term0) <= 1e-17 * cnorm(i0) && cnorm(term1) <= 1e-17 * cnorm(i1)) break;
    }
    return cdiv(i0, i1);
}

/* loads.rs:73-81 wire_internal_impedance (skin-effect series impedance). */
static c64 wire_internal_impedance(double sigma, double a, double dl, double omega) {
    const double MU0 = 4.0 * OR_PI * 1e-7;
    if (omega <= 0.0) return cmk(dl / (sigma * OR_PI * a * a), 0.0);
    double delta = sqrt(2.0 / (omega * MU0 * sigma));
    c64 gamma = cmk(1.0 / delta, 1.0 / delta);
    c64 g = cdivr(gamma, 2.0 * OR_PI * a * sigma);
    c64 r = cmul(g, i0_over_i1(crs(a, gamma)));
    return cmk(r.re * dl, r.im * dl);
}

/* loads.rs:209-222 segment_matches. */
static int load_matches(const or_load *ld, const or_seg *s) {
    if (ld->tag != 0 && s->tag != ld->tag) return 0;
    if (ld->seg_first == 0) return 1;
    uint32_t last = ld->seg_last == 0 ? ld->seg_first : ld->seg_last;
    return s->tag_index >= ld->seg_first && s->tag_index <= last;
}

int64_t or_build_loads(const or_seg *segs, int64_t n, double freq_hz, const or_load *ld, int64_t nl,
                       double *out) {
    for (int64_t i = 0; i < 2 * n; ++i) out[i] = 0.0;
    const double omega = 2.0 * OR_PI * freq_hz;
    int64_t ignored = 0;
    for (int64_t q = 0; q < nl; ++q) {
        const or_load *L = &ld[q];
        if (L->load_type < 0 || L->load_type > 5) {  /* unsupported: warned, ignored */
            ignored++;
            continue;
        }
        for (int64_t i = 0; i < n; ++i) {
            if (!load_matches(L, &segs[i])) continue;
            c64 z;
            switch (L->load_type) {
            case 0: {
                double x_l = omega * L->f2;
                double x_c = L->f3 > 0.0 ? 1.0 / (omega * L->f3) : 0.0;
                z = cmk(L->f1, x_l - x_c);
                break;
            }
            case 1: {
                c64 y = cmk(0.0, 0.0);
                if (L->f1 > 0.0) y = cadd(y, cmk(1.0 / L->f1, 0.0));
                if (L->f2 > 0.0) y = cadd(y, cmk(0.0, -1.0 / (omega * L->f2)));
                if (L->f3 > 0.0) y = cadd(y, cmk(0.0, omega * L->f3));
                z = cnorm(y) < 1e-30 ? cmk(0.0, 0.0) : cdiv(cmk(1.0, 0.0), y);
                break;
            }
            case 2: z = cmk(L->f1, omega * L->f2); break;
            case 3: z = cmk(L->f1, -(L->f3 > 0.0 ? 1.0 / (omega * L->f3) : 0.0)); break;
            case 4: z = cmk(L->f1, L->f2); break;
            default: /* 5 */
                if (L->f1 <= 0.0) {
                    ignored++;
                    continue;
                }
                z = wire_internal_impedance(L->f1, segs[i].radius, segs[i].length, omega);
                break;
            }
            cst(&out[2 * i], cadd(cld(&out[2 * i]), z));
        }
    }
    return ignored;
}

/* tl.rs:186-241 find_segment_index: segment 0 is the tag's centre (the
 * middle one of an odd count; the lower centre of an even count). */
static int64_t tl_find_segment(const or_seg *segs, int64_t n, uint32_t tag, uint32_t seg) {
    if (seg != 0) return find_seg(segs, n, tag, seg);
    int64_t cnt = 0;
    for (int64_t i = 0; i < n; ++i)
        if (segs[i].tag == tag) cnt++;
    if (cnt == 0) return -1;
    int64_t pick;
    if (cnt % 2 == 1) {
        pick = cnt / 2;
    } else {
        uint32_t lower = (uint32_t)(cnt / 2);
        pick = -1;
        int64_t q = 0;
        for (int64_t i = 0; i < n && pick < 0; ++i)
            if (segs[i].tag == tag) {
                if (segs[i].tag_index == lower) pick = q;
                q++;
            }
        if (pick < 0) pick = cnt / 2 >= 1 ? cnt / 2 - 1 : 0;
    }
    int64_t q = 0;
    for (int64_t i = 0; i < n; ++i)
        if (segs[i].tag == tag) {
            if (q == pick) return i;
            q++;
        }
    return -1;
}

static int64_t put4(int64_t c, int64_t cap, int64_t *rows, int64_t *cols, double *vals, int64_t i1, int64_t i2,
                    c64 zd1, c64 zd2, c64 z12, c64 z21) {
    int64_t r[4] = {i1, i2, i1, i2}, cc[4] = {i1, i2, i2, i1};
    c64 v[4] = {zd1, zd2, z12, z21};
    for (int q = 0; q < 4; ++q, ++c)
        if (c < cap) {
            rows[c] = r[q];
            cols[c] = cc[q];
            cst(&vals[2 * c], v[q]);
        }
    return c;
}

int64_t or_tl_stamps(const or_seg *segs, int64_t n, double freq_hz, const or_tl *tl, int64_t ntl, int64_t *rows,
                     int64_t *cols, double *vals, int64_t cap) {
    const double k = 2.0 * OR_PI * freq_hz / C0;
    int64_t c = 0;
    for (int64_t q = 0; q < ntl; ++q) {
        const or_tl *T = &tl[q];
        int64_t i1 = tl_find_segment(segs, n, T->tag1, T->seg1);
        if (i1 < 0) continue;
        int64_t i2 = tl_find_segment(segs, n, T->tag2, T->seg2);
        if (i2 < 0 || i1 == i2 || T->z0 <= 0.0 || T->length <= 0.0) continue;
        if (T->tl_type != 0) {  /* lossy: Z0 coth(gl), Z0 csch(gl), velocity factor 1 */
            double beta_l = k * T->length;
            double alpha_l = T->f3 * M_LN10 / 20.0;
            /* num-complex sinh / cosh of (alpha_l + j beta_l) */
            c64 sh = cmk(sinh(alpha_l) * cos(beta_l), cosh(alpha_l) * sin(beta_l));
            c64 ch = cmk(cosh(alpha_l) * cos(beta_l), sinh(alpha_l) * sin(beta_l));
            if (cnorm(sh) < 1e-9) continue;
            c64 z0c = cmk(T->z0, 0.0);
            c64 zd = cdiv(cmul(z0c, ch), sh), zo = cdiv(z0c, sh);
            c = put4(c, cap, rows, cols, vals, i1, i2, zd, zd, zo, zo);
            continue;
        }
        double vf = (T->f3 >= 0.0 && T->f3 <= 1.0 && T->f3 > 0.0) ? T->f3 : 1.0;
        double theta = k * T->length / vf;
        double sin_t = sin(theta);
        if (fabs(sin_t) < 1e-9) continue;
        double cot = cos(theta) / sin_t, csc = 1.0 / sin_t;
        c64 zd = cmk(0.0, -T->z0 * cot), zo = cmk(0.0, -T->z0 * csc);
        c = put4(c, cap, rows, cols, vals, i1, i2, zd, zd, zo, zo);
    }
    return c;
}

int64_t or_nt_stamps(const or_seg *segs, int64_t n, const or_nt *nt, int64_t nnt, int64_t *rows, int64_t *cols,
                     double *vals, int64_t cap) {
    int64_t c = 0;
    for (int64_t q = 0; q < nnt; ++q) {
        const or_nt *N = &nt[q];
        c64 y11 = cmk(N->y11r, N->y11i), y12 = cmk(N->y12r, N->y12i), y21 = y12, y22 = cmk(N->y22r, N->y22i);
        int64_t i1 = tl_find_segment(segs, n, N->tag1, N->seg1);
        if (i1 < 0) continue;
        int64_t i2 = tl_find_segment(segs, n, N->tag2, N->seg2);
        if (i2 < 0 || i1 == i2) continue;
        c64 det = csub(cmul(y11, y22), cmul(y12, y21));
        if (cnorm(det) < 1e-30) continue;
        c64 z11 = cdiv(y22, det), z22 = cdiv(y11, det);
        c64 z12 = cdiv(cmk(-y12.re, -y12.im), det), z21 = cdiv(cmk(-y21.re, -y21.im), det);
        c = put4(c, cap, rows, cols, vals, i1, i2, z11, z22, z12, z21);
    }
    return c;
}

void or_near_field(const or_seg *segs, int64_t n, const double *cur, double freq_hz, const double *pts, int64_t p,
                   double *e_out, double *h_out) {
    const double C = 299792458.0;
    const double k = 2.0 * OR_PI * freq_hz / C;
    const double ETA0 = 4.0 * OR_PI * 1e-7 * C;
    const double coeff_e = ETA0 / (4.0 * OR_PI), coeff_h = 1.0 / (4.0 * OR_PI);
    for (int64_t q = 0; q < p; ++q) {
        const double *P = &pts[3 * q];
        c64 e[3] = {{0, 0}, {0, 0}, {0, 0}}, h[3] = {{0, 0}, {0, 0}, {0, 0}};
        for (int64_t m = 0; m < n; ++m) {
            const or_seg *s = &segs[m];
            double d[3] = {P[0] - s->mid[0], P[1] - s->mid[1], P[2] - s->mid[2]};
            double r = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
            if (r < 1e-9) continue; /* on the segment itself */
            double rh[3] = {d[0] / r, d[1] / r, d[2] / r};
            const double *u = s->dir;
            double kr_c = cos(k * r), kr_s = sin(k * r);
            c64 phase = cmk(kr_c, -kr_s);
            c64 jkr = cmk(0.0, k * r);
            c64 inv_jkr = cdiv(cmk(1.0, 0.0), jkr);
            c64 I = cld(&cur[2 * m]);
            if (e_out) {
                double c = u[0] * rh[0] + u[1] * rh[1] + u[2] * rh[2];
                c64 pref = cmul(crs(s->length * coeff_e, I), phase);
                double inv_kr2 = 1.0 / (k * r * k * r);
                c64 rad = crs(2.0 * c / (r * r), cadd(cmk(1.0, 0.0), inv_jkr));
                c64 th = cmul(cdivr(jkr, r * r), csub(cadd(cmk(1.0, 0.0), inv_jkr), cmk(inv_kr2, 0.0)));
                for (int a = 0; a < 3; ++a) {
                    double tan_a = c * rh[a] - u[a];
                    e[a] = cadd(e[a], cmul(pref, cadd(crs(rh[a], rad), crs(tan_a, th))));
                }
            }
            if (h_out) {
                double cr[3] = {u[1] * rh[2] - u[2] * rh[1], u[2] * rh[0] - u[0] * rh[2], u[0] * rh[1] - u[1] * rh[0]};
                c64 factor = cmul(cdivr(jkr, r * r), cadd(cmk(1.0, 0.0), inv_jkr));
                c64 pref = cmul(cmul(crs(s->length * coeff_h, I), phase), factor);
                for (int a = 0; a < 3; ++a) h[a] = cadd(h[a], crs(cr[a], pref));
            }
        }
        for (int a = 0; a < 3; ++a) {
            if (e_out) cst(&e_out[6 * q + 2 * a], e[a]);
            if (h_out) cst(&h_out[6 * q + 2 * a], h[a]);
        }
    }
}

int64_t or_near_field_points(uint32_t coord_type, uint32_t nx, uint32_t ny, uint32_t nz, double x0, double y0,
                             double z0, double dx, double dy, double dz, double *pts) {
    uint32_t mx = nx ? nx : 1, my = ny ? ny : 1, mz = nz ? nz : 1;
    int64_t c = 0;
    if (coord_type == 0) {
        for (uint32_t ix = 0; ix < mx; ++ix)
            for (uint32_t iy = 0; iy < my; ++iy)
                for (uint32_t iz = 0; iz < mz; ++iz, ++c)
                    if (pts) {
                        pts[3 * c] = x0 + (double)ix * dx;
                        pts[3 * c + 1] = y0 + (double)iy * dy;
                        pts[3 * c + 2] = z0 + (double)iz * dz;
                    }
    } else { /* theta outer, phi, then R inner */
        for (uint32_t it = 0; it < mz; ++it) {
            double th = (z0 + (double)it * dz) * RADS_PER_DEG;
            for (uint32_t ip = 0; ip < my; ++ip) {
                double ph = (y0 + (double)ip * dy) * RADS_PER_DEG;
                for (uint32_t ir = 0; ir < mx; ++ir, ++c)
                    if (pts) {
                        double r = x0 + (double)ir * dx;
                        pts[3 * c] = r * sin(th) * cos(ph);
                        pts[3 * c + 1] = r * sin(th) * sin(ph);
                        pts[3 * c + 2] = r * cos(th);
                    }
            }
        }
    }
    return c;
}

/* ------------------------------------------------------------------------- */
/* Z-matrix fill                                                              */
/* ------------------------------------------------------------------------- */

/* matrix.rs:397 green_k: exp(-jkR)/R. */
static inline c64 green_k(double r, double k) {
    double t = -k * r;
    return cdivr(cmk(cos(t), sin(t)), r);
}

/* matrix.rs:297-331 elem.  src_mid/src_dir may be an image. */
static c64 elem(const double *obs_mid, const double *obs_dir, const double *src_mid,
                const double *src_dir, double src_len, double src_rad, double k, int is_self) {
    double cos_alpha = dot3(obs_dir, src_dir);
    double half = src_len * 0.5;
    double a = src_rad;
    c64 int_k;
    if (is_self) {
        c64 smooth = cmk(0.0, 0.0);
        for (int m = 0; m < 4; ++m) {
            double l = GL_N4[m] * half;
            double r_eff = sqrt(l * l + a * a);
            c64 g = green_k(r_eff, k);
            c64 dyn = cmk(g.re - 1.0 / r_eff, g.im);
            smooth = cadd(smooth, crs(GL_W4[m], dyn));
        }
        smooth = cmk(smooth.re * half, smooth.im * half);
        double r_end = sqrt(half * half + a * a);
        double analytic = 2.0 * log((half + r_end) / a);
        int_k = cmk(smooth.re + analytic, smooth.im);
    } else {
        c64 sum = cmk(0.0, 0.0);
        for (int m = 0; m < 8; ++m) {
            double sc = GL_N8[m] * half;
            double rs[3] = {src_mid[0] + sc * src_dir[0], src_mid[1] + sc * src_dir[1],
                            src_mid[2] + sc * src_dir[2]};
            double rho[3] = {obs_mid[0] - rs[0], obs_mid[1] - rs[1], obs_mid[2] - rs[2]};
            double r_sq = rho[0] * rho[0] + rho[1] * rho[1] + rho[2] * rho[2];
            double r_eff = sqrt(r_sq + a * a);
            sum = cadd(sum, crs(GL_W8[m], green_k(r_eff, k)));
        }
        int_k = cmk(sum.re * half, sum.im * half);
    }
    return cmk(int_k.re * cos_alpha, int_k.im * cos_alpha);
}

static c64 z_entry(const or_seg *obs, const or_seg *src, double k, int ground, int is_self) {
    c64 direct = elem(obs->mid, obs->dir, src->mid, src->dir, src->length, src->radius, k, is_self);
    c64 img = cmk(0.0, 0.0);
    if (ground == OR_GROUND_PEC) {
        /* matrix.rs:265-279 image_segment: (x,y,-z), current (-Jx,-Jy,+Jz). */
        double im_mid[3] = {src->mid[0], src->mid[1], -src->mid[2]};
        double im_dir[3] = {-src->dir[0], -src->dir[1], src->dir[2]};
        img = elem(obs->mid, obs->dir, im_mid, im_dir, src->length, src->radius, k, 0);
    }
    return cadd(direct, img);
}

void or_z_element(const or_seg *obs, const or_seg *src, double freq_hz, int ground,
                  int is_self, double *out2) {
    double k = 2.0 * OR_PI * freq_hz / C0;
    cst(out2, z_entry(obs, src, k, ground, is_self));
}

/* matrix.rs:186-218 assemble_z_matrix_with_ground. */
void or_assemble_z(const or_seg *segs, int64_t n, double freq_hz, int ground, double *z) {
    double k = 2.0 * OR_PI * freq_hz / C0;
    for (int64_t i = 0; i < n; ++i)
        for (int64_t j = 0; j < n; ++j)
            cst(&z[2 * (i * n + j)], z_entry(&segs[i], &segs[j], k, ground, i == j));
}

/* ------------------------------------------------------------------------- */
/* Dense solve                                                                */
/* ------------------------------------------------------------------------- */

typedef struct {
    c64 *aug;
    int64_t s, w; /* rows, row width (s+1) */
    int64_t col;
    c64 diag;
    int64_t r0, r1;
} elim_job;

static void elim_rows(c64 *aug, int64_t s, int64_t col, c64 diag, int64_t r0, int64_t r1) {
    int64_t w = s + 1;
    const c64 *prow = &aug[col * w];
    for (int64_t row = r0; row < r1; ++row) {
        c64 *rr = &aug[row * w];
        c64 factor = cdiv(rr[col], diag);
        for (int64_t kk = col; kk <= s; ++kk) {
            c64 sub = cmul(factor, prow[kk]);
            rr[kk] = csub(rr[kk], sub);
        }
    }
}

typedef struct {
    c64 *aug;
    int64_t s;
    int nthreads;
    int tid;
    pthread_barrier_t *bar;
    volatile int64_t *col;
    volatile int *stop;
    c64 *diag;
} gepp_worker;

/* Row-parallel elimination: rows below the pivot are split among threads.
 * Each element still receives exactly the same sequence of operations as in
 * the serial loop, so the result is bit-identical. */
static void *gepp_thread(void *arg) {
    gepp_worker *g = (gepp_worker *)arg;
    for (;;) {
        pthread_barrier_wait(g->bar);
        if (*g->stop) break;
        int64_t col = *g->col;
        int64_t rows = g->s - (col + 1);
        int64_t chunk = (rows + g->nthreads - 1) / g->nthreads;
        int64_t r0 = col + 1 + chunk * g->tid;
        int64_t r1 = r0 + chunk;
        if (r1 > g->s) r1 = g->s;
        if (r0 < r1) elim_rows(g->aug, g->s, col, *g->diag, r0, r1);
        pthread_barrier_wait(g->bar);
    }
    return NULL;
}

/* linear.rs:1321-1383 solve_square_in_place on aug = [A|b] (s x (s+1)). */
static int gepp_aug(c64 *aug, int64_t s, c64 *x, int32_t *pivots, int nthreads) {
    int64_t w = s + 1;
    c64 *tmp = (c64 *)malloc(sizeof(c64) * (size_t)w);
    pthread_barrier_t bar;
    pthread_t *th = NULL;
    gepp_worker *wk = NULL;
    volatile int64_t shared_col = 0;
    volatile int stop = 0;
    c64 shared_diag;
    int nt = nthreads > 1 ? nthreads : 1;
    if (nt > 1) {
        pthread_barrier_init(&bar, NULL, (unsigned)nt + 1);
        th = (pthread_t *)malloc(sizeof(pthread_t) * (size_t)nt);
        wk = (gepp_worker *)malloc(sizeof(gepp_worker) * (size_t)nt);
        for (int t = 0; t < nt; ++t) {
            wk[t].aug = aug;
            wk[t].s = s;
            wk[t].nthreads = nt;
            wk[t].tid = t;
            wk[t].bar = &bar;
            wk[t].col = &shared_col;
            wk[t].stop = &stop;
            wk[t].diag = &shared_diag;
            pthread_create(&th[t], NULL, gepp_thread, &wk[t]);
        }
    }
    int status = OR_OK;
    for (int64_t col = 0; col < s; ++col) {
        /* Iterator::max_by keeps the LAST maximum: a later row replaces the
         * running best unless best compares strictly Greater. */
        int64_t piv = col;
        double best = cnorm(aug[col * w + col]);
        for (int64_t r = col + 1; r < s; ++r) {
            double v = cnorm(aug[r * w + col]);
            if (!(best > v)) {
                piv = r;
                best = v;
            }
        }
        if (pivots) pivots[col] = (int32_t)piv;
        if (cnorm(aug[piv * w + col]) < 1e-30) {
            status = OR_ERR_SINGULAR;
            if (pivots) pivots[col] = -1;
            break;
        }
        if (piv != col) {
            memcpy(tmp, &aug[col * w], sizeof(c64) * (size_t)w);
            memcpy(&aug[col * w], &aug[piv * w], sizeof(c64) * (size_t)w);
            memcpy(&aug[piv * w], tmp, sizeof(c64) * (size_t)w);
        }
        c64 diag = aug[col * w + col];
        if (nt > 1 && (s - col - 1) >= 64) {
            shared_col = col;
            shared_diag = diag;
            pthread_barrier_wait(&bar);
            pthread_barrier_wait(&bar);
        } else {
            elim_rows(aug, s, col, diag, col + 1, s);
        }
    }
    if (nt > 1) {
        stop = 1;
        pthread_barrier_wait(&bar);
        for (int t = 0; t < nt; ++t) pthread_join(th[t], NULL);
        pthread_barrier_destroy(&bar);
        free(th);
        free(wk);
    }
    free(tmp);
    if (status != OR_OK) return status;
    for (int64_t i = s - 1; i >= 0; --i) {
        c64 sum = aug[i * w + s];
        for (int64_t j = i + 1; j < s; ++j) sum = csub(sum, cmul(aug[i * w + j], x[j]));
        x[i] = cdiv(sum, aug[i * w + i]);
    }
    return OR_OK;
}

int or_solve_square(double *a, double *b, int64_t s, double *x, int32_t *pivots, int nthreads) {
    c64 *aug = (c64 *)malloc(sizeof(c64) * (size_t)(s * (s + 1) + 1));
    for (int64_t i = 0; i < s; ++i) {
        for (int64_t j = 0; j < s; ++j) aug[i * (s + 1) + j] = cld(&a[2 * (i * s + j)]);
        aug[i * (s + 1) + s] = cld(&b[2 * i]);
    }
    c64 *xx = (c64 *)malloc(sizeof(c64) * (size_t)(s + 1));
    int st = gepp_aug(aug, s, xx, pivots, nthreads);
    if (st == OR_OK)
        for (int64_t i = 0; i < s; ++i) cst(&x[2 * i], xx[i]);
    free(aug);
    free(xx);
    return st;
}

/* linear.rs:672-797 solve_hallen.
 *
 * The literal reference loop (naive != 0) forms the dense M (rows x cols)
 * and sums conj(M[r][i]) * M[r][j] over every r.  The default path skips
 * products that are structurally zero: adding +-0 to a running sum that
 * started at +0 never changes its value or its sign under round-to-nearest,
 * so the skipped form is value-identical (checked bit-for-bit by the tests).
 * Per element, the surviving terms are still added in ascending r. */
static int solve_core(const double *z, int64_t n, const double *rhs, const double *cosv, const double *sinv,
                      const int64_t *row_wire, int64_t w, const int64_t *cc0, const int64_t *cc1,
                      const double *cv1, int64_t nc, double *x, int32_t *pivots, double *gram, int naive,
                      int nthreads);

int or_solve_hallen(const double *z, int64_t n, const double *rhs, const double *cosv,
                    const int64_t *ep_in, int64_t w_in, const int64_t *ja, const int64_t *jb,
                    const double *jsign, int64_t nj, double *x, int32_t *pivots, double *gram,
                    int naive, int nthreads) {
    int64_t fallback[2];
    const int64_t *ep = ep_in;
    int64_t w = w_in;
    if (w_in == 0 || n == 0) {
        if (n > 0) {
            fallback[0] = 0;
            fallback[1] = n - 1;
            ep = fallback;
            w = 1;
        } else {
            w = 0;
        }
    }
    /* junction endpoint set */
    char *injunc = (char *)calloc((size_t)(n > 0 ? n : 1), 1);
    for (int64_t t = 0; t < nj; ++t) {
        injunc[ja[t]] = 1;
        injunc[jb[t]] = 1;
    }
    int64_t nfree = 0;
    for (int64_t q = 0; q < w; ++q) {
        if (!injunc[ep[2 * q]]) nfree++;
        if (!injunc[ep[2 * q + 1]]) nfree++;
    }
    int64_t rows = n + nfree + nj;
    int64_t *row_wire = (int64_t *)calloc((size_t)(n > 0 ? n : 1), sizeof(int64_t));
    for (int64_t q = 0; q < w; ++q)
        for (int64_t r = ep[2 * q]; r <= ep[2 * q + 1]; ++r) row_wire[r] = q;

    /* constraint rows as sparse lists: up to two (col, value) entries */
    int64_t nc = nfree + nj;
    int64_t *cc0 = (int64_t *)malloc(sizeof(int64_t) * (size_t)(nc + 1));
    int64_t *cc1 = (int64_t *)malloc(sizeof(int64_t) * (size_t)(nc + 1));
    double *cv1 = (double *)malloc(sizeof(double) * (size_t)(nc + 1));
    int64_t crow = 0;
    for (int64_t q = 0; q < w; ++q) {
        if (!injunc[ep[2 * q]]) {
            cc0[crow] = ep[2 * q];
            cc1[crow] = -1;
            cv1[crow] = 0.0;
            crow++;
        }
        if (!injunc[ep[2 * q + 1]]) {
            cc0[crow] = ep[2 * q + 1];
            cc1[crow] = -1;
            cv1[crow] = 0.0;
            crow++;
        }
    }
    for (int64_t t = 0; t < nj; ++t) {
        cc0[crow] = ja[t];
        cc1[crow] = jb[t];
        cv1[crow] = jsign[t];
        crow++;
    }
    (void)rows;
    int st = solve_core(z, n, rhs, cosv, NULL, row_wire, w, cc0, cc1, cv1, nc, x, pivots, gram, naive, nthreads);
    free(cc0);
    free(cc1);
    free(cv1);
    free(row_wire);
    free(injunc);
    return st;
}

/* linear.rs:823-894 solve_hallen_paths: one homogeneous column per path
 * (path_of), I = 0 rows only at the listed free-end segments (in order),
 * no junction rows; the normal equations and elimination as solve_hallen. */
int or_solve_hallen_paths(const double *z, int64_t n, const double *rhs, const double *cosv,
                          const int64_t *path_of, const int64_t *free_ends, int64_t n_free, double *x,
                          int32_t *pivots, double *gram, int naive, int nthreads) {
    int64_t w = 0;
    for (int64_t m = 0; m < n; ++m)
        if (path_of[m] + 1 > w) w = path_of[m] + 1;
    int64_t *cc1 = (int64_t *)malloc(sizeof(int64_t) * (size_t)(n_free + 1));
    double *cv1 = (double *)malloc(sizeof(double) * (size_t)(n_free + 1));
    for (int64_t q = 0; q < n_free; ++q) {
        cc1[q] = -1;
        cv1[q] = 0.0;
    }
    int st = solve_core(z, n, rhs, cosv, NULL, path_of, w, free_ends, cc1, cv1, n_free, x, pivots, gram, naive,
                        nthreads);
    free(cc1);
    free(cv1);
    return st;
}

int or_solve_hallen_planewave(const double *z, int64_t n, const double *rhs, const double *cosv,
                              const double *sinv, const int64_t *row_wire, int64_t w, const int64_t *free_ends,
                              int64_t n_free, double *x, int32_t *pivots, double *gram, int naive) {
    /* per-tag wires: rows I = 0 at (first, last) of each wire in order */
    int64_t nc = free_ends ? n_free : 2 * w;
    int64_t *cc0 = (int64_t *)malloc(sizeof(int64_t) * (size_t)(nc + 1));
    int64_t *cc1 = (int64_t *)malloc(sizeof(int64_t) * (size_t)(nc + 1));
    double *cv1 = (double *)malloc(sizeof(double) * (size_t)(nc + 1));
    if (free_ends) {
        for (int64_t q = 0; q < nc; ++q) cc0[q] = free_ends[q];
    } else {
        for (int64_t q = 0; q < w; ++q) {
            int64_t first = -1, last = -1;
            for (int64_t r = 0; r < n; ++r)
                if (row_wire[r] == q) {
                    if (first < 0) first = r;
                    last = r;
                }
            cc0[2 * q] = first;
            cc0[2 * q + 1] = last;
        }
    }
    for (int64_t q = 0; q < nc; ++q) {
        cc1[q] = -1;
        cv1[q] = 0.0;
    }
    int st = solve_core(z, n, rhs, cosv, sinv, row_wire, w, cc0, cc1, cv1, nc, x, pivots, gram, naive, 1);
    free(cc0);
    free(cc1);
    free(cv1);
    return st;
}

/* The normal equations (MᴴM + 1e-8 I) x = Mᴴy of M = [Z | -cos columns]
 * over constraint rows (cc0, cc1, cv1), then GEPP. */
static int solve_core(const double *z, int64_t n, const double *rhs, const double *cosv, const double *sinv,
                      const int64_t *row_wire, int64_t w, const int64_t *cc0, const int64_t *cc1,
                      const double *cv1, int64_t nc, double *x, int32_t *pivots, double *gram, int naive,
                      int nthreads) {
    /* sinv != NULL: two homogeneous columns (cos, sin) per wire, the
     * plane-wave form (linear.rs:955-961) */
    const int64_t hw = sinv ? 2 : 1;
    int64_t rows = n + nc;
    int64_t cols = n + hw * w;
    int64_t aw = cols + 1;
    c64 *aug = (c64 *)calloc((size_t)(cols * aw + 1), sizeof(c64));

    if (naive) {
        c64 *m = (c64 *)calloc((size_t)(rows * cols + 1), sizeof(c64));
        c64 *y = (c64 *)calloc((size_t)(rows + 1), sizeof(c64));
        for (int64_t r = 0; r < n; ++r) {
            for (int64_t c = 0; c < n; ++c) m[r * cols + c] = cld(&z[2 * (r * n + c)]);
            m[r * cols + n + hw * row_wire[r]] = cmk(-cosv[r], 0.0);
            if (sinv) m[r * cols + n + hw * row_wire[r] + 1] = cmk(-sinv[r], 0.0);
            y[r] = cld(&rhs[2 * r]);
        }
        for (int64_t q = 0; q < nc; ++q) {
            m[(n + q) * cols + cc0[q]] = cmk(1.0, 0.0);
            if (cc1[q] >= 0) m[(n + q) * cols + cc1[q]] = cmk(cv1[q], 0.0);
        }
        for (int64_t i = 0; i < cols; ++i) {
            for (int64_t j = 0; j < cols; ++j) {
                c64 sum = cmk(0.0, 0.0);
                for (int64_t r = 0; r < rows; ++r)
                    sum = cadd(sum, cmul(cconj(m[r * cols + i]), m[r * cols + j]));
                aug[i * aw + j] = sum;
            }
            c64 sum = cmk(0.0, 0.0);
            for (int64_t r = 0; r < rows; ++r) sum = cadd(sum, cmul(cconj(m[r * cols + i]), y[r]));
            aug[i * aw + cols] = sum;
        }
        free(m);
        free(y);
    } else {
        /* r-outer accumulation: each element still sees its terms in
         * ascending r, and structurally-zero products are skipped. */
        for (int64_t r = 0; r < n; ++r) {
            const double *zr = &z[2 * r * n];
            int64_t cw = n + hw * row_wire[r];
            c64 cval = cmk(-cosv[r], 0.0);
            c64 sval = cmk(sinv ? -sinv[r] : 0.0, 0.0);
            c64 yr = cld(&rhs[2 * r]);
            for (int64_t i = 0; i < n; ++i) {
                c64 ci = cconj(cld(&zr[2 * i]));
                c64 *arow = &aug[i * aw];
                for (int64_t j = 0; j < n; ++j) arow[j] = cadd(arow[j], cmul(ci, cld(&zr[2 * j])));
                arow[cw] = cadd(arow[cw], cmul(ci, cval));
                if (sinv) arow[cw + 1] = cadd(arow[cw + 1], cmul(ci, sval));
                arow[cols] = cadd(arow[cols], cmul(ci, yr));
            }
            for (int64_t h = 0; h < hw; ++h) { /* the cos row, then the sin row */
                c64 cc = cconj(h ? sval : cval);
                c64 *crw = &aug[(cw + h) * aw];
                for (int64_t j = 0; j < n; ++j) crw[j] = cadd(crw[j], cmul(cc, cld(&zr[2 * j])));
                crw[cw] = cadd(crw[cw], cmul(cc, cval));
                if (sinv) crw[cw + 1] = cadd(crw[cw + 1], cmul(cc, sval));
                crw[cols] = cadd(crw[cols], cmul(cc, yr));
            }
        }
        /* constraint rows r = n .. rows-1 in order; y = 0 there, so their
         * aty products are structurally zero. */
        for (int64_t q = 0; q < nc; ++q) {
            int64_t idx[2] = {cc0[q], cc1[q]};
            c64 val[2] = {cmk(1.0, 0.0), cmk(cv1[q], 0.0)};
            int cntq = cc1[q] >= 0 ? 2 : 1;
            for (int u = 0; u < cntq; ++u)
                for (int v = 0; v < cntq; ++v) {
                    c64 *e = &aug[idx[u] * aw + idx[v]];
                    *e = cadd(*e, cmul(cconj(val[u]), val[v]));
                }
        }
    }
    for (int64_t i = 0; i < cols; ++i) aug[i * aw + i] = cadd(aug[i * aw + i], cmk(1e-8, 0.0));
    if (gram)
        for (int64_t i = 0; i < cols * aw; ++i) cst(&gram[2 * i], aug[i]);

    c64 *xx = (c64 *)malloc(sizeof(c64) * (size_t)(cols + 1));
    int st = gepp_aug(aug, cols, xx, pivots, nthreads);
    if (st == OR_OK)
        for (int64_t i = 0; i < cols; ++i) cst(&x[2 * i], xx[i]);
    free(xx);
    free(aug);
    return st;
}

/* solve_session.rs:846-947 build_feedpoint_rows, voltage-source rows. */
int64_t or_feedpoints(const or_seg *segs, int64_t n, const or_source *src, int64_t ns,
                      const double *cur, double *out, int64_t cap) {
    double *v = (double *)malloc(sizeof(double) * 2 * (size_t)(n > 0 ? n : 1));
    or_excitation(segs, n, src, ns, v);
    int64_t cnt = 0;
    for (int64_t e = 0; e < ns; ++e) {
        int64_t idx = find_seg(segs, n, src[e].tag, src[e].segment);
        if (idx < 0) continue;
        c64 current = cld(&cur[2 * idx]);
        c64 vs = cmk(v[2 * idx] * segs[idx].length, v[2 * idx + 1] * segs[idx].length);
        c64 zin = cnorm(current) > 1e-60 ? cdiv(vs, current) : vs;
        if (cnt < cap) {
            double *o = &out[7 * cnt];
            o[0] = (double)idx;
            o[1] = vs.re;
            o[2] = vs.im;
            o[3] = current.re;
            o[4] = current.im;
            o[5] = zin.re;
            o[6] = zin.im;
        }
        cnt++;
    }
    free(v);
    return cnt;
}

/* ------------------------------------------------------------------------- */
/* Far field                                                                  */
/* ------------------------------------------------------------------------- */

/* farfield.rs:85-94 unit_vectors. */
static void unit_vectors(double th_deg, double ph_deg, double *rh, double *thh, double *phh) {
    double th = th_deg * RADS_PER_DEG;
    double ph = ph_deg * RADS_PER_DEG;
    double st = sin(th), ct = cos(th);
    double sp = sin(ph), cp = cos(ph);
    rh[0] = st * cp;
    rh[1] = st * sp;
    rh[2] = ct;
    thh[0] = ct * cp;
    thh[1] = ct * sp;
    thh[2] = -st;
    phh[0] = -sp;
    phh[1] = cp;
    phh[2] = 0.0;
}

/* farfield.rs:265-291 far_field_components and :514-546 _with_image. */
static void ff_components(const or_seg *segs, int64_t n, const double *cur, double k,
                          double th_deg, double ph_deg, int pec, c64 *ft, c64 *fp) {
    double rh[3], thh[3], phh[3];
    unit_vectors(th_deg, ph_deg, rh, thh, phh);
    c64 f_t = cmk(0.0, 0.0), f_p = cmk(0.0, 0.0);
    for (int64_t i = 0; i < n; ++i) {
        c64 in = cld(&cur[2 * i]);
        double pa = k * dot3(segs[i].mid, rh);
        c64 ph = cmk(cos(pa), sin(pa));
        c64 wtd = cmul(in, crs(segs[i].length, ph));
        double pt = dot3(segs[i].dir, thh);
        double pp = dot3(segs[i].dir, phh);
        f_t = cadd(f_t, cmk(wtd.re * pt, wtd.im * pt));
        f_p = cadd(f_p, cmk(wtd.re * pp, wtd.im * pp));
        if (pec) {
            double im_mid[3] = {segs[i].mid[0], segs[i].mid[1], -segs[i].mid[2]};
            double im_dir[3] = {-segs[i].dir[0], -segs[i].dir[1], segs[i].dir[2]};
            double ipa = k * dot3(im_mid, rh);
            c64 iph = cmk(cos(ipa), sin(ipa));
            c64 iw = cmul(in, crs(segs[i].length, iph));
            double ipt = dot3(im_dir, thh);
            double ipp = dot3(im_dir, phh);
            f_t = cadd(f_t, cmk(iw.re * ipt, iw.im * ipt));
            f_p = cadd(f_p, cmk(iw.re * ipp, iw.im * ipp));
        }
    }
    *ft = f_t;
    *fp = f_p;
}

/* farfield.rs:422-464 integrate_power_for_ground. */
static double integrate_power_k(const or_seg *segs, int64_t n, const double *cur, double k,
                                int ground) {
    int has_ground = ground == OR_GROUND_PEC;
    int64_t n_theta = has_ground ? 91 : 181;
    double theta_max = has_ground ? 90.0 : 180.0;
    int64_t n_phi = 360;
    double d_theta = (theta_max * RADS_PER_DEG) / ((double)n_theta - 1.0);
    double d_phi = 2.0 * OR_PI / (double)n_phi;
    double total = 0.0;
    for (int64_t it = 0; it < n_theta; ++it) {
        double th_deg = (double)it * theta_max / ((double)n_theta - 1.0);
        double sin_t = sin(th_deg * RADS_PER_DEG);
        if (sin_t == 0.0) continue;
        double w_t = (it == 0 || it == n_theta - 1) ? 0.5 * d_theta : d_theta;
        for (int64_t ip = 0; ip < n_phi; ++ip) {
            double ph_deg = (double)ip;
            c64 ft, fp;
            ff_components(segs, n, cur, k, th_deg, ph_deg, has_ground, &ft, &fp);
            total += (cnorm_sqr(ft) + cnorm_sqr(fp)) * sin_t * w_t * d_phi;
        }
    }
    return total;
}

double or_integrate_power(const or_seg *segs, int64_t n, const double *cur, double freq_hz,
                          int ground) {
    double lambda = C0 / freq_hz;
    double k = 2.0 * OR_PI / lambda;
    return integrate_power_k(segs, n, cur, k, ground);
}

/* farfield.rs:659-667 polarization_axial_ratio. */
static double axial_ratio(c64 et, c64 ep) {
    double s0 = cnorm_sqr(et) + cnorm_sqr(ep);
    if (s0 <= 1e-30) return 0.0;
    double s3 = 2.0 * cmul(et, cconj(ep)).im;
    double q = s3 / s0;
    if (q < -1.0) q = -1.0;
    if (q > 1.0) q = 1.0;
    double chi = 0.5 * asin(q);
    return tan(chi);
}

/* farfield.rs:563-647 compute_radiation_pattern. */
void or_radiation_pattern(const or_seg *segs, int64_t n, const double *cur, double freq_hz,
                          int ground, const double *pts, int64_t p, double *out,
                          double *total_out, double *uf_out) {
    double lambda = C0 / freq_hz;
    double k = 2.0 * OR_PI / lambda;
    int pec = ground == OR_GROUND_PEC;
    double total = integrate_power_k(segs, n, cur, k, ground);
    if (total_out) *total_out = total;
    double norm = total > 0.0 ? 4.0 * OR_PI / total : 0.0;
    for (int64_t q = 0; q < p; ++q) {
        double th = pts[2 * q], ph = pts[2 * q + 1];
        double *o = &out[4 * q];
        if (pec && th > 90.0) {
            o[0] = o[1] = o[2] = -999.99;
            o[3] = 0.0;
            if (uf_out) memset(&uf_out[4 * q], 0, 4 * sizeof(double));
            continue;
        }
        c64 ft, fp;
        ff_components(segs, n, cur, k, th, ph, pec, &ft, &fp);
        double ut = cnorm_sqr(ft) + cnorm_sqr(fp);
        double uth = cnorm_sqr(ft);
        double uph = cnorm_sqr(fp);
        o[0] = ut * norm > 1e-20 ? 10.0 * log10(ut * norm) : -999.99;
        o[1] = uth * norm > 1e-20 ? 10.0 * log10(uth * norm) : -999.99;
        o[2] = uph * norm > 1e-20 ? 10.0 * log10(uph * norm) : -999.99;
        o[3] = axial_ratio(ft, fp);
        if (uf_out) {
            uf_out[4 * q] = ft.re;
            uf_out[4 * q + 1] = ft.im;
            uf_out[4 * q + 2] = fp.re;
            uf_out[4 * q + 3] = fp.im;
        }
    }
}

/* farfield.rs:677-699 rp_card_points (phi outer, theta inner). */
int64_t or_rp_card_points(uint32_t n_theta, uint32_t n_phi, double theta0, double phi0,
                          double d_theta, double d_phi, double *pts) {
    int64_t nt = n_theta > 0 ? n_theta : 1;
    int64_t np = n_phi > 0 ? n_phi : 1;
    int64_t c = 0;
    for (int64_t ip = 0; ip < np; ++ip) {
        double phi = phi0 + (double)ip * d_phi;
        for (int64_t it = 0; it < nt; ++it) {
            double theta = theta0 + (double)it * d_theta;
            if (pts) {
                pts[2 * c] = theta;
                pts[2 * c + 1] = phi;
            }
            c++;
        }
    }
    return c;
}

/* ------------------------------------------------------------------------- */
/* Whole per-frequency solve (CLI standard Hallen branch)                     */
/* ------------------------------------------------------------------------- */

/* solve_session.rs:1285-1289: the LD loads on Z's diagonal (matrix.rs:131-139
 * add_to_diagonal), before the branch is chosen. */
static void add_stamps(double *z, int64_t n, const int64_t *r, const int64_t *c, const double *v, int64_t cnt) {
    for (int64_t q = 0; q < cnt; ++q) {
        double *e = &z[2 * (r[q] * n + c[q])];
        cst(e, cadd(cld(e), cld(&v[2 * q])));  /* matrix.rs add_to_entry */
    }
}

static void add_loads(const or_problem *p, const or_seg *segs, int64_t n, double *z) {
    if (p->loads && p->n_loads > 0) {
        double *ld = (double *)malloc(sizeof(double) * 2 * (size_t)(n > 0 ? n : 1));
        or_build_loads(segs, n, p->freq_hz, p->loads, p->n_loads, ld);
        for (int64_t i = 0; i < n; ++i) cst(&z[2 * (i * n + i)], cadd(cld(&z[2 * (i * n + i)]), cld(&ld[2 * i])));
        free(ld);
    }
    /* then the TL stamps, then the NT stamps (solve_session.rs:1290-1309) */
    int64_t cap = 4 * ((p->tls ? p->n_tls : 0) + (p->nts ? p->n_nts : 0)) + 1;
    int64_t *r = (int64_t *)malloc(sizeof(int64_t) * (size_t)cap), *cc = (int64_t *)malloc(sizeof(int64_t) * (size_t)cap);
    double *v = (double *)malloc(sizeof(double) * 2 * (size_t)cap);
    if (p->tls && p->n_tls > 0) add_stamps(z, n, r, cc, v, or_tl_stamps(segs, n, p->freq_hz, p->tls, p->n_tls, r, cc, v, cap));
    if (p->nts && p->n_nts > 0) add_stamps(z, n, r, cc, v, or_nt_stamps(segs, n, p->nts, p->n_nts, r, cc, v, cap));
    free(r);
    free(cc);
    free(v);
}

/* solve_session.rs:262-301 solve_plane_wave_hallen: a non-trivial
 * degree-2 path deck takes the path form, any other deck the per-tag wire
 * form (junctioned decks fail there); no feed rows. */
static int planewave_problem(or_problem *p, const or_seg *segs, int64_t n) {
    size_t nn = (size_t)(n > 0 ? n : 1);
    int64_t *path_of = (int64_t *)malloc(sizeof(int64_t) * nn);
    int64_t *fe = (int64_t *)malloc(sizeof(int64_t) * 2 * nn);
    int64_t *row_wire = (int64_t *)malloc(sizeof(int64_t) * nn);
    double *sgn = (double *)malloc(sizeof(double) * nn), *smid = (double *)malloc(sizeof(double) * nn);
    double *rhs = (double *)malloc(sizeof(double) * 2 * nn);
    double *cosv = (double *)malloc(sizeof(double) * nn), *sinv = (double *)malloc(sizeof(double) * nn);
    int nontrivial = 0;
    int64_t np = or_conductor_paths(segs, n, path_of, sgn, smid, fe, &nontrivial);
    int paths = np >= 0 && nontrivial;
    int st = or_planewave_rhs(segs, n, p->freq_hz, p->wave, paths ? path_of : NULL, sgn, smid, rhs, cosv, sinv);
    int64_t w = 0;
    if (paths) {
        w = np;
        memcpy(row_wire, path_of, sizeof(int64_t) * (size_t)n);
    } else {
        w = or_wire_endpoints(segs, n, NULL, 0);
        int64_t *ep = (int64_t *)malloc(sizeof(int64_t) * 2 * (size_t)(w > 0 ? w : 1));
        or_wire_endpoints(segs, n, ep, w);
        for (int64_t q = 0; q < w; ++q)
            for (int64_t r = ep[2 * q]; r <= ep[2 * q + 1]; ++r) row_wire[r] = q;
        free(ep);
    }
    double *z = NULL, *x = NULL;
    if (st == OR_OK) {
        z = (double *)malloc(sizeof(double) * 2 * nn * nn);
        or_assemble_z(segs, n, p->freq_hz, p->ground, z);
        add_loads(p, segs, n, z);
        x = (double *)malloc(sizeof(double) * 2 * (size_t)(n + 2 * w));
        st = or_solve_hallen_planewave(z, n, rhs, cosv, sinv, row_wire, w, paths ? fe : NULL, 2 * np, x, p->pivots,
                                       NULL, 0);
    }
    if (st == OR_OK) {
        memcpy(p->currents, x, sizeof(double) * 2 * (size_t)n);
        if (p->n_feed) *p->n_feed = 0;
        if (p->n_points > 0 && p->points && p->pattern)
            or_radiation_pattern(segs, n, x, p->freq_hz, p->ground, p->points, p->n_points, p->pattern, NULL, NULL);
    }
    free(path_of);
    free(fe);
    free(row_wire);
    free(sgn);
    free(smid);
    free(rhs);
    free(cosv);
    free(sinv);
    free(z);
    free(x);
    return st;
}

int or_solve_problem(or_problem *p) {
    int64_t cap = 0;
    for (int64_t w = 0; w < p->n_wires; ++w) cap += p->wires[w].segments;
    or_seg *segs = (or_seg *)malloc(sizeof(or_seg) * (size_t)(cap > 0 ? cap : 1));
    int64_t n = or_build_geometry(p->wires, p->n_wires, segs, cap);
    if (n < 0) {
        free(segs);
        return p->status = (int)n;
    }
    if (p->wave) {
        int st = planewave_problem(p, segs, n);
        free(segs);
        return p->status = st;
    }
    double *rhs = (double *)malloc(sizeof(double) * 2 * (size_t)n);
    double *cosv = (double *)malloc(sizeof(double) * (size_t)n);
    /* solve_session.rs:1338-1378: decks with a non-trivial degree-2
     * conductor path take the path solve */
    {
        int64_t *path_of = (int64_t *)malloc(sizeof(int64_t) * (size_t)n);
        double *sgn = (double *)malloc(sizeof(double) * (size_t)n);
        double *smid = (double *)malloc(sizeof(double) * (size_t)n);
        int64_t *fe = (int64_t *)malloc(sizeof(int64_t) * 2 * (size_t)n);
        int nontrivial = 0;
        int64_t np = or_conductor_paths(segs, n, path_of, sgn, smid, fe, &nontrivial);
        int st = OR_OK;
        int taken = np >= 0 && nontrivial;
        if (taken) {
            st = or_hallen_rhs_paths(segs, n, p->freq_hz, p->sources, p->n_sources, path_of, sgn, smid, rhs,
                                     cosv);
            double *x = (double *)malloc(sizeof(double) * 2 * (size_t)(n + np));
            double *z = NULL;
            if (st == OR_OK) {
                z = (double *)malloc(sizeof(double) * 2 * (size_t)(n * n));
                or_assemble_z(segs, n, p->freq_hz, p->ground, z);
                add_loads(p, segs, n, z);
                st = or_solve_hallen_paths(z, n, rhs, cosv, path_of, fe, 2 * np, x, p->pivots, NULL, 0, 1);
            }
            if (st == OR_OK) {
                memcpy(p->currents, x, sizeof(double) * 2 * (size_t)n);
                int64_t nf = or_feedpoints(segs, n, p->sources, p->n_sources, x, p->feed, p->n_sources);
                if (p->n_feed) *p->n_feed = nf;
                if (p->n_points > 0 && p->points && p->pattern)
                    or_radiation_pattern(segs, n, x, p->freq_hz, p->ground, p->points, p->n_points, p->pattern,
                                         NULL, NULL);
            }
            free(x);
            free(z);
        }
        free(path_of);
        free(sgn);
        free(smid);
        free(fe);
        if (taken) {
            free(segs);
            free(rhs);
            free(cosv);
            return p->status = st;
        }
    }
    int st = or_hallen_rhs(segs, n, p->freq_hz, p->sources, p->n_sources, rhs, cosv);
    if (st != OR_OK) {
        free(segs);
        free(rhs);
        free(cosv);
        return p->status = st;
    }
    double *z = (double *)malloc(sizeof(double) * 2 * (size_t)(n * n));
    or_assemble_z(segs, n, p->freq_hz, p->ground, z);
    add_loads(p, segs, n, z);
    int64_t w = or_merge_collinear(segs, n, NULL, 0);
    int64_t *ep = (int64_t *)malloc(sizeof(int64_t) * 2 * (size_t)w);
    or_merge_collinear(segs, n, ep, w);
    int64_t nj = or_cli_junctions(segs, n, ep, w, NULL, NULL, NULL, 0);
    int64_t *ja = (int64_t *)malloc(sizeof(int64_t) * (size_t)(nj + 1));
    int64_t *jb = (int64_t *)malloc(sizeof(int64_t) * (size_t)(nj + 1));
    double *js = (double *)malloc(sizeof(double) * (size_t)(nj + 1));
    or_cli_junctions(segs, n, ep, w, ja, jb, js, nj);
    double *x = (double *)malloc(sizeof(double) * 2 * (size_t)(n + w));
    st = or_solve_hallen(z, n, rhs, cosv, ep, w, ja, jb, js, nj, x, p->pivots, NULL, 0, 1);
    if (st == OR_OK) {
        memcpy(p->currents, x, sizeof(double) * 2 * (size_t)n);
        int64_t nf = or_feedpoints(segs, n, p->sources, p->n_sources, x, p->feed, p->n_sources);
        if (p->n_feed) *p->n_feed = nf;
        if (p->n_points > 0 && p->points && p->pattern)
            or_radiation_pattern(segs, n, x, p->freq_hz, p->ground, p->points, p->n_points,
                                 p->pattern, NULL, NULL);
    }
    free(segs);
    free(rhs);
    free(cosv);
    free(z);
    free(ep);
    free(ja);
    free(jb);
    free(js);
    free(x);
    return p->status = st;
}

typedef struct {
    or_problem *ps;
    int64_t count;
    int64_t *next;
    pthread_mutex_t *mu;
} pool_arg;

static void *pool_thread(void *arg) {
    pool_arg *a = (pool_arg *)arg;
    for (;;) {
        pthread_mutex_lock(a->mu);
        int64_t i = (*a->next)++;
        pthread_mutex_unlock(a->mu);
        if (i >= a->count) break;
        or_solve_problem(&a->ps[i]);
    }
    return NULL;
}

void or_solve_problems(or_problem *ps, int64_t count, int nthreads) {
    if (nthreads <= 1) {
        for (int64_t i = 0; i < count; ++i) or_solve_problem(&ps[i]);
        return;
    }
    int64_t next = 0;
    pthread_mutex_t mu;
    pthread_mutex_init(&mu, NULL);
    pool_arg a = {ps, count, &next, &mu};
    pthread_t *th = (pthread_t *)malloc(sizeof(pthread_t) * (size_t)nthreads);
    for (int t = 0; t < nthreads; ++t) pthread_create(&th[t], NULL, pool_thread, &a);
    for (int t = 0; t < nthreads; ++t) pthread_join(th[t], NULL);
    free(th);
    pthread_mutex_destroy(&mu);
}

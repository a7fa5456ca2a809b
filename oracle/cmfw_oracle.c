/* CPU oracle for the pFq Conservative Matrix Field walk — TEST INFRASTRUCTURE.
 *
 * A plain-C restatement of the reference algorithm, one function per
 * reference function, each citing the file:line it follows (paths are within
 * the VesterlundCoder/RamanujanDreams-CUDA project). The operation order of
 * every floating-point expression is kept as in the reference so that, with
 * fused = 0 and this file compiled with -ffp-contract=off, results are
 * bitwise identical to the reference's kernel bodies compiled for the host.
 *
 * Only tests/, the smoke check and bench.py's CPU-baseline leg use this file.
 */
#include "cmfw_oracle.h"

#include <math.h>
#include <omp.h>
#include <stdlib.h>
#include <string.h>

#define EPS64 2.220446049250313e-16
#define ORC_MAX_LIMITS 256 /* cmf_walk_f64.cu:33 */

typedef struct { double a[ORC_MAX_DIM][ORC_MAX_DIM]; } mat64;

/* ------------------------------------------------------------------ */
/* Descriptor and start points                                         */
/* ------------------------------------------------------------------ */

/* cmf_pfq.cuh:50-61 — rank = max(p, q+1), minus one at z == 1, p == q+1. */
orc_desc orc_make_desc(int p, int q, double z) {
    orc_desc d;
    d.p = p;
    d.q = q;
    d.z = z;
    d.naxes = p + q;
    d.rank = (p > q + 1) ? p : q + 1;
    if (z == 1.0 && p == q + 1) d.rank -= 1;
    return d;
}

/* MT19937-64 (Matsumoto & Nishimura, 2000), the generator behind the
 * reference's std::mt19937_64(42) (cmf_walk_f64.cu:62, 77). */
typedef struct { uint64_t s[312]; int i; } mt64;

static void mt64_seed(mt64 *g, uint64_t seed) {
    g->s[0] = seed;
    for (int k = 1; k < 312; ++k)
        g->s[k] = 6364136223846793005ULL * (g->s[k - 1] ^ (g->s[k - 1] >> 62)) + (uint64_t)k;
    g->i = 312;
}

static uint64_t mt64_next(mt64 *g) {
    const uint64_t upper = 0xFFFFFFFF80000000ULL, lower = 0x7FFFFFFFULL;
    if (g->i >= 312) {
        for (int k = 0; k < 312; ++k) {
            uint64_t y = (g->s[k] & upper) | (g->s[(k + 1) % 312] & lower);
            uint64_t v = g->s[(k + 156) % 312] ^ (y >> 1);
            if (y & 1ULL) v ^= 0xB5026F5AA96619E9ULL;
            g->s[k] = v;
        }
        g->i = 0;
    }
    uint64_t x = g->s[g->i++];
    x ^= (x >> 29) & 0x5555555555555555ULL;
    x ^= (x << 17) & 0x71D67FFFEDA60000ULL;
    x ^= (x << 37) & 0xFFF7EEE000000000ULL;
    x ^= x >> 43;
    return x;
}

void orc_mt64_stream(uint64_t seed, uint64_t *out, int n) {
    mt64 g;
    mt64_seed(&g, seed);
    for (int k = 0; k < n; ++k) out[k] = mt64_next(&g);
}

/* Byte offsets inside a 192-byte input record (cmf_walk_f64.cu:36-39). */
#define REC_BYTES 192
#define REC_START 64

static void put_f64(unsigned char *b, size_t off, double v) { memcpy(b + off, &v, 8); }
static void put_i32(unsigned char *b, size_t off, int v) { memcpy(b + off, &v, 4); }
static int get_i32(const unsigned char *b, size_t off) { int v; memcpy(&v, b + off, 4); return v; }

/* Input records as run_benchmark builds them (cmf_walk_f64.cu:166-199),
 * with its two generators (cmf_walk_f64.cu:61-71 and 75-91). Both
 * generators address the record array with the stride of the type they
 * write (128-byte positions, 16-int directions), not the 192-byte record
 * stride; that placement is reproduced byte for byte here. */
void orc_make_inputs(int p, int q, int n, int mode, int use_zeta, void *buf) {
    unsigned char *b = (unsigned char *)buf;
    const int naxes = p + q;
    mt64 g;
    if (mode == 0) {
        if (use_zeta) {
            for (int i = 0; i < n; ++i)
                for (int a = 0; a < naxes; ++a)
                    put_f64(b, (size_t)i * REC_BYTES + REC_START + 8 * a, a < p ? 1.0 : 2.0);
        } else {
            mt64_seed(&g, 42);
            for (int i = 0; i < n; ++i)
                for (int a = 0; a < naxes; ++a) {
                    int val = 2 + (int)(mt64_next(&g) % 19);
                    put_f64(b, (size_t)i * 128 + 8 * a, (double)val);
                }
        }
        for (int i = 0; i < n; ++i) {
            memset(b + (size_t)i * REC_BYTES, 0, 64);
            put_i32(b, (size_t)i * REC_BYTES, 1);
        }
    } else {
        for (int i = 0; i < n; ++i)
            for (int a = 0; a < naxes; ++a) {
                double v = use_zeta ? (a < p ? 1.0 : 2.0) : (a < p ? 2.0 : 3.0);
                put_f64(b, (size_t)i * REC_BYTES + REC_START + 8 * a, v);
            }
        mt64_seed(&g, 42);
        const int dmax = 3;
        for (int i = 0; i < n; ++i) {
            size_t base = (size_t)i * 64;
            int all_zero = 1;
            for (int a = 0; a < naxes; ++a) {
                int d = (int)(mt64_next(&g) % (uint64_t)(2 * dmax + 1)) - dmax;
                put_i32(b, base + 4 * a, d);
            }
            for (int a = 0; a < naxes; ++a)
                if (get_i32(b, base + 4 * a) != 0) { all_zero = 0; break; }
            if (all_zero) put_i32(b, base, 1);
        }
    }
}

/* ------------------------------------------------------------------ */
/* Companion column                                                    */
/* ------------------------------------------------------------------ */

/* cmf_pfq.cuh:127-141 — coefficients of prod_j (theta + v_j), ascending. */
static void orc_poly(const double *v, int count, double *out, int fused) {
    for (int k = 0; k <= count; ++k) out[k] = 0.0;
    out[0] = 1.0;
    int deg = 0;
    for (int j = 0; j < count; ++j) {
        double nx[ORC_MAX_DIM + 1] = {0};
        for (int k = 0; k <= deg; ++k) {
            nx[k] = fused ? fma(out[k], v[j], nx[k]) : nx[k] + out[k] * v[j];
            nx[k + 1] += out[k];
        }
        ++deg;
        for (int k = 0; k <= deg; ++k) out[k] = nx[k];
    }
}

/* cmf_pfq.cuh:146-181 — last column of the monic companion matrix of
 * D(theta) = theta prod(theta + y_i - 1) - z prod(theta + x_j), with the
 * reference's near-zero test on the leading coefficient. */
int orc_column(const double *pos, double z, int dim, int p, int q, double *col, int fused) {
    double xv[ORC_MAX_AXES], yv[ORC_MAX_AXES];
    for (int i = 0; i < p; ++i) xv[i] = pos[i];
    for (int i = 0; i < q; ++i) yv[i] = pos[p + i] - 1.0;
    double px[ORC_MAX_DIM + 1] = {0}, py[ORC_MAX_DIM + 1] = {0};
    orc_poly(xv, p, px, fused);
    orc_poly(yv, q, py, fused);
    double d[ORC_MAX_DIM + 1] = {0};
    for (int k = 0; k <= p; ++k) d[k] = -z * px[k];
    for (int k = 0; k <= q; ++k) d[k + 1] += py[k];
    double lead = d[dim];
    double lead_scale = 1.0;
    if (dim == p && p == q + 1) {
        lead_scale = fmax(1.0, fabs(1.0 - z));
    } else {
        for (int i = 0; i < p; ++i) lead_scale += fabs(pos[i]);
        for (int i = 0; i < q; ++i) lead_scale += fabs(pos[p + i] - 1.0);
    }
    if (!isfinite(lead) || fabs(lead) <= 64.0 * EPS64 * lead_scale) return 0;
    for (int i = 0; i < dim; ++i) {
        col[i] = -d[i] / lead;
        if (!isfinite(col[i])) return 0;
    }
    return 1;
}

/* ------------------------------------------------------------------ */
/* f64 walk                                                            */
/* ------------------------------------------------------------------ */

/* cmf_pfq.cuh:100-116 */
static int orc_normalize(mat64 *M, int dim, double *log_scale) {
    double mx = 0.0;
    for (int i = 0; i < dim; ++i)
        for (int j = 0; j < dim; ++j) {
            double x = fabs(M->a[i][j]);
            if (x > mx) mx = x;
        }
    if (!(mx > 0.0) || !isfinite(mx)) return 0;
    double inv = 1.0 / mx;
    for (int i = 0; i < dim; ++i)
        for (int j = 0; j < dim; ++j) M->a[i][j] *= inv;
    *log_scale += log(mx);
    return 1;
}

/* cmf_pfq.cuh:186-239 — M <- M (I + C/a), or M <- M (I + C/a)^-1 by the
 * per-row back-substitution and scalar solve. */
static int orc_right_mul(mat64 *M, int dim, const double *col, double denom, int inverse,
                         double *log_scale) {
    if (!isfinite(denom) || fabs(denom) <= 64.0 * EPS64) return 0;
    mat64 out;
    double inva = 1.0 / denom;
    if (!inverse) {
        for (int r = 0; r < dim; ++r) {
            double dot = 0.0;
            for (int k = 0; k < dim; ++k) dot += M->a[r][k] * col[k];
            for (int j = 0; j < dim - 1; ++j) out.a[r][j] = M->a[r][j] + M->a[r][j + 1] * inva;
            out.a[r][dim - 1] = M->a[r][dim - 1] + dot * inva;
        }
    } else {
        for (int r = 0; r < dim; ++r) {
            double al[ORC_MAX_DIM] = {0}, be[ORC_MAX_DIM] = {0};
            al[dim - 1] = 0.0;
            be[dim - 1] = 1.0;
            for (int j = dim - 2; j >= 0; --j) {
                al[j] = M->a[r][j] - al[j + 1] * inva;
                be[j] = -be[j + 1] * inva;
            }
            double da = 0.0, db = 0.0;
            for (int k = 0; k < dim; ++k) {
                da += al[k] * col[k];
                db += be[k] * col[k];
            }
            double sd = 1.0 + db * inva;
            double ss = fmax(1.0, fabs(db * inva));
            if (!isfinite(sd) || fabs(sd) <= 128.0 * EPS64 * ss) return 0;
            double t = (M->a[r][dim - 1] - da * inva) / sd;
            if (!isfinite(t)) return 0;
            for (int j = 0; j < dim; ++j) {
                out.a[r][j] = al[j] + be[j] * t;
                if (!isfinite(out.a[r][j])) return 0;
            }
        }
    }
    for (int r = 0; r < dim; ++r)
        for (int j = 0; j < dim; ++j) M->a[r][j] = out.a[r][j];
    return orc_normalize(M, dim, log_scale);
}

/* cmf_pfq.cuh:255-291 (and the identical selection in cmf_walk_df64.cu:237-243,
 * cmf_walk_rns.cu:111-117): evaluation point, denominator and direction. */
static void orc_axis_setup(const double *pos, int axis, int sign, int p, double *eval,
                           double *denom, int *inverse) {
    for (int a = 0; a < ORC_MAX_AXES; ++a) eval[a] = pos[a];
    *inverse = 0;
    if (axis < p) {
        if (sign > 0) {
            *denom = pos[axis];
        } else {
            eval[axis] -= 1.0;
            *denom = pos[axis] - 1.0;
            *inverse = 1;
        }
    } else {
        if (sign < 0) {
            *denom = pos[axis] - 1.0;
        } else {
            eval[axis] += 1.0;
            *denom = pos[axis];
            *inverse = 1;
        }
    }
}

static int orc_axis_step64(mat64 *M, int dim, double *pos, int axis, int sign, const orc_desc *d,
                           double *ls, int fused) {
    double eval[ORC_MAX_AXES], denom, col[ORC_MAX_DIM] = {0};
    int inverse;
    orc_axis_setup(pos, axis, sign, d->p, eval, &denom, &inverse);
    if (!orc_column(eval, d->z, dim, d->p, d->q, col, fused)) return 0;
    if (!orc_right_mul(M, dim, col, denom, inverse, ls)) return 0;
    pos[axis] += (double)sign;
    return 1;
}

/* cmf_pfq.cuh:305-322 — one lattice displacement: levels from max|dir| down
 * to 1, and within a level the axes in descending order. */
typedef int (*orc_axis_fn)(void *state, int axis, int sign);

static int orc_traj_step(const int *dir, int naxes, orc_axis_fn fn, void *state) {
    int max_abs = 0;
    for (int a = 0; a < naxes; ++a) {
        int v = abs(dir[a]);
        max_abs = max_abs > v ? max_abs : v;
    }
    for (int level = max_abs; level >= 1; --level)
        for (int axis = naxes - 1; axis >= 0; --axis) {
            if (abs(dir[axis]) < level) continue;
            if (!fn(state, axis, dir[axis] > 0 ? 1 : -1)) return 0;
        }
    return 1;
}

typedef struct {
    mat64 M;
    double pos[ORC_MAX_AXES];
    double ls;
    const orc_desc *d;
    int fused;
} walk64_state;

static int walk64_axis(void *s, int axis, int sign) {
    walk64_state *w = (walk64_state *)s;
    return orc_axis_step64(&w->M, w->d->rank, w->pos, axis, sign, w->d, &w->ls, w->fused);
}

typedef struct {
    mat64 m[3];
    double ls[3];
    int valid;
} snaps64;

static void mat_identity(mat64 *M) {
    for (int i = 0; i < ORC_MAX_DIM; ++i)
        for (int j = 0; j < ORC_MAX_DIM; ++j) M->a[i][j] = (i == j) ? 1.0 : 0.0;
}

/* cmf_pfq.cuh:348-371 */
static int orc_forward_walk(const int *dir, const double *start, const orc_desc *d, int N, int h,
                            snaps64 *sn, int fused) {
    memset(sn, 0, sizeof(*sn));
    if (N <= 0 || h <= 0 || N - 2 * h <= 0) return 0;
    walk64_state w;
    mat_identity(&w.M);
    for (int a = 0; a < ORC_MAX_AXES; ++a) w.pos[a] = start[a];
    w.ls = 0.0;
    w.d = d;
    w.fused = fused;
    const int cp1 = N - 2 * h, cp2 = N - h;
    for (int step = 1; step <= N; ++step) {
        if (!orc_traj_step(dir, d->naxes, walk64_axis, &w)) return 0;
        int k = step == cp1 ? 0 : step == cp2 ? 1 : step == N ? 2 : -1;
        if (k >= 0) {
            sn->m[k] = w.M;
            sn->ls[k] = w.ls;
        }
    }
    sn->valid = 1;
    return 1;
}

/* ------------------------------------------------------------------ */
/* Snapshot reduction                                                  */
/* ------------------------------------------------------------------ */

/* One limit estimate and where it came from: the ratio M[i][c] / M[j][c]
 * and the method (1 = Aitken, 0 = raw). */
typedef struct { double L; int method, i, j, c; } limit_entry;

/* cmf_pfq.cuh:385-460 — primary Aitken and raw ratio of M[0][d-1]/M[1][d-1],
 * then every other (i != j, column) ratio, capped at max_results. */
static int orc_limits(const snaps64 *s, int dim, limit_entry *res, int max_results) {
    const double DEN_MIN = 1e-280;
    int n = 0;
    {
        int c = dim - 1;
        double p3 = s->m[2].a[0][c], q3 = s->m[2].a[1][c];
        double p2 = s->m[1].a[0][c], q2 = s->m[1].a[1][c];
        double p1 = s->m[0].a[0][c], q1 = s->m[0].a[1][c];
        if (fabs(q3) > DEN_MIN && fabs(q2) > DEN_MIN && fabs(q1) > DEN_MIN) {
            double r1 = p1 / q1, r2 = p2 / q2, r3 = p3 / q3;
            if (isfinite(r1) && isfinite(r2) && isfinite(r3)) {
                double sc = fmax(1.0, fmax(fabs(r1), fmax(fabs(r2), fabs(r3))));
                double den = r1 - 2.0 * r2 + r3;
                if (fabs(den) > 1e-14 * sc) {
                    double dd = r2 - r3;
                    double L = r3 - dd * dd / den;
                    if (isfinite(L) && n < max_results) res[n++] = (limit_entry){L, 1, 0, 1, c};
                }
                if (fabs(r3) > 1e-15 && n < max_results) res[n++] = (limit_entry){r3, 0, 0, 1, c};
            }
        }
    }
    for (int c = 0; c < dim; ++c)
        for (int i = 0; i < dim; ++i)
            for (int j = 0; j < dim; ++j) {
                if (i == j) continue;
                if (c == dim - 1 && i == 0 && j == 1) continue;
                double d1 = s->m[0].a[j][c], d2 = s->m[1].a[j][c], d3 = s->m[2].a[j][c];
                if (fabs(d1) < DEN_MIN || fabs(d2) < DEN_MIN || fabs(d3) < DEN_MIN) continue;
                double r1 = s->m[0].a[i][c] / d1;
                double r2 = s->m[1].a[i][c] / d2;
                double r3 = s->m[2].a[i][c] / d3;
                if (!isfinite(r1) || !isfinite(r2) || !isfinite(r3)) continue;
                double sc = fmax(1.0, fmax(fabs(r1), fmax(fabs(r2), fabs(r3))));
                double den = r1 - 2.0 * r2 + r3;
                if (fabs(den) > 1e-14 * sc) {
                    double dd = r2 - r3;
                    double L = r3 - dd * dd / den;
                    if (isfinite(L) && fabs(L) > 1e-15 && n < max_results) res[n++] = (limit_entry){L, 1, i, j, c};
                }
                if (fabs(r3) > 1e-15 && n < max_results) res[n++] = (limit_entry){r3, 0, i, j, c};
            }
    return n;
}

/* cmf_pfq.cuh:476-527 */
static double orc_delta(const snaps64 *s, int dim, double L) {
    if (!s->valid) return NAN;
    const int c = dim - 1;
    double pa = s->m[1].a[0][c], qa = s->m[1].a[1][c];
    if (fabs(qa) < 1e-280) return NAN;
    double log_q = log(fabs(qa)) + s->ls[1];
    if (log_q <= 0.0) return NAN;
    double pN = s->m[2].a[0][c], qN = s->m[2].a[1][c];
    double LN = (fabs(qN) > 1e-280) ? pN / qN : NAN;
    double Lu = L;
    if (!isfinite(Lu)) {
        double pNh = s->m[1].a[0][c], qNh = s->m[1].a[1][c];
        double pN2h = s->m[0].a[0][c], qN2h = s->m[0].a[1][c];
        if (fabs(qNh) > 1e-280 && fabs(qN2h) > 1e-280) {
            double r1 = pN2h / qN2h, r2 = pNh / qNh, r3 = LN;
            double den = r1 - 2.0 * r2 + r3;
            if (isfinite(den) && fabs(den) > 1e-30) {
                double dd = r2 - r3;
                Lu = r3 - dd * dd / den;
            }
        }
        if (!isfinite(Lu)) Lu = LN;
    }
    if (!isfinite(Lu)) return NAN;
    double approx = pa / qa;
    if (!isfinite(approx)) return NAN;
    double diff = fabs(Lu - approx);
    if (diff <= 0.0) return INFINITY;
    if (!isfinite(diff)) return NAN;
    double log_diff = log(diff);
    return -(1.0 + log_diff / log_q);
}

/* cmf_pfq.cuh:531-552 */
static double orc_precision(const snaps64 *s, int dim) {
    if (!s->valid) return NAN;
    const int c = dim - 1;
    double pN = s->m[2].a[0][c], qN = s->m[2].a[1][c];
    double pNh = s->m[1].a[0][c], qNh = s->m[1].a[1][c];
    if (fabs(qN) < 1e-280 || fabs(qNh) < 1e-280) return NAN;
    double LN = pN / qN, LNh = pNh / qNh;
    if (!isfinite(LN) || !isfinite(LNh)) return NAN;
    double diff = fabs(LN - LNh);
    if (diff <= 0.0) return INFINITY;
    return -log10(diff);
}

/* cmf_pfq.cuh:563-596 */
static double orc_kamidelta(const snaps64 *s, int dim, double Lt) {
    if (!s->valid) return NAN;
    const int c = dim - 1;
    double pN = s->m[2].a[0][c], qN = s->m[2].a[1][c];
    double pNh = s->m[1].a[0][c], qNh = s->m[1].a[1][c];
    double pN2h = s->m[0].a[0][c], qN2h = s->m[0].a[1][c];
    if (fabs(qN) < 1e-280 || fabs(qNh) < 1e-280 || fabs(qN2h) < 1e-280) return NAN;
    double LN = pN / qN, LNh = pNh / qNh, LN2h = pN2h / qN2h;
    if (!isfinite(LN) || !isfinite(LNh) || !isfinite(LN2h)) return NAN;
    double La = NAN;
    double den = LN2h - 2.0 * LNh + LN;
    if (fabs(den) > 1e-30) {
        double dd = LNh - LN;
        La = LN - dd * dd / den;
    }
    double L = isfinite(Lt) ? Lt : (isfinite(La) ? La : LN);
    return orc_delta(s, dim, L);
}

/* Result fill shared by all variants (cmf_walk_f64.cu:122-153,
 * cmf_walk_df64.cu:333-348, cmf_walk_rns.cu:304-319). *src (optional) gets
 * the chosen estimate's source, (method << 12) | (i << 8) | (j << 4) | c, or
 * -1 when there is none. */
static void orc_reduce_src(const snaps64 *s, int dim, double *limit, double *delta, double *p,
                           double *q, double *precision, double *log_scale, int *n_limits, int *src) {
    limit_entry lim[ORC_MAX_LIMITS];
    int n = orc_limits(s, dim, lim, ORC_MAX_LIMITS);
    *n_limits = n;
    double L = NAN;
    int pick = -1;
    for (int i = 0; i < n; ++i)
        if (lim[i].method == 1) { L = lim[i].L; pick = i; break; }
    if (isnan(L) && n > 0) { L = lim[0].L; pick = 0; }
    *limit = L;
    if (src)
        *src = pick < 0 ? -1 : (lim[pick].method << 12) | (lim[pick].i << 8) | (lim[pick].j << 4) | lim[pick].c;
    *p = s->m[2].a[0][dim - 1];
    *q = s->m[2].a[1][dim - 1];
    *log_scale = s->ls[2];
    *precision = orc_precision(s, dim);
    *delta = orc_kamidelta(s, dim, L);
}

static void orc_reduce(const snaps64 *s, int dim, double *limit, double *delta, double *p,
                       double *q, double *precision, double *log_scale, int *n_limits) {
    orc_reduce_src(s, dim, limit, delta, p, q, precision, log_scale, n_limits, NULL);
}

static void orc_fill_invalid(double *limit, double *delta, double *p, double *q, double *precision,
                             double *log_scale, int *n_limits) {
    *limit = *delta = *p = *q = *precision = *log_scale = NAN;
    *n_limits = 0;
}

static void set_threads(int threads) {
    if (threads > 0) omp_set_num_threads(threads);
}

/* cmf_walk_f64.cu:94-154; limit_src (optional, n ints) gets each row's
 * estimate source (orc_reduce_src), -1 for invalid rows. */
int orc_walk_f64_src(int p, int q, double z, int N, int h, const orc_in *in, orc_out_f64 *out, int n,
                     int fused, int threads, int *limit_src) {
    orc_desc d = orc_make_desc(p, q, z);
    set_threads(threads);
#pragma omp parallel for schedule(dynamic, 4)
    for (int i = 0; i < n; ++i) {
        snaps64 s;
        orc_out_f64 *r = &out[i];
        int ok = orc_forward_walk(in[i].dir, in[i].start, &d, N, h, &s, fused);
        int src = -1;
        r->valid = ok;
        if (!ok)
            orc_fill_invalid(&r->limit, &r->delta, &r->p, &r->q, &r->precision, &r->log_scale, &r->n_limits);
        else
            orc_reduce_src(&s, d.rank, &r->limit, &r->delta, &r->p, &r->q, &r->precision, &r->log_scale,
                           &r->n_limits, &src);
        r->elapsed_ms = 0.0;
        if (limit_src) limit_src[i] = src;
    }
    return 0;
}

int orc_walk_f64(int p, int q, double z, int N, int h, const orc_in *in, orc_out_f64 *out, int n,
                 int fused, int threads) {
    return orc_walk_f64_src(p, q, z, N, h, in, out, n, fused, threads, NULL);
}

int orc_f64_snapshots(int p, int q, double z, int N, int h, const int *dir, const double *start,
                      int fused, double *m123, double *ls123) {
    orc_desc d = orc_make_desc(p, q, z);
    snaps64 s;
    int ok = orc_forward_walk(dir, start, &d, N, h, &s, fused);
    for (int k = 0; k < 3; ++k) {
        for (int i = 0; i < 8; ++i)
            for (int j = 0; j < 8; ++j) m123[k * 64 + i * 8 + j] = s.m[k].a[i][j];
        ls123[k] = s.ls[k];
    }
    return ok;
}

/* ------------------------------------------------------------------ */
/* df64 (float-float) walk, cmf_walk_df64.cu                           */
/* ------------------------------------------------------------------ */

typedef struct { float hi, lo; } ff;

/* cmf_walk_df64.cu:40-45 */
static ff ff_make(double x) {
    ff r;
    r.hi = (float)x;
    r.lo = (float)(x - (double)r.hi);
    return r;
}
static double ff_to_double(ff x) { return (double)x.hi + (double)x.lo; } /* :48-50 */

/* Knuth two-sum and FMA two-product (cmf_walk_df64.cu:54-69). */
static void ff_two_sum(float a, float b, float *hi, float *lo) {
    float s = a + b;
    float bv = s - a;
    *lo = (a - (s - bv)) + (b - bv);
    *hi = s;
}
static void ff_two_prod(float a, float b, float *hi, float *lo) {
    float pr = a * b;
    *lo = fmaf(a, b, -pr);
    *hi = pr;
}
static ff ff_add(ff a, ff b) { /* :73-79 */
    float sh, sl;
    ff_two_sum(a.hi, b.hi, &sh, &sl);
    sl += a.lo + b.lo;
    ff_two_sum(sh, sl, &sh, &sl);
    return (ff){sh, sl};
}
static ff ff_sub(ff a, ff b) { return ff_add(a, (ff){-b.hi, -b.lo}); } /* :83-86 */
static ff ff_mul(ff a, ff b) { /* :90-96 */
    float ph, pl;
    ff_two_prod(a.hi, b.hi, &ph, &pl);
    pl += a.hi * b.lo + a.lo * b.hi;
    ff_two_sum(ph, pl, &ph, &pl);
    return (ff){ph, pl};
}
static ff ff_mul_f(ff a, float b) { /* :100-106 */
    float ph, pl;
    ff_two_prod(a.hi, b, &ph, &pl);
    pl += a.lo * b;
    ff_two_sum(ph, pl, &ph, &pl);
    return (ff){ph, pl};
}
static ff ff_div_f(ff a, float b) { return ff_mul_f(a, 1.0f / b); } /* :110-113 */
static int ff_finite(ff a) { return isfinite(a.hi) && isfinite(a.lo); }

typedef struct { ff a[ORC_MAX_DIM][ORC_MAX_DIM]; } matff;

/* cmf_walk_df64.cu:138-153 — float max of the high parts, float reciprocal. */
static int ff_normalize(matff *M, int dim, double *ls) {
    float mx = 0.0f;
    for (int i = 0; i < dim; ++i)
        for (int j = 0; j < dim; ++j) {
            float x = fabsf(M->a[i][j].hi);
            if (x > mx) mx = x;
        }
    if (!(mx > 0.0f) || !isfinite(mx)) return 0;
    float inv = 1.0f / mx;
    for (int i = 0; i < dim; ++i)
        for (int j = 0; j < dim; ++j) M->a[i][j] = ff_mul_f(M->a[i][j], inv);
    *ls += log((double)mx);
    return 1;
}

/* cmf_walk_df64.cu:174-219 */
static int ff_right_mul(matff *M, int dim, const ff *col, ff denom, int inverse, double *ls) {
    if (!ff_finite(denom) || fabsf(denom.hi) <= 64.0f * 1.19e-7f) return 0;
    matff out;
    ff one = ff_make(1.0), zero = ff_make(0.0);
    ff inva = ff_div_f(one, denom.hi);
    if (!inverse) {
        for (int r = 0; r < dim; ++r) {
            ff dot = zero;
            for (int k = 0; k < dim; ++k) dot = ff_add(dot, ff_mul(M->a[r][k], col[k]));
            for (int j = 0; j < dim - 1; ++j) out.a[r][j] = ff_add(M->a[r][j], ff_mul(M->a[r][j + 1], inva));
            out.a[r][dim - 1] = ff_add(M->a[r][dim - 1], ff_mul(dot, inva));
        }
    } else {
        for (int r = 0; r < dim; ++r) {
            ff al[ORC_MAX_DIM], be[ORC_MAX_DIM];
            al[dim - 1] = zero;
            be[dim - 1] = one;
            for (int j = dim - 2; j >= 0; --j) {
                al[j] = ff_sub(M->a[r][j], ff_mul(al[j + 1], inva));
                be[j] = ff_sub(zero, ff_mul(be[j + 1], inva));
            }
            ff da = zero, db = zero;
            for (int k = 0; k < dim; ++k) {
                da = ff_add(da, ff_mul(al[k], col[k]));
                db = ff_add(db, ff_mul(be[k], col[k]));
            }
            ff sd = ff_add(one, ff_mul(db, inva));
            if (!ff_finite(sd) || fabsf(sd.hi) <= 1e-10f) return 0;
            ff inv_sd = ff_div_f(one, sd.hi);
            ff t = ff_mul(ff_sub(M->a[r][dim - 1], ff_mul(da, inva)), inv_sd);
            for (int j = 0; j < dim; ++j) out.a[r][j] = ff_add(al[j], ff_mul(be[j], t));
        }
    }
    for (int r = 0; r < dim; ++r)
        for (int j = 0; j < dim; ++j) M->a[r][j] = out.a[r][j];
    return ff_normalize(M, dim, ls);
}

typedef struct {
    matff M;
    double pos[ORC_MAX_AXES];
    double ls;
    const orc_desc *d;
    int fused;
} walkff_state;

/* cmf_walk_df64.cu:229-252 — f64 column (cmf_walk_df64.cu:163-171) split
 * into float-float. */
static int walkff_axis(void *s, int axis, int sign) {
    walkff_state *w = (walkff_state *)s;
    const orc_desc *d = w->d;
    double eval[ORC_MAX_AXES], denom, cold[ORC_MAX_DIM] = {0};
    int inverse;
    orc_axis_setup(w->pos, axis, sign, d->p, eval, &denom, &inverse);
    if (!orc_column(eval, d->z, d->rank, d->p, d->q, cold, w->fused)) return 0;
    ff col[ORC_MAX_DIM];
    for (int i = 0; i < ORC_MAX_DIM; ++i) col[i] = ff_make(i < d->rank ? cold[i] : 0.0);
    if (!ff_right_mul(&w->M, d->rank, col, ff_make(denom), inverse, &w->ls)) return 0;
    w->pos[axis] += (double)sign;
    return 1;
}

/* cmf_walk_df64.cu:304-349. Where N - 2h <= 0 the reference never writes
 * the first snapshot and then reads it; here that case is reported as an
 * invalid trajectory instead. */
int orc_walk_df64(int p, int q, double z, int N, int h, const orc_in *in, orc_out *out, int n,
                  int fused, int threads) {
    orc_desc d = orc_make_desc(p, q, z);
    set_threads(threads);
#pragma omp parallel for schedule(dynamic, 4)
    for (int i = 0; i < n; ++i) {
        orc_out *r = &out[i];
        walkff_state w;
        snaps64 s;
        memset(&s, 0, sizeof(s));
        for (int a = 0; a < ORC_MAX_DIM; ++a)
            for (int b = 0; b < ORC_MAX_DIM; ++b) w.M.a[a][b] = ff_make(a == b ? 1.0 : 0.0);
        for (int a = 0; a < ORC_MAX_AXES; ++a) w.pos[a] = in[i].start[a];
        w.ls = 0.0;
        w.d = &d;
        w.fused = fused;
        int ok = !(N <= 0 || h <= 0 || N - 2 * h <= 0);
        const int cp1 = N - 2 * h, cp2 = N - h;
        for (int step = 1; ok && step <= N; ++step) {
            if (!orc_traj_step(in[i].dir, d.naxes, walkff_axis, &w)) { ok = 0; break; }
            int k = -1;
            if (step == cp1) k = 0;
            if (step == cp2) k = 1;
            if (step == N) k = 2;
            if (k >= 0) {
                for (int a = 0; a < d.rank; ++a)
                    for (int b = 0; b < d.rank; ++b) s.m[k].a[a][b] = ff_to_double(w.M.a[a][b]);
                s.ls[k] = w.ls;
            }
        }
        r->valid = ok;
        if (!ok) {
            orc_fill_invalid(&r->limit, &r->delta, &r->p, &r->q, &r->precision, &r->log_scale, &r->n_limits);
            continue;
        }
        s.valid = 1;
        orc_reduce(&s, d.rank, &r->limit, &r->delta, &r->p, &r->q, &r->precision, &r->log_scale, &r->n_limits);
    }
    return 0;
}

/* ------------------------------------------------------------------ */
/* RNS walk, cmf_walk_rns.cu                                           */
/* ------------------------------------------------------------------ */

/* The reference's modulus table (cmf_walk_rns.cu:26-43), kept entry for
 * entry because residues are compared bit for bit. Only the first twelve
 * entries are prime; the walk arithmetic does not depend on primality
 * except through the Fermat-exponent inverse, which is reproduced as is. */
static const uint32_t ORC_MODULI[ORC_MAX_PRIMES] = {
    1073741789u, 1073741783u, 1073741741u, 1073741723u, 1073741717u, 1073741707u, 1073741693u,
    1073741683u, 1073741669u, 1073741657u, 1073741641u, 1073741623u, 1073741611u, 1073741597u,
    1073741587u, 1073741573u, 1073741563u, 1073741551u, 1073741537u, 1073741527u, 1073741513u,
    1073741503u, 1073741491u, 1073741477u, 1073741467u, 1073741453u, 1073741441u, 1073741427u,
    1073741413u, 1073741403u, 1073741391u, 1073741377u, 1073741363u, 1073741353u, 1073741341u,
    1073741329u, 1073741317u, 1073741307u, 1073741293u, 1073741281u, 1073741267u, 1073741257u,
    1073741243u, 1073741231u, 1073741219u, 1073741207u, 1073741193u, 1073741183u, 1073741171u,
    1073741157u, 1073741147u, 1073741137u, 1073741123u, 1073741111u, 1073741097u, 1073741087u,
    1073741077u, 1073741063u, 1073741051u, 1073741039u, 1073741027u, 1073741017u, 1073741003u,
    1073740991u};

void orc_rns_moduli(uint32_t *out, int n) {
    for (int k = 0; k < n && k < ORC_MAX_PRIMES; ++k) out[k] = ORC_MODULI[k];
}

/* cmf_walk_rns.cu:45-78 */
static uint64_t m_mul(uint64_t a, uint64_t b, uint64_t m) { return (a * b) % m; }
static uint64_t m_add(uint64_t a, uint64_t b, uint64_t m) {
    uint64_t r = a + b;
    return r >= m ? r - m : r;
}
static uint64_t m_sub(uint64_t a, uint64_t b, uint64_t m) { return a >= b ? a - b : a + m - b; }
static uint32_t m_from_double(double x, uint32_t p) {
    int64_t v = (int64_t)llround(x);
    if (v >= 0) return (uint32_t)((uint64_t)v % p);
    uint64_t mag = (uint64_t)0 - (uint64_t)v;
    return (uint32_t)(((uint64_t)p - mag % p) % p);
}
static uint32_t m_inv(uint32_t a, uint32_t p) { /* Fermat exponent p - 2 */
    uint64_t r = 1, b = a % p;
    uint32_t e = p - 2;
    while (e > 0) {
        if (e & 1) r = (r * b) % p;
        b = (b * b) % p;
        e >>= 1;
    }
    return (uint32_t)r;
}

typedef struct { uint32_t a[ORC_MAX_PRIMES][ORC_MAX_DIM][ORC_MAX_DIM]; } matrns;

typedef struct {
    matrns M, tmp;
    double pos[ORC_MAX_AXES];
    const orc_desc *d;
    int K, fused;
} walkrns_state;

/* cmf_walk_rns.cu:101-128 (column to residues) and 130-183 (update). */
static int walkrns_axis(void *s, int axis, int sign) {
    walkrns_state *w = (walkrns_state *)s;
    const orc_desc *d = w->d;
    const int dim = d->rank;
    double eval[ORC_MAX_AXES], denom, col[ORC_MAX_DIM] = {0};
    int inverse;
    orc_axis_setup(w->pos, axis, sign, d->p, eval, &denom, &inverse);
    if (!orc_column(eval, d->z, dim, d->p, d->q, col, w->fused)) return 0;
    if (!isfinite(denom) || fabs(denom) <= 64.0 * EPS64) return 0;
    for (int k = 0; k < w->K; ++k) {
        const uint64_t pk = ORC_MODULI[k];
        uint32_t cr[ORC_MAX_DIM];
        for (int i = 0; i < dim; ++i) cr[i] = m_from_double(col[i], (uint32_t)pk);
        uint32_t inva = m_inv(m_from_double(denom, (uint32_t)pk), (uint32_t)pk);
        uint32_t(*M)[ORC_MAX_DIM] = w->M.a[k];
        uint32_t(*O)[ORC_MAX_DIM] = w->tmp.a[k];
        if (!inverse) {
            for (int r = 0; r < dim; ++r) {
                uint64_t dot = 0;
                for (int i = 0; i < dim; ++i) dot = m_add(dot, m_mul(M[r][i], cr[i], pk), pk);
                for (int j = 0; j < dim - 1; ++j) O[r][j] = (uint32_t)m_add(M[r][j], m_mul(M[r][j + 1], inva, pk), pk);
                O[r][dim - 1] = (uint32_t)m_add(M[r][dim - 1], m_mul((uint32_t)dot, inva, pk), pk);
            }
        } else {
            for (int r = 0; r < dim; ++r) {
                uint32_t al[ORC_MAX_DIM] = {0}, be[ORC_MAX_DIM] = {0};
                al[dim - 1] = 0;
                be[dim - 1] = 1;
                for (int j = dim - 2; j >= 0; --j) {
                    al[j] = (uint32_t)m_sub(M[r][j], m_mul(al[j + 1], inva, pk), pk);
                    be[j] = (uint32_t)m_sub(0, m_mul(be[j + 1], inva, pk), pk);
                }
                uint64_t da = 0, db = 0;
                for (int i = 0; i < dim; ++i) {
                    da = m_add(da, m_mul(al[i], cr[i], pk), pk);
                    db = m_add(db, m_mul(be[i], cr[i], pk), pk);
                }
                uint32_t sd = (uint32_t)m_add(1, m_mul((uint32_t)db, inva, pk), pk);
                if (sd == 0) return 0;
                uint32_t isd = m_inv(sd, (uint32_t)pk);
                uint32_t t = (uint32_t)m_mul(m_sub(M[r][dim - 1], m_mul((uint32_t)da, inva, pk), pk), isd, pk);
                for (int j = 0; j < dim; ++j) O[r][j] = (uint32_t)m_add(al[j], m_mul(be[j], t, pk), pk);
            }
        }
    }
    for (int k = 0; k < w->K; ++k)
        for (int r = 0; r < dim; ++r)
            for (int j = 0; j < dim; ++j) w->M.a[k][r][j] = w->tmp.a[k][r][j];
    w->pos[axis] += (double)sign;
    return 1;
}

/* cmf_walk_rns.cu:225-251 — signed CRT over the first two moduli, then
 * the projective normalisation of cmf_pfq.cuh:100-116 (return value unused,
 * as in the reference). */
static void orc_rns_to_double(const matrns *M, int dim, int K, mat64 *out, double *ls) {
    for (int i = 0; i < dim; ++i)
        for (int j = 0; j < dim; ++j) {
            if (K >= 2) {
                uint64_t p0 = ORC_MODULI[0], p1 = ORC_MODULI[1];
                uint32_t r0 = M->a[0][i][j], r1 = M->a[1][i][j];
                uint64_t diff = (r1 >= r0) ? (uint64_t)(r1 - r0) : ((uint64_t)r1 + p1 - r0);
                uint64_t base = p0 % p1, res = 1, e = p1 - 2;
                while (e > 0) {
                    if (e & 1) res = (res * base) % p1;
                    base = (base * base) % p1;
                    e >>= 1;
                }
                uint64_t t = (diff * res) % p1;
                uint64_t val = r0 + p0 * t;
                uint64_t half = (p0 * p1) / 2;
                out->a[i][j] = (val > half) ? -(double)(p0 * p1 - val) : (double)val;
            } else {
                out->a[i][j] = (double)M->a[0][i][j];
            }
        }
    (void)orc_normalize(out, dim, ls);
}

static int orc_rns_run(const orc_desc *d, const int *dir, const double *start, int N, int h, int K,
                       int steps, int fused, walkrns_state *w, snaps64 *s, double *ls_out) {
    const int dim = d->rank;
    memset(s, 0, sizeof(*s));
    for (int k = 0; k < K; ++k)
        for (int i = 0; i < dim; ++i)
            for (int j = 0; j < dim; ++j) w->M.a[k][i][j] = (i == j) ? 1u : 0u;
    for (int a = 0; a < ORC_MAX_AXES; ++a) w->pos[a] = start[a];
    w->d = d;
    w->K = K;
    w->fused = fused;
    const int cp1 = N - 2 * h, cp2 = N - h;
    double ls = 0.0;
    int ok = 1;
    for (int step = 1; step <= steps; ++step) {
        if (!orc_traj_step(dir, d->naxes, walkrns_axis, w)) { ok = 0; break; }
        if (step % 100 == 0 || step == cp1 || step == cp2 || step == N) {
            mat64 wm;
            orc_rns_to_double(&w->M, dim, K, &wm, &ls);
            int k = -1;
            if (step == cp1) k = 0;
            if (step == cp2) k = 1;
            if (step == N) k = 2;
            if (k >= 0) {
                s->m[k] = wm;
                s->ls[k] = ls;
            }
            for (int kk = 0; kk < K; ++kk)
                for (int i = 0; i < dim; ++i)
                    for (int j = 0; j < dim; ++j) w->M.a[kk][i][j] = m_from_double(wm.a[i][j], ORC_MODULI[kk]);
        }
    }
    *ls_out = ls;
    return ok;
}

/* cmf_walk_rns.cu:260-320, with the N - 2h <= 0 case reported invalid. */
int orc_walk_rns(int p, int q, double z, int N, int h, const orc_in *in, orc_out *out, int n,
                 int n_primes, int fused, int threads) {
    orc_desc d = orc_make_desc(p, q, z);
    set_threads(threads);
#pragma omp parallel
    {
        walkrns_state *w = (walkrns_state *)malloc(sizeof(walkrns_state));
#pragma omp for schedule(dynamic, 1)
        for (int i = 0; i < n; ++i) {
            orc_out *r = &out[i];
            snaps64 s;
            double ls;
            int ok = !(N <= 0 || h <= 0 || N - 2 * h <= 0);
            if (ok) ok = orc_rns_run(&d, in[i].dir, in[i].start, N, h, n_primes, N, fused, w, &s, &ls);
            r->valid = ok;
            if (!ok) {
                orc_fill_invalid(&r->limit, &r->delta, &r->p, &r->q, &r->precision, &r->log_scale, &r->n_limits);
                continue;
            }
            s.valid = 1;
            orc_reduce(&s, d.rank, &r->limit, &r->delta, &r->p, &r->q, &r->precision, &r->log_scale, &r->n_limits);
        }
        free(w);
    }
    return 0;
}

int orc_rns_trace(int p, int q, double z, int N, int h, const int *dir, const double *start,
                  int n_primes, int steps, int fused, uint32_t *out, double *log_scale_out) {
    orc_desc d = orc_make_desc(p, q, z);
    walkrns_state *w = (walkrns_state *)malloc(sizeof(walkrns_state));
    snaps64 s;
    int ok = orc_rns_run(&d, dir, start, N, h, n_primes, steps, fused, w, &s, log_scale_out);
    const int dim = d.rank;
    for (int k = 0; k < n_primes; ++k)
        for (int i = 0; i < dim; ++i)
            for (int j = 0; j < dim; ++j) out[(k * dim + i) * dim + j] = w->M.a[k][i][j];
    free(w);
    return ok;
}

/* ------------------------------------------------------------------ */
/* Exact walk modulo primes                                            */
/* ------------------------------------------------------------------ */

/* The walk of cmf_pfq.cuh without rounding: every quantity of the f64 walk
 * is a rational number (integer start, rational z = zn / zd), so the walk
 * matrix is computed exactly in the field of residues modulo a prime m
 * (one (trajectory, prime) pair per task). The steps are the reference's
 * own formulas -- the column -d[i] / lead of D(theta) (cmf_pfq.cuh:146-181,
 * scaled by zd, which leaves the column unchanged), the forward update and
 * the row back-substitution of the inverse update (cmf_pfq.cuh:186-239),
 * the evaluation point and denominator of each axis step
 * (cmf_pfq.cuh:255-291), the path order (cmf_pfq.cuh:305-322) -- with
 * divisions as multiplications by inverses modulo m. A prime for which a
 * divisor (a * lead, or a row solve's scalar) vanishes is marked unusable;
 * the rational value is then taken from the other primes. The projective
 * normalisation is left out: it scales the whole matrix, and the ratios of
 * entries that the limits are formed from do not depend on it.
 *
 * Arithmetic: Montgomery multiplication (P. L. Montgomery, Math. Comp. 44,
 * 1985) with R = 2^32 for odd moduli below 2^31; inverses by Fermat's
 * little theorem, a^(m-2). */
typedef struct { uint32_t m, ninv, r2; } mont32;

static mont32 mont_make(uint32_t m) {
    mont32 M;
    uint32_t inv = m; /* Newton's iteration for m^-1 mod 2^32 (m odd) */
    for (int i = 0; i < 5; ++i) inv *= 2u - m * inv;
    M.m = m;
    M.ninv = 0u - inv;
    uint64_t r1 = ((uint64_t)1 << 32) % m;
    M.r2 = (uint32_t)((r1 * r1) % m);
    return M;
}
static inline uint32_t mont_redc(uint64_t T, const mont32 *M) {
    uint32_t u = (uint32_t)T * M->ninv;
    uint64_t t = (T + (uint64_t)u * M->m) >> 32;
    return t >= M->m ? (uint32_t)(t - M->m) : (uint32_t)t;
}
static inline uint32_t mont_mul(uint32_t a, uint32_t b, const mont32 *M) { return mont_redc((uint64_t)a * b, M); }
static inline uint32_t mont_add(uint32_t a, uint32_t b, const mont32 *M) {
    uint32_t r = a + b;
    return r >= M->m ? r - M->m : r;
}
static inline uint32_t mont_sub(uint32_t a, uint32_t b, const mont32 *M) { return a >= b ? a - b : a + M->m - b; }
static inline uint32_t mont_in(long long v, const mont32 *M) {
    long long r = v % (long long)M->m;
    if (r < 0) r += M->m;
    return mont_mul((uint32_t)r, M->r2, M);
}
static inline uint32_t mont_out(uint32_t a, const mont32 *M) { return mont_redc(a, M); }
static uint32_t mont_inv(uint32_t a, const mont32 *M) {
    uint32_t r = mont_in(1, M), b = a;
    for (uint32_t e = M->m - 2; e; e >>= 1) {
        if (e & 1) r = mont_mul(r, b, M);
        b = mont_mul(b, b, M);
    }
    return r;
}

/* Coefficients (ascending) of prod_j (theta + v_j) modulo m
 * (cmf_pfq.cuh:127-141). */
static void exact_poly(const uint32_t *v, int count, uint32_t *out, const mont32 *M) {
    uint32_t one = mont_in(1, M);
    for (int k = 0; k <= ORC_MAX_DIM; ++k) out[k] = 0;
    out[0] = one;
    for (int j = 0; j < count; ++j) {
        for (int k = j + 1; k >= 1; --k) out[k] = mont_add(mont_mul(out[k], v[j], M), out[k - 1], M);
        out[0] = mont_mul(out[0], v[j], M);
    }
}

/* One trajectory modulo one prime; returns 1 if every divisor was
 * invertible. snap gets entries (si, sc) and (sj, sc) at N-2h, N-h, N
 * (plain residues, [3][2]). */
static int exact_walk_one(const orc_desc *d, long long zn, long long zd, const int *dir, const double *start,
                          int N, int h, uint32_t prime, int si, int sj, int sc, uint32_t snap[3][2]) {
    const int dim = d->rank, p = d->p, q = d->q, naxes = d->naxes;
    const mont32 Mo = mont_make(prime), *M = &Mo;
    long long pos[ORC_MAX_AXES];
    int maxabs = 0;
    for (int a = 0; a < naxes; ++a) {
        if (start[a] != floor(start[a]) || fabs(start[a]) >= 9.0e15) return 0;
        if (abs(dir[a]) > 4096) return 0;
        pos[a] = (long long)start[a];
        maxabs = abs(dir[a]) > maxabs ? abs(dir[a]) : maxabs;
    }
    const uint32_t one = mont_in(1, M), zr = mont_in(zn, M), zdr = mont_in(zd, M);
    uint32_t m[ORC_MAX_DIM][ORC_MAX_DIM];
    for (int i = 0; i < dim; ++i)
        for (int j = 0; j < dim; ++j) m[i][j] = (i == j) ? one : 0u;
    const int cp1 = N - 2 * h, cp2 = N - h;
    for (int step = 1; step <= N; ++step) {
        for (int level = maxabs; level >= 1; --level)
            for (int axis = naxes - 1; axis >= 0; --axis) {
                if (abs(dir[axis]) < level) continue;
                const int sign = dir[axis] > 0 ? 1 : -1;
                const int is_x = axis < p;
                const int inverse = is_x ? (sign < 0) : (sign > 0);
                /* evaluation point and denominator (cmf_pfq.cuh:255-291) */
                long long ev[ORC_MAX_AXES];
                for (int a = 0; a < naxes; ++a) ev[a] = pos[a];
                long long den;
                if (is_x) {
                    if (sign > 0) den = pos[axis];
                    else { ev[axis] -= 1; den = pos[axis] - 1; }
                } else {
                    if (sign < 0) den = pos[axis] - 1;
                    else { ev[axis] += 1; den = pos[axis]; }
                }
                uint32_t xv[ORC_MAX_AXES], yv[ORC_MAX_AXES], px[ORC_MAX_DIM + 1], py[ORC_MAX_DIM + 1];
                for (int j = 0; j < p; ++j) xv[j] = mont_in(ev[j], M);
                for (int i = 0; i < q; ++i) yv[i] = mont_in(ev[p + i] - 1, M);
                exact_poly(xv, p, px, M);
                exact_poly(yv, q, py, M);
                /* zd * D(theta) = zd theta prod(theta + y_i - 1) - zn prod(theta + x_j) */
                uint32_t dc[ORC_MAX_DIM + 2];
                for (int k = 0; k <= dim; ++k) {
                    uint32_t v = (k <= p) ? mont_sub(0, mont_mul(zr, px[k], M), M) : 0u;
                    if (k >= 1 && k - 1 <= q) v = mont_add(v, mont_mul(zdr, py[k - 1], M), M);
                    dc[k] = v;
                }
                const uint32_t lead = dc[dim], ar = mont_in(den, M);
                const uint32_t al_ = mont_mul(ar, lead, M);
                if (al_ == 0u) return 0;
                const uint32_t inv_al = mont_inv(al_, M);
                const uint32_t inva = mont_mul(inv_al, lead, M), il = mont_mul(inv_al, ar, M);
                uint32_t col[ORC_MAX_DIM];
                for (int i = 0; i < dim; ++i) col[i] = mont_sub(0, mont_mul(dc[i], il, M), M);
                if (!inverse) {
                    for (int r = 0; r < dim; ++r) {
                        uint32_t dot = 0;
                        for (int i = 0; i < dim; ++i) dot = mont_add(dot, mont_mul(m[r][i], col[i], M), M);
                        for (int j = 0; j < dim - 1; ++j) m[r][j] = mont_add(m[r][j], mont_mul(m[r][j + 1], inva, M), M);
                        m[r][dim - 1] = mont_add(m[r][dim - 1], mont_mul(dot, inva, M), M);
                    }
                } else {
                    uint32_t be[ORC_MAX_DIM];
                    be[dim - 1] = one;
                    for (int j = dim - 2; j >= 0; --j) be[j] = mont_sub(0, mont_mul(be[j + 1], inva, M), M);
                    uint32_t db = 0;
                    for (int i = 0; i < dim; ++i) db = mont_add(db, mont_mul(be[i], col[i], M), M);
                    const uint32_t sd = mont_add(one, mont_mul(db, inva, M), M);
                    if (sd == 0u) return 0;
                    const uint32_t isd = mont_inv(sd, M);
                    for (int r = 0; r < dim; ++r) {
                        uint32_t al[ORC_MAX_DIM];
                        al[dim - 1] = 0;
                        for (int j = dim - 2; j >= 0; --j) al[j] = mont_sub(m[r][j], mont_mul(al[j + 1], inva, M), M);
                        uint32_t da = 0;
                        for (int i = 0; i < dim; ++i) da = mont_add(da, mont_mul(al[i], col[i], M), M);
                        const uint32_t t = mont_mul(mont_sub(m[r][dim - 1], mont_mul(da, inva, M), M), isd, M);
                        for (int j = 0; j < dim; ++j) m[r][j] = mont_add(al[j], mont_mul(be[j], t, M), M);
                    }
                }
                pos[axis] += sign;
            }
        const int s = step == cp1 ? 0 : step == cp2 ? 1 : step == N ? 2 : -1;
        if (s >= 0) {
            snap[s][0] = mont_out(m[si][sc], M);
            snap[s][1] = mont_out(m[sj][sc], M);
        }
    }
    return 1;
}

int orc_exact_residues(int p, int q, long long zn, long long zd, int N, int h, const orc_in *in, int n,
                       const uint32_t *primes, int K, const int *pairs, uint32_t *res, uint8_t *ok, int threads) {
    orc_desc d = orc_make_desc(p, q, zd != 0 ? (double)zn / (double)zd : 0.0);
    const int dim = d.rank;
    set_threads(threads);
    const long long tasks = (long long)n * K;
#pragma omp parallel for schedule(dynamic, 8)
    for (long long g = 0; g < tasks; ++g) {
        const int t = (int)(g / K), k = (int)(g % K);
        int si = 0, sj = 1, sc = dim - 1;
        if (pairs && pairs[t] >= 0) {
            si = (pairs[t] >> 8) & 15;
            sj = (pairs[t] >> 4) & 15;
            sc = pairs[t] & 15;
            if (si >= dim) si = dim - 1;
            if (sj >= dim) sj = dim - 1;
            if (sc >= dim) sc = dim - 1;
        }
        uint32_t snap[3][2] = {{0, 0}, {0, 0}, {0, 0}};
        int good = !(N <= 0 || h <= 0 || N - 2 * h <= 0) && (primes[k] & 1u) && primes[k] < (1u << 31);
        if (good) good = exact_walk_one(&d, zn, zd, in[t].dir, in[t].start, N, h, primes[k], si, sj, sc, snap);
        for (int s = 0; s < 3; ++s)
            for (int e = 0; e < 2; ++e) res[(((size_t)t * 3 + s) * 2 + e) * K + k] = good ? snap[s][e] : 0u;
        ok[(size_t)t * K + k] = (uint8_t)good;
    }
    return 0;
}

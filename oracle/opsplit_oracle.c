/*
 * TEST INFRASTRUCTURE ONLY — CPU oracle of the operator-split SSA step.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference arms
 * may load this file's library, and only as the checker or the timed CPU baseline,
 * never as part of the product path.
 *
 * It restates, in plain C, the algorithm of STEPS' TetOpSplitP split window
 * (src/steps/mpi/tetopsplit/tetopsplit.cpp, "TOS") with the project's counter-based
 * random streams, so that the GPU solver fed the same Philox counters must match it
 * bit for bit.  It is written independently of the CUDA sources: its own Philox, its
 * own samplers (same published algorithms, same operation order), its own table build.
 *
 * Pinning:
 *   - Philox4x32-10 is checked against the reference's vendored Random123
 *     (src/third_party/Random123/philox.h) by tests/golden/philox_kat.json, produced
 *     by oracle/ref_philox_kat.c compiled from that header.
 *   - The binomial sampler is checked by the chi-squared test of the reference's
 *     test/unit/cpp/test_rng.cpp:51-90 (same n, p grid and thresholds) and by a
 *     proper chi-squared goodness of fit over the BINV, mode-search and BTRD regimes.
 *   - Trajectory statistics are checked against the analytic kinetics of
 *     test/validation/API_1/validation_rd_mpi/parallel_spatial_tetopsplit.py.
 *
 * Compile with -ffp-contract=off (explicit fma() only).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------- */
/* Philox4x32 (Salmon et al., SC'11), 8 rounds as the reference's R123         */
/* ------------------------------------------------------------------------- */
typedef struct {
    uint32_t v[4];
} or_ctr;

/* Rounds of the stream generator: 8, as the reference's R123 (src/steps/rng/r123.hpp:76
   Philox4x32_R<8>). */
#define OR_PHILOX_ROUNDS 8

static or_ctr or_philox_r(or_ctr c, uint32_t k0, uint32_t k1, int rounds) {
    for (int r = 0; r < rounds; ++r) {
        uint64_t p0 = (uint64_t)0xD2511F53u * c.v[0];
        uint64_t p1 = (uint64_t)0xCD9E8D57u * c.v[2];
        or_ctr n;
        n.v[0] = (uint32_t)(p1 >> 32) ^ c.v[1] ^ k0;
        n.v[1] = (uint32_t)p1;
        n.v[2] = (uint32_t)(p0 >> 32) ^ c.v[3] ^ k1;
        n.v[3] = (uint32_t)p0;
        c = n;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    return c;
}

static or_ctr or_philox(or_ctr c, uint32_t k0, uint32_t k1) { return or_philox_r(c, k0, k1, OR_PHILOX_ROUNDS); }

/* Exported for the known-answer test (any round count). */
void or_philox4x32_r(int rounds, const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
    or_ctr c = {{ctr[0], ctr[1], ctr[2], ctr[3]}};
    or_ctr r = or_philox_r(c, key[0], key[1], rounds);
    memcpy(out, r.v, 16);
}

/* Stream of one (realization, unit, window): draw j = word j%4 of Philox(block j/4). */
typedef struct {
    uint32_t k0, k1, unit, wlo, whi, block;
    uint32_t buf[4];
    int pos;
} or_stream;

static void or_stream_init(or_stream* s, uint64_t seed, uint32_t real, uint32_t unit,
                           uint64_t window, uint32_t purpose) {
    s->k0 = (uint32_t)seed;
    s->k1 = (uint32_t)(seed >> 32) + real * 0x9E3779B9u;
    s->unit = unit;
    s->wlo = (uint32_t)window;
    s->whi = (purpose << 24) | ((uint32_t)(window >> 32) & 0xFFFFFFu);
    s->block = 0;
    s->pos = 4;
}

static uint32_t or_u32(or_stream* s) {
    if (s->pos == 4) {
        or_ctr c = {{s->block, s->unit, s->wlo, s->whi}};
        or_ctr r = or_philox(c, s->k0, s->k1);
        memcpy(s->buf, r.v, 16);
        s->block += 1;
        s->pos = 0;
    }
    return s->buf[s->pos++];
}

static const double TWO_M32 = 2.3283064365386963e-10;
static double u_co(uint32_t x) { return (double)x * TWO_M32; }
static double u_oc(uint32_t x) { return ((double)x + 1.0) * TWO_M32; }

/* ------------------------------------------------------------------------- */
/* log via 2 atanh((m-1)/(m+1)) Taylor series (same terms and order as the GPU) */
/* ------------------------------------------------------------------------- */
static double or_log(double x) {
    uint64_t b;
    memcpy(&b, &x, 8);
    int e = (int)((b >> 52) & 0x7FF);
    if (e == 0) {
        x = x * 18014398509481984.0;
        memcpy(&b, &x, 8);
        e = (int)((b >> 52) & 0x7FF) - 54;
    }
    e -= 1023;
    uint64_t mb = (b & 0x000FFFFFFFFFFFFFull) | 0x3FF0000000000000ull;
    double m;
    memcpy(&m, &mb, 8);
    if (m > 1.4142135623730951) {
        m = m * 0.5;
        e += 1;
    }
    double s = (m - 1.0) / (m + 1.0);
    double z = s * s;
    static const double inv_odd[10] = {1.0 / 21.0, 1.0 / 19.0, 1.0 / 17.0, 1.0 / 15.0, 1.0 / 13.0,
                                       1.0 / 11.0, 1.0 / 9.0,  1.0 / 7.0,  1.0 / 5.0,  1.0 / 3.0};
    double p = 1.0 / 23.0;
    for (int i = 0; i < 10; ++i) p = fma(p, z, inv_odd[i]);
    double t = 2.0 * s;
    double lm = fma(t * z, p, t);
    double de = (double)e;
    return fma(de, 0.6931471803691238, fma(de, 1.9082149292705877e-10, lm));
}

double or_log_export(double x) { return or_log(x); }

/* ------------------------------------------------------------------------- */
/* Binomial: BINV (Kachitvichyanukul & Schmeiser 1988), inversion from the mode,   */
/* BTRD (Hormann 1993) for very large n p                                     */
/* ------------------------------------------------------------------------- */
static double or_powu(double q, uint32_t n) {
    double r = 1.0, b = q;
    while (n) {
        if (n & 1u) r = r * b;
        b = b * b;
        n >>= 1;
    }
    return r;
}

static uint32_t or_binv(or_stream* st, uint32_t n, double p) {
    double q = 1.0 - p;
    double s = p / q;
    double a = ((double)n + 1.0) * s;
    double r = or_powu(q, n);
    double u = u_co(or_u32(st));
    uint32_t x = 0;
    /* Unbounded search, clamped: the factor turns negative from x = n + 2. */
    while (u >= r) {
        u = u - r;
        x += 1;
        r = r * fma(a, 1.0 / (double)x, -s);
        if (!(r > 0.0)) break;
    }
    return x < n ? x : n;
}

static double or_fc(uint32_t k) {
    static const double tab[10] = {0.08106146679532733,  0.04134069595540946,
                                   0.027677925684997717, 0.02079067210376584,
                                   0.01664469118982126,  0.013876128823072875,
                                   0.011896709945893313, 0.010411265261973668,
                                   0.00925546218270945,  0.008330563433359472};
    if (k < 10) return tab[k];
    double k1 = (double)k + 1.0;
    double k1sq = k1 * k1;
    return (1.0 / 12.0 - (1.0 / 360.0 - 1.0 / 1260.0 / k1sq) / k1sq) / k1;
}

static uint32_t or_btrd(or_stream* st, uint32_t n, double p) {
    double dn = (double)n, q = 1.0 - p;
    double m = floor((dn + 1.0) * p);
    double r = p / q, nr = (dn + 1.0) * r, npq = dn * p * q;
    double sq = sqrt(npq);
    double b = 1.15 + 2.53 * sq;
    double a = -0.0873 + 0.0248 * b + 0.01 * p;
    double c = dn * p + 0.5;
    double alpha = (2.83 + 5.1 / b) * sq;
    double vr = 0.92 - 4.2 / b;
    double urvr = 0.86 * vr;
    uint32_t mi = (uint32_t)m;
    for (int iter = 0; iter < 256; ++iter) {
        double v = u_co(or_u32(st)), u;
        if (v <= urvr) {
            u = v / vr - 0.43;
            double kq = floor((2.0 * a / (0.5 - fabs(u)) + b) * u + c);
            if (kq < 0.0 || kq > dn) continue;
            return (uint32_t)kq;
        }
        if (v >= vr) {
            u = u_co(or_u32(st)) - 0.5;
        } else {
            u = v / vr - 0.93;
            u = (u < 0.0 ? -0.5 : 0.5) - u;
            v = u_co(or_u32(st)) * vr;
        }
        double us = 0.5 - fabs(u);
        double kd = floor((2.0 * a / us + b) * u + c);
        if (kd < 0.0 || kd > dn) continue;
        v = v * alpha / (a / (us * us) + b);
        double km = fabs(kd - m);
        uint32_t k = (uint32_t)kd;
        if (km <= 15.0) {
            double f = 1.0;
            if (mi < k) {
                for (uint32_t i = mi + 1; i <= k; ++i) f = f * (nr / (double)i - r);
            } else if (mi > k) {
                for (uint32_t i = k + 1; i <= mi; ++i) v = v * (nr / (double)i - r);
            }
            if (v <= f) return k;
            continue;
        }
        v = or_log(v);
        double rho = (km / npq) * (((km / 3.0 + 0.625) * km + 1.0 / 6.0) / npq + 0.5);
        double t = -km * km / (2.0 * npq);
        if (v < t - rho) return k;
        if (v > t + rho) continue;
        double nm = dn - m + 1.0;
        double h = (m + 0.5) * or_log((m + 1.0) / (r * nm)) + or_fc(mi) + or_fc(n - mi);
        double nk = dn - kd + 1.0;
        double bound = h + (dn + 1.0) * or_log(nm / nk) + (kd + 0.5) * or_log(nk * r / (kd + 1.0)) -
                       or_fc(k) - or_fc(n - k);
        if (v <= bound) return k;
    }
    return mi;
}

/* e^x: k = round(x / ln 2), r = x - k ln 2 (two-part ln 2), Taylor series of e^r to r^14,
   2^k through the exponent bits (same steps as the GPU's). */
static double or_exp(double x) {
    if (!(x < 709.78)) {
        if (x != x) return x;
        uint64_t inf = 0x7FF0000000000000ull;
        double d;
        memcpy(&d, &inf, 8);
        return d;
    }
    if (x < -708.39) return 0.0;
    const double k = floor(x * 1.4426950408889634 + 0.5);
    double r = fma(-k, 0.6931471803691238, x);
    r = fma(-k, 1.9082149292705877e-10, r);
    static const double c[14] = {1.0 / 6227020800.0, 1.0 / 479001600.0, 1.0 / 39916800.0, 1.0 / 3628800.0,
                                 1.0 / 362880.0,     1.0 / 40320.0,     1.0 / 5040.0,     1.0 / 720.0,
                                 1.0 / 120.0,        1.0 / 24.0,        1.0 / 6.0,        0.5,
                                 1.0,                1.0};
    double p = 1.0 / 87178291200.0;
    for (int i = 0; i < 14; ++i) p = fma(p, r, c[i]);
    int ki = (int)k;
    if (ki > 1023) {
        p = p * 2.0;
        ki -= 1;
    }
    if (ki < -1022) {
        p = p * 0.5;
        ki += 1;
    }
    uint64_t b = (uint64_t)(ki + 1023) << 52;
    double sc;
    memcpy(&sc, &b, 8);
    return p * sc;
}

double or_exp_export(double x) { return or_exp(x); }

/* ln k! by Stirling's form with the remainder fc. */
static double or_lnfact(uint32_t k) {
    const double k1 = (double)k + 1.0;
    return (k1 - 0.5) * or_log(k1) - k1 + 0.91893853320467274 + or_fc(k);
}

/* Inversion from the mode for p <= 1/2: support in the order m, m+1, m-1, m+2, m-2, ...
   (one side alone once the other end is reached); f(m) from the log-factorials, the
   neighbours by the pmf ratios (n+1) s / (x+1) - s upwards and x r / (n-x+1) downwards. */
static uint32_t or_binom_mode(or_stream* st, uint32_t n, double p) {
    const double q = 1.0 - p;
    const double s = p / q;
    const double dn = (double)n;
    uint32_t m = (uint32_t)floor((dn + 1.0) * p);
    if (m > n) m = n;
    const double lf = ((or_lnfact(n) - or_lnfact(m)) - or_lnfact(n - m)) + (double)m * or_log(p) +
                      (double)(n - m) * or_log(q);
    const double fm = or_exp(lf);
    const double a = (dn + 1.0) * s;
    const double r = q / p;
    double u = u_co(or_u32(st)) - fm;
    if (u < 0.0) return m;
    double fu = fm, fd = fm;
    uint32_t xu = m, xd = m;
    for (;;) {
        const int cu = xu < n, cd = xd > 0u;
        if (!cu && !cd) return m;
        if (cu) {
            fu = fu * fma(a, 1.0 / (double)(xu + 1u), -s);
            xu += 1u;
            u = u - fu;
            if (u < 0.0) return xu;
        }
        if (cd) {
            fd = fd * ((double)xd * r) * (1.0 / (double)(n - xd + 1u));
            xd -= 1u;
            u = u - fd;
            if (u < 0.0) return xd;
        }
    }
}

/* Up to OR_PM_MAX molecules the leave draws each molecule's fate with one uniform v: it
   leaves when v < t1 and then takes face f when v < t1 cum_f, cum_f the cumulative face
   probabilities of the conditional selectors c (a selector of 1 takes all that remain).
   v < x is decided as u32 v < ceil(x 2^32).  Returns the leavers, per face in k. */
#define OR_PM_MAX 16u
static uint64_t or_thr(double x) { return x > 0.0 ? (uint64_t)ceil(x * 4294967296.0) : 0ull; }
static uint32_t or_leave_molecules(or_stream* st, uint32_t n, double t1, const double c[3], uint32_t k[4]) {
    const double c0 = c[0], c1 = c[1], c2 = c[2];
    const double r0 = 1.0 - c0;
    const double cum0 = c0;
    const double cum1 = cum0 + c1 * r0;
    const double cum2 = cum1 + c2 * (r0 * (1.0 - c1));
    uint64_t thr[4];
    thr[3] = or_thr(t1);
    thr[2] = c2 >= 1.0 ? thr[3] : or_thr(t1 * cum2);
    thr[1] = c1 >= 1.0 ? thr[3] : or_thr(t1 * cum1);
    thr[0] = c0 >= 1.0 ? thr[3] : or_thr(t1 * cum0);
    if (c1 >= 1.0) thr[2] = thr[3];
    if (c0 >= 1.0) thr[1] = thr[2] = thr[3];
    for (int f = 2; f >= 0; --f)
        if (thr[f] > thr[f + 1]) thr[f] = thr[f + 1];
    uint32_t below[4] = {0, 0, 0, 0};
    for (uint32_t i = 0; i < n; ++i) {
        const uint64_t v = or_u32(st);
        for (int f = 0; f < 4; ++f) below[f] += v < thr[f];
    }
    k[0] = below[0];
    for (int f = 1; f < 4; ++f) k[f] = below[f] - below[f - 1];
    return below[3];
}

static uint32_t or_binom(or_stream* st, uint32_t n, double p) {
    if (n == 0 || !(p > 0.0)) return 0;
    if (p >= 1.0) return n;
    int flip = p > 0.5;
    double pp = flip ? 1.0 - p : p;
    const double np = (double)n * pp;
    uint32_t k;
    if (np < 24.0)
        k = or_binv(st, n, pp);
    else if (np < 1000.0)
        k = or_binom_mode(st, n, pp);
    else
        k = or_btrd(st, n, pp);
    return flip ? n - k : k;
}

/* ------------------------------------------------------------------------- */
/* Placement of a compartment count over its tets (util/distribute.hpp:102-193, */
/* math/sample.hpp:59-200): volume-weighted floor allocation, then the remainder */
/* by adjusted Pareto order sampling on the fractional parts.  Draws come from   */
/* the stream the solver uses for its n-th setter call (key (seed, 0), unit =   */
/* call index, purpose 1), so the result can be compared bit for bit.          */
/* ------------------------------------------------------------------------- */
typedef struct {
    double key;
    int idx;
} or_keyed;

static int or_keyed_cmp(const void* a, const void* b) {
    const or_keyed* x = (const or_keyed*)a;
    const or_keyed* y = (const or_keyed*)b;
    if (x->key < y->key) return -1;
    if (x->key > y->key) return 1;
    return (x->idx > y->idx) - (x->idx < y->idx);
}

/* Returns 0, or -1 for a non-positive total weight, -2 if the floors exceed x. */
int or_distribute(uint64_t seed, uint64_t call, int n, const double* w, double x, uint32_t* out) {
    if (n <= 0) return 0;
    if (x == 0.0) {
        for (int i = 0; i < n; ++i) out[i] = 0;
        return 0;
    }
    or_stream st;
    or_stream_init(&st, seed, 0u, (uint32_t)(call & 0xFFFFFFFFu), call >> 32, 1u);
    double total = 0.0;
    for (int i = 0; i < n; ++i) total += w[i];
    if (!(total > 0.0)) return -1;
    if (u_co(or_u32(&st)) < x - floor(x))
        x = 1.0 + floor(x);
    else
        x = floor(x);
    double xot = x / total;
    unsigned long long allocated = 0;
    double* pi = (double*)malloc(sizeof(double) * (size_t)n);
    for (int i = 0; i < n; ++i) {
        double xi = xot * w[i];
        double fl = floor(xi);
        pi[i] = xi - fl;
        out[i] = (uint32_t)fl;
        allocated += (unsigned long long)fl;
    }
    if ((double)allocated > x) {
        free(pi);
        return -2;
    }
    size_t rem = (size_t)(x - (double)allocated);
    if (rem > 0) {
        double psum = 0.0;
        for (int i = 0; i < n; ++i) psum += pi[i];
        double rescale = (double)rem / psum;
        double d = 0.0;
        for (int i = 0; i < n; ++i) {
            pi[i] *= rescale;
            if (pi[i] > 1.0) pi[i] = 1.0;
            d += pi[i] * (1.0 - pi[i]);
        }
        double ood2 = (d == 0.0) ? 1.0 : 1.0 / (d * d);
        or_keyed* keys = (or_keyed*)malloc(sizeof(or_keyed) * (size_t)n);
        size_t nk = 0;
        for (int i = 0; i < n; ++i) {
            double q = pi[i];
            if (q == 0.0) continue;
            /* Rosen's adjusted Pareto rank: q_c U / (1 - U), q_c = (1-q)/q exp(q(1-q)(q-1/2)/d^2)
               with the exponential to second order. */
            double la = q * (1.0 - q) * (q - 0.5) * ood2;
            double aa = 1.0 + la + 0.5 * la * la;
            double qc = (1.0 - q) / q * aa;
            double u = u_co(or_u32(&st));
            keys[nk].key = qc * u / (1.0 - u);
            keys[nk].idx = i;
            ++nk;
        }
        if (nk < rem) rem = nk;
        qsort(keys, nk, sizeof(or_keyed), or_keyed_cmp);
        for (size_t j = 0; j < rem; ++j) out[keys[j].idx] += 1;
        free(keys);
    }
    free(pi);
    return 0;
}

/* Draw count binomials from one stream (sampler tests): out[i] = Binom(n, p). */
/* count per-molecule leaves of n molecules from one stream: out[4 i + f] leave through face f. */
void or_leave_many(uint64_t seed, uint32_t unit, uint32_t n, double t1, double c0, double c1, double c2,
                   uint32_t count, uint32_t* out) {
    or_stream st;
    or_stream_init(&st, seed, 0u, unit, 0u, 16u);
    const double c[3] = {c0, c1, c2};
    for (uint32_t i = 0; i < count; ++i) or_leave_molecules(&st, n, t1, c, out + 4 * (size_t)i);
}

void or_binom_many(uint64_t seed, uint32_t unit, uint32_t n, double p, uint32_t count, uint32_t* out) {
    or_stream st;
    or_stream_init(&st, seed, 0, unit, 0, 0);
    for (uint32_t i = 0; i < count; ++i) out[i] = or_binom(&st, n, p);
}

/* ------------------------------------------------------------------------- */
/* Model x mesh tables                                                        */
/* ------------------------------------------------------------------------- */
#define OR_MAXR 256
#define OR_MAXS 32

typedef struct {
    int comp;
    uint32_t lhs[OR_MAXS];
    int32_t upd[OR_MAXS];
    int order;
} or_reac;

typedef struct {
    uint64_t seed;
    int ntets, nspec, ncomp, nreal, nreac;
    const double* vol;
    const int32_t* neighb;
    const double* area;
    const double* dist;
    const int32_t* tcomp;
    const int32_t* real_begin; /* nreal + 1 */
    or_reac reac[OR_MAXR];
    double* kcst;              /* [nreal][nreac] */
    double* dcst;              /* [nreal][ncomp][nspec] */
    int has_rule[OR_MAXS];
    /* derived */
    float* geo;                /* [T][4]: c0 c1 c2 G */
    int32_t* nbr;              /* [T][4]: neighbour or -1 */
    int32_t* rface;            /* [T][4]: face of the neighbour pointing back */
    double* ivs;               /* [T] */
    uint32_t* clamp;           /* [T] */
    uint32_t* counts;          /* [S][T] */
    uint32_t* outflow;         /* [S][T][4] scratch of one window */
    double* t;                 /* [nreal] */
    double* period;            /* [nreal] */
    uint64_t* window;          /* [nreal] */
    uint64_t ext[OR_MAXR];
    uint64_t diff_moved;
    /* Diffusion boundaries (diffboundary.cpp; Diff::setDiffBndActive diff.cpp:307 and
     * setDirectionDcst :394): boundary of each face, the two compartments of each boundary,
     * the rate table [nbnd][S][side] (-1 closed, -2 at the source's own constant, >= 0 at
     * that constant), face coefficients A/(V d) of tets with a boundary face (float), and
     * the face of the neighbour behind each boundary face. */
    int nbnd;
    const int32_t* face_bnd;
    const int32_t* bnd_comps;
    double* btab;
    float* bcoef;
    int32_t* bnbr;
    /* Membrane (sreac.cpp, vdepsreac.cpp, ghkcurr.cpp, sdiff.cpp): triangles m = 0..M-1
     * with inner tet, patch and area; surface counts [SS][M]; the triangles of each tet's
     * SSA unit (slot order = ascending m); surface reactions grouped by patch; k(V) tables;
     * GHK currents; surface diffusion tables.  Triangle potentials (mV) default to 0. */
    int nsspec, ntris, npatch;
    const int32_t* tri_inner;
    const int32_t* tri_patch;
    const double* tri_area;
    int32_t* tet_tris;         /* [T][4] */
    uint32_t* tri_counts;      /* [SS][M] */
    double* tri_v;             /* [M] mV */
    double* spec_int;          /* [SS][M] count time integrals */
    int64_t* echarge;          /* [M] elementary charges carried by GHK events */
    uint64_t surf_ext;
    struct or_sreac* sreacs;
    int nsreac;
    int* patch_sb;             /* [npatch + 1] */
    double* vt_vmin;
    double* vt_dv;
    int* vt_off;
    int* vt_n;
    int nvt;
    double* vt_vals;
    int nvt_vals;
    struct or_ghk* ghks;
    int nghk;
    double temp;
    double* sdcst;             /* [npatch][SS] */
    const int32_t* tri_nbr;    /* [M][3] */
    const int32_t* tri_nbr_edge;
    const double* tri_len;
    const double* tri_dist;
    int32_t* sdiff_slot;       /* [SS] */
    int nsdiff;
    int32_t* sdspec;           /* [SD] */
    float* sgeo;               /* [M][4] */
    int32_t* snbr;             /* [M][4] (q << 2) | edge */
    double* tri_occ;           /* [SD][M] */
    uint32_t* tri_out;         /* [SD][M][4] */
    /* Merged SSA units (sreac.cpp:200-300: a triangle and both its tets in one SSA): outer
     * tet of each triangle, unit of each tet (-1), the units' tets and triangles (ascending),
     * and the change-time sums their SSA hands to the diffusion leave. */
    const int32_t* tri_outer;  /* [M] or NULL */
    int nunits;
    int32_t* tet_unit;         /* [T] */
    int32_t* u_tb;             /* [U + 1] */
    int32_t* u_tets;
    int32_t* u_mb;             /* [U + 1] */
    int32_t* u_tris;
    double* utdel;             /* [T][S] */
} or_solver;

typedef struct or_sreac {
    int patch, order, surf_surf, vdep;
    int nslhs, nilhs, nsupd, niupd;
    int slhs_spec[4], slhs_ord[4], ilhs_spec[4], ilhs_ord[4];
    int supd_spec[8], supd_delta[8], iupd_spec[8], iupd_delta[8];
    int vside, noupd, oupd_spec[8], oupd_delta[8]; /* volume reactants in the outer tet; outer changes */
    double k;
} or_sreac;

typedef struct or_ghk {
    int patch, sspec, ion, valence, realflux;
    double perm, vshift, voconc;
} or_ghk;

static void or_setup_surface(or_solver* s);

or_solver* or_create(uint64_t seed, int ntets, int nspec, int ncomp, const double* vol,
                     const int32_t* neighb, const double* area, const double* dist,
                     const int32_t* tcomp, int nreal, const int32_t* real_begin) {
    if (nspec > OR_MAXS) return NULL;
    or_solver* s = (or_solver*)calloc(1, sizeof(or_solver));
    s->seed = seed;
    s->ntets = ntets;
    s->nspec = nspec;
    s->ncomp = ncomp;
    s->nreal = nreal;
    s->vol = vol;
    s->neighb = neighb;
    s->area = area;
    s->dist = dist;
    s->tcomp = tcomp;
    s->real_begin = real_begin;
    s->dcst = (double*)calloc((size_t)nreal * ncomp * nspec, sizeof(double));
    s->counts = (uint32_t*)calloc((size_t)nspec * ntets, 4);
    s->outflow = (uint32_t*)calloc((size_t)nspec * ntets * 4, 4);
    s->clamp = (uint32_t*)calloc((size_t)ntets, 4);
    s->t = (double*)calloc(nreal, sizeof(double));
    s->period = (double*)calloc(nreal, sizeof(double));
    s->window = (uint64_t*)calloc(nreal, sizeof(uint64_t));
    return s;
}

void or_destroy(or_solver* s) {
    if (!s) return;
    free(s->kcst);
    free(s->dcst);
    free(s->geo);
    free(s->nbr);
    free(s->rface);
    free(s->ivs);
    free(s->clamp);
    free(s->counts);
    free(s->outflow);
    free(s->t);
    free(s->period);
    free(s->window);
    free(s->btab);
    free(s->bcoef);
    free(s->bnbr);
    free(s->tet_tris);
    free(s->tet_unit);
    free(s->u_tb);
    free(s->u_tets);
    free(s->u_mb);
    free(s->u_tris);
    free(s->utdel);
    free(s->tri_counts);
    free(s->tri_v);
    free(s->spec_int);
    free(s->echarge);
    free(s->sreacs);
    free(s->patch_sb);
    free(s->vt_vmin);
    free(s->vt_dv);
    free(s->vt_off);
    free(s->vt_n);
    free(s->vt_vals);
    free(s->ghks);
    free(s->sdcst);
    free(s->sdiff_slot);
    free(s->sdspec);
    free(s->sgeo);
    free(s->snbr);
    free(s->tri_occ);
    free(s->tri_out);
    free(s);
}

/* Before or_setup: the boundary tables (the arrays are kept by reference). */
void or_set_boundaries(or_solver* s, int nbnd, const int32_t* face_bnd, const int32_t* bnd_comps) {
    s->nbnd = nbnd;
    s->face_bnd = face_bnd;
    s->bnd_comps = bnd_comps;
    s->btab = (double*)malloc(sizeof(double) * (size_t)nbnd * s->nspec * 2);
    for (size_t i = 0; i < (size_t)nbnd * s->nspec * 2; ++i) s->btab[i] = -1.0;
}

static int or_has_bnd(const or_solver* s, int t) {
    if (!s->nbnd) return 0;
    for (int f = 0; f < 4; ++f)
        if (s->face_bnd[(size_t)t * 4 + f] >= 0) return 1;
    return 0;
}

/* Face rates of tet t for species sp at constant D when it has boundary faces; returns the
 * total and the float conditional selectors (last open face takes the rest). */
static double or_bnd_split(const or_solver* s, int t, int sp, double D, float cs[3]) {
    double r[4];
    const int c = s->tcomp[t];
    for (int f = 0; f < 4; ++f) {
        r[f] = 0.0;
        const double cf = (double)s->bcoef[(size_t)t * 4 + f];
        if (s->nbr[(size_t)t * 4 + f] >= 0) {
            r[f] = cf * D;
            continue;
        }
        const int b = s->face_bnd[(size_t)t * 4 + f];
        if (b < 0) continue;
        const int side = (c == s->bnd_comps[(size_t)b * 2]) ? 0 : 1;
        const double v = s->btab[((size_t)b * s->nspec + sp) * 2 + side];
        if (v < -1.5) r[f] = cf * D;
        else if (v >= 0.0) r[f] = cf * v;
    }
    const double tot = r[0] + r[1] + r[2] + r[3];
    int lastf = -1;
    for (int f = 0; f < 4; ++f)
        if (r[f] > 0.0) lastf = f;
    double rem = tot;
    for (int f = 0; f < 3; ++f) {
        double q = 0.0;
        if (r[f] > 0.0) {
            q = (f == lastf) ? 1.0 : r[f] / rem;
            if (q > 1.0) q = 1.0;
            rem -= r[f];
        }
        cs[f] = (float)q;
    }
    return tot;
}

/* Reactions are appended per compartment in the order given (the caller passes them
 * grouped by compartment, keeping the model order inside a compartment). */
int or_add_reac(or_solver* s, int comp, const uint32_t* lhs, const int32_t* upd, double kcst) {
    if (s->nreac >= OR_MAXR) return -1;
    or_reac* r = &s->reac[s->nreac];
    r->comp = comp;
    r->order = 0;
    for (int i = 0; i < s->nspec; ++i) {
        r->lhs[i] = lhs[i];
        r->upd[i] = upd[i];
        r->order += (int)lhs[i];
    }
    int R = s->nreac;
    double* k = (double*)malloc(sizeof(double) * (size_t)s->nreal * (R + 1));
    for (int rr = 0; rr < s->nreal; ++rr) {
        for (int i = 0; i < R; ++i) k[(size_t)rr * (R + 1) + i] = s->kcst[(size_t)rr * R + i];
        k[(size_t)rr * (R + 1) + R] = kcst;
    }
    free(s->kcst);
    s->kcst = k;
    s->nreac = R + 1;
    return R;
}

void or_add_diff(or_solver* s, int comp, int spec, double dcst) {
    s->has_rule[spec] = 1;
    for (int r = 0; r < s->nreal; ++r) s->dcst[((size_t)r * s->ncomp + comp) * s->nspec + spec] = dcst;
}

void or_set_reac_k(or_solver* s, int reac, int real, double k) {
    s->kcst[(size_t)real * s->nreac + reac] = k;
}

static void or_periods(or_solver* s) {
    for (int r = 0; r < s->nreal; ++r) {
        double mx = 0.0;
        for (int t = s->real_begin[r]; t < s->real_begin[r + 1]; ++t) {
            int c = s->tcomp[t];
            if (c < 0) continue;
            double G = (double)s->geo[(size_t)t * 4 + 3];
            for (int sp = 0; sp < s->nspec; ++sp) {
                if (!s->has_rule[sp]) continue;
                const double D = s->dcst[((size_t)r * s->ncomp + c) * s->nspec + sp];
                double sd = D * G;
                if (or_has_bnd(s, t)) {
                    float cs[3];
                    sd = or_bnd_split(s, t, sp, D, cs);
                }
                if (sd > mx) mx = sd;
            }
        }
        /* Surface diffusion rules count too (TOS:5373-5411 takes the max over both). */
        for (int m = 0; s->nsdiff > 0 && m < s->ntris; ++m) {
            const int t = s->tri_inner[m];
            if (t < s->real_begin[r] || t >= s->real_begin[r + 1]) continue;
            const double G = (double)s->sgeo[(size_t)m * 4 + 3];
            for (int sp = 0; sp < s->nsspec; ++sp) {
                const double sd = s->sdcst[(size_t)s->tri_patch[m] * s->nsspec + sp] * G;
                if (sd > mx) mx = sd;
            }
        }
        s->period[r] = (mx > 0.0) ? 1.0 / mx : INFINITY;
    }
}

/* Scaled diffusion constant and face selector as Diff::Diff (diff.cpp:41-90): faces to a
 * neighbour of the same compartment with positive distance carry A_f / (V d_f); the
 * conditional selectors c_f = g_f / (G - sum_{j<f} g_j) drive the sequential binomial split
 * of Diff::apply (diff.cpp:515-585); the last active face takes the remainder. */
int or_setup(or_solver* s) {
    int T = s->ntets;
    s->geo = (float*)calloc((size_t)T * 4, sizeof(float));
    s->nbr = (int32_t*)malloc((size_t)T * 4 * 4);
    s->rface = (int32_t*)malloc((size_t)T * 4 * 4);
    s->ivs = (double*)calloc(T, sizeof(double));
    for (int t = 0; t < T; ++t) {
        int c = s->tcomp[t];
        s->ivs[t] = 1.0 / (1.0e3 * s->vol[t] * 6.02214179e23); /* math/constants.hpp:45 */
        double g[4] = {0, 0, 0, 0};
        for (int f = 0; f < 4; ++f) {
            int n = s->neighb[(size_t)t * 4 + f];
            s->nbr[(size_t)t * 4 + f] = -1;
            s->rface[(size_t)t * 4 + f] = -1;
            if (n < 0) continue;
            int rf = -1;
            for (int j = 0; j < 4; ++j)
                if (s->neighb[(size_t)n * 4 + j] == t) rf = j;
            if (rf < 0) return -1;
            double d = s->dist[(size_t)t * 4 + f];
            if (c >= 0 && d > 0.0 && s->tcomp[n] == c) {
                g[f] = s->area[(size_t)t * 4 + f] / (s->vol[t] * d);
                s->nbr[(size_t)t * 4 + f] = n;
                s->rface[(size_t)t * 4 + f] = rf;
            }
        }
        double G = g[0] + g[1] + g[2] + g[3];
        int lastf = -1;
        for (int f = 0; f < 4; ++f)
            if (g[f] > 0.0) lastf = f;
        double rem = G;
        for (int f = 0; f < 3; ++f) {
            double cf = 0.0;
            if (g[f] > 0.0) {
                cf = (f == lastf) ? 1.0 : g[f] / rem;
                if (cf > 1.0) cf = 1.0;
                rem -= g[f];
            }
            s->geo[(size_t)t * 4 + f] = (float)cf;
        }
        s->geo[(size_t)t * 4 + 3] = (float)G;
    }
    if (s->nbnd) {
        s->bcoef = (float*)calloc((size_t)T * 4, sizeof(float));
        s->bnbr = (int32_t*)malloc((size_t)T * 4 * 4);
        for (int t = 0; t < T; ++t)
            for (int f = 0; f < 4; ++f) {
                s->bnbr[(size_t)t * 4 + f] = -1;
                int n = s->neighb[(size_t)t * 4 + f];
                if (n < 0) continue;
                if (s->face_bnd[(size_t)t * 4 + f] >= 0) {
                    int rf = -1;
                    for (int j = 0; j < 4; ++j)
                        if (s->neighb[(size_t)n * 4 + j] == t) rf = j;
                    s->bnbr[(size_t)t * 4 + f] = n * 4 + rf;
                }
            }
        for (int t = 0; t < T; ++t) {
            if (!or_has_bnd(s, t)) continue;
            for (int f = 0; f < 4; ++f) {
                const int n = s->neighb[(size_t)t * 4 + f];
                const double d = s->dist[(size_t)t * 4 + f];
                if (n >= 0 && d > 0.0)
                    s->bcoef[(size_t)t * 4 + f] = (float)(s->area[(size_t)t * 4 + f] / (s->vol[t] * d));
            }
        }
    }
    if (s->ntris > 0) or_setup_surface(s);
    or_periods(s);
    return 0;
}

/* ---- membrane builders (before or_setup; arrays kept by reference) ---- */
void or_set_surface(or_solver* s, int nsspec, int ntris, const int32_t* tri_inner, const int32_t* tri_patch,
                    const double* tri_area, int npatch) {
    s->nsspec = nsspec;
    s->ntris = ntris;
    s->npatch = npatch;
    s->tri_inner = tri_inner;
    s->tri_patch = tri_patch;
    s->tri_area = tri_area;
    s->tri_counts = (uint32_t*)calloc((size_t)nsspec * ntris, 4);
    s->tri_v = (double*)calloc((size_t)ntris, sizeof(double));
    s->spec_int = (double*)calloc((size_t)nsspec * ntris, sizeof(double));
    s->echarge = (int64_t*)calloc((size_t)ntris, sizeof(int64_t));
    s->sdcst = (double*)calloc((size_t)npatch * nsspec, sizeof(double));
    s->temp = 293.15;
}

/* One surface reaction: dense rows over the surface (slhs, supd) and volume (ilhs, iupd)
 * species, compacted in increasing species order as the GPU solver's tables; a k(V) table
 * (vmin, dv, n values) when vals is given, else the constant k.  Returns its index. */
int or_add_sreac(or_solver* s, int patch, const uint32_t* slhs, const uint32_t* ilhs, const int32_t* supd,
                 const int32_t* iupd, double k, double vmin, double dv, int ntab, const double* vals) {
    s->sreacs = (or_sreac*)realloc(s->sreacs, sizeof(or_sreac) * (size_t)(s->nsreac + 1));
    or_sreac* r = &s->sreacs[s->nsreac];
    memset(r, 0, sizeof(*r));
    r->patch = patch;
    r->vdep = -1;
    r->k = k;
    for (int i = 0; i < s->nsspec; ++i)
        if (slhs[i]) {
            r->slhs_spec[r->nslhs] = i;
            r->slhs_ord[r->nslhs++] = (int)slhs[i];
            r->order += (int)slhs[i];
        }
    for (int i = 0; i < s->nspec; ++i)
        if (ilhs[i]) {
            r->ilhs_spec[r->nilhs] = i;
            r->ilhs_ord[r->nilhs++] = (int)ilhs[i];
            r->order += (int)ilhs[i];
        }
    r->surf_surf = r->nilhs == 0;
    for (int i = 0; i < s->nsspec; ++i)
        if (supd[i]) {
            r->supd_spec[r->nsupd] = i;
            r->supd_delta[r->nsupd++] = supd[i];
        }
    for (int i = 0; i < s->nspec; ++i)
        if (iupd[i]) {
            r->iupd_spec[r->niupd] = i;
            r->iupd_delta[r->niupd++] = iupd[i];
        }
    if (vals) {
        int v = s->nvt++;
        s->vt_vmin = (double*)realloc(s->vt_vmin, sizeof(double) * s->nvt);
        s->vt_dv = (double*)realloc(s->vt_dv, sizeof(double) * s->nvt);
        s->vt_off = (int*)realloc(s->vt_off, sizeof(int) * s->nvt);
        s->vt_n = (int*)realloc(s->vt_n, sizeof(int) * s->nvt);
        s->vt_vmin[v] = vmin;
        s->vt_dv[v] = dv;
        s->vt_off[v] = s->nvt_vals;
        s->vt_n[v] = ntab;
        s->vt_vals = (double*)realloc(s->vt_vals, sizeof(double) * (size_t)(s->nvt_vals + ntab));
        memcpy(s->vt_vals + s->nvt_vals, vals, sizeof(double) * (size_t)ntab);
        s->nvt_vals += ntab;
        r->vdep = v;
        r->k = 0.0;
    }
    return s->nsreac++;
}

void or_add_ghk(or_solver* s, int patch, int sspec, int ion, int valence, double perm, double vshift,
                double voconc, int realflux) {
    s->ghks = (or_ghk*)realloc(s->ghks, sizeof(or_ghk) * (size_t)(s->nghk + 1));
    or_ghk* g = &s->ghks[s->nghk++];
    g->patch = patch;
    g->sspec = sspec;
    g->ion = ion;
    g->valence = valence;
    g->perm = perm;
    g->vshift = vshift;
    g->voconc = voconc;
    g->realflux = realflux;
}

void or_set_temp(or_solver* s, double kelvin) { s->temp = kelvin; }

/* Outer tet of every membrane triangle (-1 none); kept by reference. */
void or_set_tri_outer(or_solver* s, const int32_t* tri_outer) { s->tri_outer = tri_outer; }

/* Outer-volume terms of surface reaction idx (the index or_add_sreac returned): reactants
 * olhs in the outer tet (SReacdef::outside; the constant then scales with the outer tet's
 * volume) and changes oupd of outer-tet species, dense over the volume species. */
void or_set_sreac_outer(or_solver* s, int idx, const uint32_t* olhs, const int32_t* oupd) {
    or_sreac* r = &s->sreacs[idx];
    int n = 0;
    for (int i = 0; i < s->nspec; ++i)
        if (olhs[i]) ++n;
    if (n > 0) {
        r->nilhs = 0;
        for (int i = 0; i < s->nspec; ++i)
            if (olhs[i]) {
                r->ilhs_spec[r->nilhs] = i;
                r->ilhs_ord[r->nilhs++] = (int)olhs[i];
                r->order += (int)olhs[i];
            }
        r->vside = 1;
        r->surf_surf = 0;
    }
    r->noupd = 0;
    for (int i = 0; i < s->nspec; ++i)
        if (oupd[i]) {
            r->oupd_spec[r->noupd] = i;
            r->oupd_delta[r->noupd++] = oupd[i];
        }
}

static int or_patch_coupled(const or_solver* s, int p) {
    for (int i = 0; i < s->nsreac; ++i)
        if (s->sreacs[i].patch == p && (s->sreacs[i].vside || s->sreacs[i].noupd > 0)) return 1;
    for (int g = 0; g < s->nghk; ++g)
        if (s->ghks[g].patch == p && s->ghks[g].voconc < 0.0) return 1;
    return 0;
}

static int or_find(int32_t* par, int x) {
    while (par[x] != x) x = par[x] = par[par[x]];
    return x;
}

/* Units: tets joined through the triangles of coupled patches (inner with outer tet);
 * groups of two or more tets, numbered by their lowest tet, each with the triangles whose
 * inner tet is in the group. */
static void or_setup_units(or_solver* s) {
    const int T = s->ntets, M = s->ntris;
    s->nunits = 0;
    if (!s->tri_outer) return;
    int any = 0;
    for (int p = 0; p < s->npatch; ++p) any |= or_patch_coupled(s, p);
    if (!any) return;
    int32_t* par = (int32_t*)malloc(sizeof(int32_t) * (size_t)T);
    int32_t* sz = (int32_t*)calloc((size_t)T, sizeof(int32_t));
    int32_t* uid = (int32_t*)malloc(sizeof(int32_t) * (size_t)T);
    for (int t = 0; t < T; ++t) par[t] = t, uid[t] = -1;
    for (int m = 0; m < M; ++m) {
        if (!or_patch_coupled(s, s->tri_patch[m]) || s->tri_outer[m] < 0) continue;
        int a = or_find(par, s->tri_inner[m]), b = or_find(par, s->tri_outer[m]);
        if (a != b) par[a < b ? b : a] = a < b ? a : b;
    }
    for (int t = 0; t < T; ++t) sz[or_find(par, t)] += 1;
    s->tet_unit = (int32_t*)malloc(sizeof(int32_t) * (size_t)T);
    for (int t = 0; t < T; ++t) {
        const int root = or_find(par, t);
        s->tet_unit[t] = -1;
        if (sz[root] < 2) continue;
        if (uid[root] < 0) uid[root] = s->nunits++;
        s->tet_unit[t] = uid[root];
    }
    const int U = s->nunits;
    s->u_tb = (int32_t*)calloc((size_t)U + 1, sizeof(int32_t));
    s->u_mb = (int32_t*)calloc((size_t)U + 1, sizeof(int32_t));
    for (int t = 0; t < T; ++t)
        if (s->tet_unit[t] >= 0) s->u_tb[s->tet_unit[t] + 1] += 1;
    for (int m = 0; m < M; ++m)
        if (s->tet_unit[s->tri_inner[m]] >= 0) s->u_mb[s->tet_unit[s->tri_inner[m]] + 1] += 1;
    for (int u = 0; u < U; ++u) {
        s->u_tb[u + 1] += s->u_tb[u];
        s->u_mb[u + 1] += s->u_mb[u];
    }
    s->u_tets = (int32_t*)malloc(sizeof(int32_t) * (size_t)(s->u_tb[U] + 1));
    s->u_tris = (int32_t*)malloc(sizeof(int32_t) * (size_t)(s->u_mb[U] + 1));
    int32_t* fill = (int32_t*)calloc((size_t)U + 1, sizeof(int32_t));
    for (int t = 0; t < T; ++t) {
        const int u = s->tet_unit[t];
        if (u >= 0) s->u_tets[s->u_tb[u] + fill[u]++] = t;
    }
    memset(fill, 0, sizeof(int32_t) * (size_t)(U + 1));
    for (int m = 0; m < M; ++m) {
        const int u = s->tet_unit[s->tri_inner[m]];
        if (u >= 0) s->u_tris[s->u_mb[u] + fill[u]++] = m;
    }
    s->utdel = (double*)calloc((size_t)T * s->nspec, sizeof(double));
    free(fill);
    free(par);
    free(sz);
    free(uid);
}

void or_set_tri_neighbours(or_solver* s, const int32_t* nbr, const int32_t* nbr_edge, const double* len,
                           const double* dist) {
    s->tri_nbr = nbr;
    s->tri_nbr_edge = nbr_edge;
    s->tri_len = len;
    s->tri_dist = dist;
}

void or_add_sdiff(or_solver* s, int patch, int sspec, double dcst) { s->sdcst[(size_t)patch * s->nsspec + sspec] = dcst; }

/* Surface reactions grouped by patch (stable), the SSA units' triangle slots, and the
 * surface diffusion tables (sdiff.cpp:62-83): edge coefficients l / (A d) towards same-patch
 * neighbours, G = their sum, conditional selectors c0 = g0 / G, c1 = g1 / (g1 + g2). */
static void or_setup_surface(or_solver* s) {
    const int R = s->nsreac, P = s->npatch, M = s->ntris, SS = s->nsspec;
    or_sreac* sorted = (or_sreac*)malloc(sizeof(or_sreac) * (size_t)(R > 0 ? R : 1));
    int n = 0;
    for (int p = 0; p < P; ++p)
        for (int i = 0; i < R; ++i)
            if (s->sreacs[i].patch == p) sorted[n++] = s->sreacs[i];
    free(s->sreacs);
    s->sreacs = sorted;
    s->patch_sb = (int*)calloc((size_t)P + 1, sizeof(int));
    for (int i = 0; i < R; ++i) s->patch_sb[s->sreacs[i].patch + 1] += 1;
    for (int p = 0; p < P; ++p) s->patch_sb[p + 1] += s->patch_sb[p];
    s->tet_tris = (int32_t*)malloc(sizeof(int32_t) * (size_t)s->ntets * 4);
    for (size_t i = 0; i < (size_t)s->ntets * 4; ++i) s->tet_tris[i] = -1;
    for (int m = 0; m < M; ++m) {
        const int t = s->tri_inner[m];
        int slot = 0;
        while (slot < 4 && s->tet_tris[(size_t)t * 4 + slot] >= 0) ++slot;
        s->tet_tris[(size_t)t * 4 + slot] = m;
    }
    or_setup_units(s);
    s->sdiff_slot = (int32_t*)malloc(sizeof(int32_t) * (size_t)(SS > 0 ? SS : 1));
    s->nsdiff = 0;
    int any = 0;
    for (size_t i = 0; i < (size_t)P * SS; ++i)
        if (s->sdcst[i] > 0.0) any = 1;
    for (int sp = 0; sp < SS; ++sp) s->sdiff_slot[sp] = -1;
    if (!any) return;
    s->sdspec = (int32_t*)malloc(sizeof(int32_t) * (size_t)SS);
    for (int sp = 0; sp < SS; ++sp) {
        int has = 0;
        for (int p = 0; p < P; ++p)
            if (s->sdcst[(size_t)p * SS + sp] > 0.0) has = 1;
        if (has) {
            s->sdiff_slot[sp] = s->nsdiff;
            s->sdspec[s->nsdiff++] = sp;
        }
    }
    s->sgeo = (float*)calloc((size_t)M * 4, sizeof(float));
    s->snbr = (int32_t*)malloc(sizeof(int32_t) * (size_t)M * 4);
    for (int m = 0; m < M; ++m) {
        double g[3] = {0.0, 0.0, 0.0};
        for (int e = 0; e < 4; ++e) s->snbr[(size_t)m * 4 + e] = -1;
        for (int e = 0; e < 3; ++e) {
            const int q = s->tri_nbr[(size_t)m * 3 + e];
            if (q < 0 || s->tri_patch[q] != s->tri_patch[m]) continue;
            const double d = s->tri_dist[(size_t)m * 3 + e];
            if (!(d > 0.0)) continue;
            g[e] = s->tri_len[(size_t)m * 3 + e] / (s->tri_area[m] * d);
            s->snbr[(size_t)m * 4 + e] = (q << 2) | s->tri_nbr_edge[(size_t)m * 3 + e];
        }
        const double G = g[0] + g[1] + g[2];
        const double r12 = g[1] + g[2];
        s->sgeo[(size_t)m * 4 + 0] = G > 0.0 ? (float)(g[0] / G) : 0.0f;
        s->sgeo[(size_t)m * 4 + 1] = r12 > 0.0 ? (float)(g[1] / r12) : 0.0f;
        s->sgeo[(size_t)m * 4 + 2] = 1.0f;
        s->sgeo[(size_t)m * 4 + 3] = (float)G;
    }
    s->tri_occ = (double*)calloc((size_t)s->nsdiff * M, sizeof(double));
    s->tri_out = (uint32_t*)calloc((size_t)s->nsdiff * M * 4, 4);
}

void or_set_tri_counts(or_solver* s, int sspec, const uint32_t* row) {
    memcpy(s->tri_counts + (size_t)sspec * s->ntris, row, (size_t)s->ntris * 4);
}
void or_get_tri_counts(or_solver* s, int sspec, uint32_t* row) {
    memcpy(row, s->tri_counts + (size_t)sspec * s->ntris, (size_t)s->ntris * 4);
}
void or_set_tri_v(or_solver* s, const double* v_mV) { memcpy(s->tri_v, v_mV, sizeof(double) * (size_t)s->ntris); }
uint64_t or_get_surf_ext(or_solver* s) { return s->surf_ext; }
void or_get_echarge(or_solver* s, int64_t* out) { memcpy(out, s->echarge, sizeof(int64_t) * (size_t)s->ntris); }
void or_get_spec_int(or_solver* s, double* out) {
    memcpy(out, s->spec_int, sizeof(double) * (size_t)s->nsspec * s->ntris);
}

/* setDiffBoundarySpecDiffusionActive / setDiffBoundarySpecDcst outcome: the rate table. */
void or_set_btab(or_solver* s, const double* btab) {
    memcpy(s->btab, btab, sizeof(double) * (size_t)s->nbnd * s->nspec * 2);
    or_periods(s);
}

void or_set_counts(or_solver* s, int spec, const uint32_t* row) {
    memcpy(s->counts + (size_t)spec * s->ntets, row, (size_t)s->ntets * 4);
}
void or_get_counts(or_solver* s, int spec, uint32_t* row) {
    memcpy(row, s->counts + (size_t)spec * s->ntets, (size_t)s->ntets * 4);
}
void or_set_clamped(or_solver* s, int tet, int spec, int on) {
    if (on)
        s->clamp[tet] |= 1u << spec;
    else
        s->clamp[tet] &= ~(1u << spec);
}
void or_set_time(or_solver* s, int real, double t, uint64_t window) {
    s->t[real] = t;
    s->window[real] = window;
}
double or_get_time(or_solver* s, int real) { return s->t[real]; }
uint64_t or_get_window(or_solver* s, int real) { return s->window[real]; }
double or_get_period(or_solver* s, int real) { return s->period[real]; }
uint64_t or_get_reac_extent(or_solver* s, int reac) { return s->ext[reac]; }
uint64_t or_get_diff_extent(or_solver* s) { return s->diff_moved; }

/* ------------------------------------------------------------------------- */
/* One split window                                                           */
/* ------------------------------------------------------------------------- */

/* Reac::rate (reac.cpp:184-232): h_mu = prod falling factorials, times
 * ccst = k (1e3 V N_A)^(1 - order) (reac.cpp:44-53). */
static double or_prop(const or_solver* s, const or_reac* r, const uint32_t* cnt, double k, double ivs) {
    double ccst;
    if (r->order == 1)
        ccst = k;
    else if (r->order == 0)
        ccst = k / ivs;
    else {
        ccst = k * ivs;
        for (int i = 2; i < r->order; ++i) ccst = ccst * ivs;
    }
    double h = 1.0;
    for (int i = 0; i < s->nspec; ++i) {
        uint32_t o = r->lhs[i];
        if (o == 0) continue;
        uint32_t c = cnt[i];
        if (o > c) return 0.0;
        if (o >= 4) h = h * (double)(c - 3);
        if (o >= 3) h = h * (double)(c - 2);
        if (o >= 2) h = h * (double)(c - 1);
        h = h * (double)c;
    }
    return h * ccst;
}

/* ---- membrane SSA units ---- */
#define OR_FARADAY 96485.3399       /* math/constants.hpp:49 */
#define OR_GAS_CONSTANT 8.314472    /* constants.hpp:53 */
#define OR_E_CHARGE 1.602176487e-19 /* constants.hpp:57 */
#define OR_AVOGADRO 6.02214179e23   /* constants.hpp:45 */

/* k(V) by linear interpolation in the table (vdepsreacdef.cpp:194-218). */
static double or_vdep_k(const or_solver* s, int v, double v_mV) {
    double vv = v_mV * 1.0e-3;
    double v2 = (vv - s->vt_vmin[v]) / s->vt_dv[v];
    if (!(v2 >= 0.0) || v2 > (double)(s->vt_n[v] - 1)) v2 = v2 < 0.0 ? 0.0 : (double)(s->vt_n[v] - 1);
    double lv = floor(v2);
    int lo = (int)lv, hi = (int)ceil(v2);
    double r = v2 - lv;
    const double* K = s->vt_vals + s->vt_off[v];
    return (1.0 - r) * K[lo] + r * K[hi];
}

/* Single-channel GHK current (math/ghk.cpp:71-90), concentrations in mol/m^3. */
static double or_ghk_current(double P, double v, int z, double temp, double ci, double co) {
    const double nu = (double)z * v * OR_FARADAY / (OR_GAS_CONSTANT * temp);
    if (!(nu < 700.0 && nu > -700.0)) return 0.0;
    if (fabs(nu) > 2.220446049250313e-16) {
        const double e = or_exp(-nu);
        return P * (double)z * OR_FARADAY * nu * (ci - co * e) / (1.0 - e);
    }
    return P * (double)z * OR_FARADAY * (ci - co);
}

/* Signed ion rate (/s) of a GHK current on a triangle with n channels (ghkcurr.cpp:168-212). */
static double or_ghk_rate(const or_ghk* g, double vm, uint32_t c_ion, uint32_t n, double ivs, double temp) {
    if (n == 0) return 0.0;
    const double ci = (double)c_ion * ivs * 1.0e3;
    const double co = g->voconc * 1.0e3;
    const double I = or_ghk_current(g->perm, vm * 1.0e-3 + g->vshift, g->valence, temp, ci, co);
    return I / (OR_E_CHARGE * (double)g->valence) * (double)n;
}

/* Scaled constant of a surface reaction (sreac.cpp:40-68: by area when no volume reactant). */
static double or_sreac_ccst(const or_sreac* r, double k, double ivs, double area) {
    if (r->surf_surf) {
        double ascale = area * OR_AVOGADRO;
        if (r->order == 0) return k * ascale;
        double c = k;
        for (int i = 1; i < r->order; ++i) c = c / ascale;
        return c;
    }
    if (r->order == 0) return k / ivs;
    double c = k;
    for (int i = 1; i < r->order; ++i) c = c * ivs;
    return c;
}

static double or_falling(uint32_t c, uint32_t o) {
    double h = 1.0;
    if (o >= 4) h = h * (double)(c - 3);
    if (o >= 3) h = h * (double)(c - 2);
    if (o >= 2) h = h * (double)(c - 1);
    return h * (double)c;
}

static double or_sreac_h(const or_sreac* r, const uint32_t* sc, const uint32_t* vc) {
    double h = 1.0;
    for (int i = 0; i < r->nslhs; ++i) {
        uint32_t c = sc[r->slhs_spec[i]], o = (uint32_t)r->slhs_ord[i];
        if (o > c) return 0.0;
        h = h * or_falling(c, o);
    }
    for (int i = 0; i < r->nilhs; ++i) {
        uint32_t c = vc[r->ilhs_spec[i]], o = (uint32_t)r->ilhs_ord[i];
        if (o > c) return 0.0;
        h = h * or_falling(c, o);
    }
    return h;
}

static uint32_t or_bump(uint32_t old, int64_t d) {
    int64_t nc = (int64_t)old + d;
    if (nc < 0) nc = 0;
    if (nc > 0xFFFFFFFFll) nc = 0xFFFFFFFFll;
    return (uint32_t)nc;
}

/* SSA of the unit tet t + its membrane triangles over [0, T) (sreac.cpp:305-520): volume
 * reactions, then each triangle's surface reactions and GHK currents, all propensities
 * re-evaluated after every event; surface counts integrate their occupancy (tri.cpp:486-561).
 * Draws continue the unit's stream st.  Surface-diffusion inflow of the last window was
 * already added to the triangle counts. */
static void or_ssa_surf(or_solver* s, int t, double T, uint32_t* cnt, double* tdel, or_stream* st, uint32_t clampm,
                        double ivs, const double* K, int rb, int re) {
    const int SS = s->nsspec, M = s->ntris;
    int mm[4], pb[4], pe[4], pj[4];
    double area[4], vm[4];
    uint32_t sc[4][OR_MAXS];
    double occ[4][OR_MAXS], last[4][OR_MAXS];
    double prop[OR_MAXR], sprop[4][OR_MAXR];
    for (int j = 0; j < 4; ++j) {
        mm[j] = s->tet_tris[(size_t)t * 4 + j];
        pb[j] = pe[j] = 0;
        pj[j] = -1;
        area[j] = vm[j] = 0.0;
        if (mm[j] < 0) continue;
        const int m = mm[j], p = s->tri_patch[m];
        pj[j] = p;
        pb[j] = s->patch_sb[p];
        pe[j] = s->patch_sb[p + 1];
        area[j] = s->tri_area[m];
        vm[j] = s->tri_v[m];
        for (int k = 0; k < SS; ++k) {
            sc[j][k] = s->tri_counts[(size_t)k * M + m];
            occ[j][k] = 0.0;
            last[j][k] = 0.0;
        }
    }
    double tt = 0.0;
    for (;;) {
        double a0 = 0.0;
        for (int q = rb; q >= 0 && q < re; ++q) {
            const double pq = or_prop(s, &s->reac[q], cnt, K[q], ivs);
            prop[q] = pq;
            a0 = a0 + pq;
        }
        for (int j = 0; j < 4; ++j) {
            for (int q = pb[j]; q < pe[j]; ++q) {
                const or_sreac* r = &s->sreacs[q];
                const double k = (r->vdep >= 0) ? or_vdep_k(s, r->vdep, vm[j]) : r->k;
                const double h = or_sreac_h(r, sc[j], cnt);
                const double pq = h * or_sreac_ccst(r, k, ivs, area[j]);
                sprop[j][q - pb[j]] = pq;
                a0 = a0 + pq;
            }
            int kk = pe[j] - pb[j];
            for (int g = 0; g < s->nghk && pj[j] >= 0; ++g) {
                const or_ghk* gh = &s->ghks[g];
                if (gh->patch != pj[j]) continue;
                const double rt = or_ghk_rate(gh, vm[j], cnt[gh->ion], sc[j][gh->sspec], ivs, s->temp);
                const double pq = fabs(rt);
                sprop[j][kk] = pq;
                a0 = a0 + pq;
                ++kk;
            }
        }
        if (!(a0 > 0.0)) break;
        double dt = -or_log(u_oc(or_u32(st))) / a0;
        if (tt + dt > T) break;
        tt = tt + dt;
        double target = u_co(or_u32(st)) * a0;
        double cum = 0.0;
        int sj = -2, sq = -1, lj = -2, lq = -1;
        for (int q = rb; q >= 0 && q < re && sj == -2; ++q) {
            double pq = prop[q];
            if (pq > 0.0) {
                lj = -1;
                lq = q;
                cum = cum + pq;
                if (target < cum) {
                    sj = -1;
                    sq = q;
                }
            }
        }
        for (int j = 0; j < 4 && sj == -2; ++j) {
            for (int q = pb[j]; q < pe[j]; ++q) {
                double pq = sprop[j][q - pb[j]];
                if (pq > 0.0) {
                    lj = j;
                    lq = q;
                    cum = cum + pq;
                    if (target < cum) {
                        sj = j;
                        sq = q;
                        break;
                    }
                }
            }
            int kk = pe[j] - pb[j];
            for (int g = 0; g < s->nghk && pj[j] >= 0 && sj == -2; ++g) {
                if (s->ghks[g].patch != pj[j]) continue;
                double pq = sprop[j][kk];
                ++kk;
                if (pq > 0.0) {
                    lj = j;
                    lq = -10 - g;
                    cum = cum + pq;
                    if (target < cum) {
                        sj = j;
                        sq = -10 - g;
                    }
                }
            }
        }
        if (sj == -2) {
            sj = lj;
            sq = lq;
        }
        if (sq <= -10) {
            /* GHK event (ghkcurr.cpp:230-280): one ion out (efflux) or in, z charges. */
            const or_ghk* gh = &s->ghks[-10 - sq];
            const int m = mm[sj];
            const double rt = or_ghk_rate(gh, vm[sj], cnt[gh->ion], sc[sj][gh->sspec], ivs, s->temp);
            const int eff = rt >= 0.0;
            if (gh->realflux && !((clampm >> gh->ion) & 1u)) {
                const int k = gh->ion;
                const uint32_t old = cnt[k];
                const uint32_t nc = or_bump(old, eff ? -1 : 1);
                tdel[k] = tdel[k] + (double)((int64_t)nc - (int64_t)old) * tt;
                cnt[k] = nc;
            }
#pragma omp atomic
            s->echarge[m] += eff ? gh->valence : -gh->valence;
#pragma omp atomic
            s->surf_ext += 1;
            continue;
        }
        if (sq < 0) break;
        if (sj == -1) {
            const or_reac* rc = &s->reac[sq];
            for (int i = 0; i < s->nspec; ++i) {
                int32_t d = rc->upd[i];
                if (d == 0 || ((clampm >> i) & 1u)) continue;
                const uint32_t old = cnt[i];
                const uint32_t nc = or_bump(old, d);
                tdel[i] = tdel[i] + (double)((int64_t)nc - (int64_t)old) * tt;
                cnt[i] = nc;
            }
#pragma omp atomic
            s->ext[sq] += 1;
        } else {
            const or_sreac* r = &s->sreacs[sq];
            for (int i = 0; i < r->nsupd; ++i) {
                const int k = r->supd_spec[i];
                const uint32_t old = sc[sj][k];
                occ[sj][k] = occ[sj][k] + (double)old * (tt - last[sj][k]);
                last[sj][k] = tt;
                sc[sj][k] = or_bump(old, r->supd_delta[i]);
            }
            for (int i = 0; i < r->niupd; ++i) {
                const int k = r->iupd_spec[i];
                if ((clampm >> k) & 1u) continue;
                const uint32_t old = cnt[k];
                const uint32_t nc = or_bump(old, r->iupd_delta[i]);
                tdel[k] = tdel[k] + (double)((int64_t)nc - (int64_t)old) * tt;
                cnt[k] = nc;
            }
#pragma omp atomic
            s->surf_ext += 1;
        }
    }
    for (int j = 0; j < 4; ++j) {
        const int m = mm[j];
        if (m < 0) continue;
        for (int k = 0; k < SS; ++k) {
            const uint32_t c = sc[j][k];
            s->tri_counts[(size_t)k * M + m] = c;
            const double o = occ[j][k] + (double)c * (T - last[j][k]);
            s->spec_int[(size_t)k * M + m] += o;
            if (s->nsdiff > 0) {
                const int sd = s->sdiff_slot[k];
                if (sd >= 0) s->tri_occ[(size_t)sd * M + m] = o;
            }
        }
    }
}

/* Signed GHK ion rate with the outer tet's concentration (ghkcurr.cpp:176-181, voconc < 0). */
static double or_ghk_rate_outer(const or_ghk* g, double vm, uint32_t c_ion, uint32_t n, double ivs, uint32_t c_out,
                                double ivs_out, double temp) {
    if (n == 0) return 0.0;
    const double ci = (double)c_ion * ivs * 1.0e3;
    const double co = (double)c_out * ivs_out * 1.0e3;
    const double I = or_ghk_current(g->perm, vm * 1.0e-3 + g->vshift, g->valence, temp, ci, co);
    return I / (OR_E_CHARGE * (double)g->valence) * (double)n;
}

/* State of one merged unit during its window: local copies of the counts of its nt tets
 * (cnt[k][S]) and nm triangles (sc[j][SS]), the tets' change-time sums, the triangles'
 * occupancy integrals, element propensities and the sum tree. */
typedef struct {
    const or_solver* s;
    int nt, nm, E, P, rmax, r;
    const int32_t* tets;
    const int32_t* tris;
    int* loc;          /* [nt + nm]: local index of the inner tet of triangle j at [nt + j] */
    int* loco;         /* [nm]: local index of the coupled outer tet, -1 */
    uint32_t* cnt;
    double* tdel;
    uint32_t* sc;
    double* occ;
    double* last;
    double* prop;
    double* tree;
} or_unit;

static int or_comp_rb(const or_solver* s, int c, int* re) {
    int rb = -1;
    *re = -1;
    for (int q = 0; q < s->nreac; ++q)
        if (s->reac[q].comp == c) {
            if (rb < 0) rb = q;
            *re = q + 1;
        }
    return rb;
}

/* Propensities of element e in reaction order (a tet: its compartment's reactions; a
 * triangle: its patch's surface reactions, then its GHK currents); returns their sum. */
static double or_unit_elem(or_unit* U, int e, int* nq) {
    const or_solver* s = U->s;
    const int S = s->nspec, SS = s->nsspec;
    double* pr = U->prop + (size_t)e * U->rmax;
    double sum = 0.0;
    int k = 0;
    if (e < U->nt) {
        const int t = U->tets[e];
        int re;
        const int rb = or_comp_rb(s, s->tcomp[t], &re);
        const double* K = s->kcst + (size_t)U->r * s->nreac;
        for (int q = rb; q >= 0 && q < re; ++q, ++k) {
            pr[k] = or_prop(s, &s->reac[q], U->cnt + (size_t)e * S, K[q], s->ivs[t]);
            sum = sum + pr[k];
        }
        *nq = k;
        return sum;
    }
    const int j = e - U->nt, m = U->tris[j];
    const int p = s->tri_patch[m];
    const int ki = U->loc[U->nt + j], ko = U->loco[j];
    const int ti = s->tri_inner[m];
    const int to = s->tri_outer ? s->tri_outer[m] : -1;
    const double ivs_i = s->ivs[ti], ivs_o = to >= 0 ? s->ivs[to] : 0.0;
    const double vm = s->tri_v[m];
    for (int q = s->patch_sb[p]; q < s->patch_sb[p + 1]; ++q, ++k) {
        const or_sreac* r = &s->sreacs[q];
        const double kk = (r->vdep >= 0) ? or_vdep_k(s, r->vdep, vm) : r->k;
        double pq = 0.0;
        const int kv = r->vside ? ko : ki;
        if (kv >= 0) {
            const double h = or_sreac_h(r, U->sc + (size_t)j * SS, U->cnt + (size_t)kv * S);
            pq = h * or_sreac_ccst(r, kk, r->vside ? ivs_o : ivs_i, s->tri_area[m]);
        }
        pr[k] = pq;
        sum = sum + pq;
    }
    for (int g = 0; g < s->nghk; ++g) {
        const or_ghk* gh = &s->ghks[g];
        if (gh->patch != p) continue;
        const uint32_t n = U->sc[(size_t)j * SS + gh->sspec];
        const uint32_t ci = U->cnt[(size_t)ki * S + gh->ion];
        const double rt = (gh->voconc >= 0.0 || ko < 0)
                              ? or_ghk_rate(gh, vm, ci, n, ivs_i, s->temp)
                              : or_ghk_rate_outer(gh, vm, ci, n, ivs_i, U->cnt[(size_t)ko * S + gh->ion], ivs_o, s->temp);
        pr[k] = fabs(rt);
        sum = sum + pr[k];
        ++k;
    }
    *nq = k;
    return sum;
}

static int or_unit_nq(const or_unit* U, int e) {
    const or_solver* s = U->s;
    if (e < U->nt) {
        int re;
        const int rb = or_comp_rb(s, s->tcomp[U->tets[e]], &re);
        return rb < 0 ? 0 : re - rb;
    }
    const int p = s->tri_patch[U->tris[e - U->nt]];
    int n = s->patch_sb[p + 1] - s->patch_sb[p];
    for (int g = 0; g < s->nghk; ++g) n += s->ghks[g].patch == p;
    return n;
}

static void or_unit_refresh(or_unit* U, int f) {
    int nq;
    int i = U->P + f;
    U->tree[i] = or_unit_elem(U, f, &nq);
    for (i >>= 1; i >= 1; i >>= 1) U->tree[i] = U->tree[2 * i] + U->tree[2 * i + 1];
}

/* A tet's counts changed: the tet and every triangle of the unit whose rates read it
 * (inner tet, or outer tet of a coupled triangle), triangles in ascending order. */
static void or_unit_refresh_tet(or_unit* U, int k) {
    if (k < 0) return;
    or_unit_refresh(U, k);
    for (int j = 0; j < U->nm; ++j)
        if (U->loc[U->nt + j] == k || U->loco[j] == k) or_unit_refresh(U, U->nt + j);
}

static void or_unit_bump(or_unit* U, int k, int sp, int d, double tt) {
    const or_solver* s = U->s;
    const int t = U->tets[k];
    if ((s->clamp[t] >> sp) & 1u) return;
    uint32_t* c = U->cnt + (size_t)k * s->nspec + sp;
    const uint32_t old = *c, nc = or_bump(old, d);
    U->tdel[(size_t)k * s->nspec + sp] += (double)((int64_t)nc - (int64_t)old) * tt;
    *c = nc;
}

/* SSA of merged unit u over [0, T) (window w of realization r): the direct method over all
 * its elements' reactions, the element chosen by descending the sum tree (left while the
 * target is below the left sum or the right sum is zero, else subtract the left sum and go
 * right), the reaction by the cumulative sum inside the element; draws from the window
 * stream of the unit's first tet. */
static void or_unit_ssa(or_solver* s, int r, int u, double T, uint64_t w) {
    const int S = s->nspec, SS = s->nsspec, M = s->ntris;
    or_unit U;
    memset(&U, 0, sizeof(U));
    U.s = s;
    U.r = r;
    U.tets = s->u_tets + s->u_tb[u];
    U.nt = s->u_tb[u + 1] - s->u_tb[u];
    U.tris = s->u_tris + s->u_mb[u];
    U.nm = s->u_mb[u + 1] - s->u_mb[u];
    U.E = U.nt + U.nm;
    U.P = 1;
    while (U.P < U.E) U.P <<= 1;
    U.rmax = 1;
    for (int c = 0; c < s->ncomp; ++c) {
        int re;
        const int rb = or_comp_rb(s, c, &re);
        if (rb >= 0 && re - rb > U.rmax) U.rmax = re - rb;
    }
    for (int p = 0; p < s->npatch; ++p) {
        int n = s->patch_sb[p + 1] - s->patch_sb[p];
        for (int g = 0; g < s->nghk; ++g) n += s->ghks[g].patch == p;
        if (n > U.rmax) U.rmax = n;
    }
    U.loc = (int*)malloc(sizeof(int) * (size_t)U.E);
    U.loco = (int*)malloc(sizeof(int) * (size_t)(U.nm + 1));
    for (int k = 0; k < U.nt; ++k) U.loc[k] = k;
    for (int j = 0; j < U.nm; ++j) {
        const int m = U.tris[j];
        U.loc[U.nt + j] = -1;
        U.loco[j] = -1;
        for (int k = 0; k < U.nt; ++k) {
            if (U.tets[k] == s->tri_inner[m]) U.loc[U.nt + j] = k;
            if (or_patch_coupled(s, s->tri_patch[m]) && s->tri_outer && U.tets[k] == s->tri_outer[m]) U.loco[j] = k;
        }
    }
    U.cnt = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)U.nt * S);
    U.tdel = (double*)calloc((size_t)U.nt * S, sizeof(double));
    U.sc = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)(U.nm * SS + 1));
    U.occ = (double*)calloc((size_t)(U.nm * SS + 1), sizeof(double));
    U.last = (double*)calloc((size_t)(U.nm * SS + 1), sizeof(double));
    U.prop = (double*)calloc((size_t)U.E * U.rmax, sizeof(double));
    U.tree = (double*)calloc((size_t)2 * U.P, sizeof(double));
    for (int k = 0; k < U.nt; ++k)
        for (int i = 0; i < S; ++i) U.cnt[(size_t)k * S + i] = s->counts[(size_t)i * s->ntets + U.tets[k]];
    for (int j = 0; j < U.nm; ++j)
        for (int i = 0; i < SS; ++i) U.sc[(size_t)j * SS + i] = s->tri_counts[(size_t)i * M + U.tris[j]];
    for (int e = 0; e < U.E; ++e) {
        int nq;
        U.tree[U.P + e] = or_unit_elem(&U, e, &nq);
    }
    for (int i = U.P - 1; i >= 1; --i) U.tree[i] = U.tree[2 * i] + U.tree[2 * i + 1];
    or_stream st;
    or_stream_init(&st, s->seed, (uint32_t)r, (uint32_t)(U.tets[0] - s->real_begin[r]), w, 0u);
    double tt = 0.0;
    for (;;) {
        const double a0 = U.tree[1];
        if (!(a0 > 0.0)) break;
        const double dt = -or_log(u_oc(or_u32(&st))) / a0;
        if (tt + dt > T) break;
        tt = tt + dt;
        double target = u_co(or_u32(&st)) * a0;
        int node = 1;
        while (node < U.P) {
            const double l = U.tree[2 * node], rr = U.tree[2 * node + 1];
            if (target < l || !(rr > 0.0))
                node = 2 * node;
            else {
                target = target - l;
                node = 2 * node + 1;
            }
        }
        const int e = node - U.P;
        const int nq = or_unit_nq(&U, e);
        const double* pq = U.prop + (size_t)e * U.rmax;
        double cum = 0.0;
        int sel = -1, lastnz = -1;
        for (int q = 0; q < nq; ++q)
            if (pq[q] > 0.0) {
                lastnz = q;
                cum = cum + pq[q];
                if (target < cum) {
                    sel = q;
                    break;
                }
            }
        if (sel < 0) sel = lastnz;
        if (sel < 0) break;
        if (e < U.nt) {
            int re;
            const int q = or_comp_rb(s, s->tcomp[U.tets[e]], &re) + sel;
            for (int i = 0; i < S; ++i)
                if (s->reac[q].upd[i]) or_unit_bump(&U, e, i, s->reac[q].upd[i], tt);
#pragma omp atomic
            s->ext[q] += 1;
            or_unit_refresh_tet(&U, e);
            continue;
        }
        const int j = e - U.nt, m = U.tris[j], p = s->tri_patch[m];
        const int pb = s->patch_sb[p], npr = s->patch_sb[p + 1] - pb;
        const int ki = U.loc[U.nt + j], ko = U.loco[j];
        int chi = 0, cho = 0;
        if (sel < npr) {
            const or_sreac* rs = &s->sreacs[pb + sel];
            for (int i = 0; i < rs->nsupd; ++i) {
                const size_t o = (size_t)j * SS + rs->supd_spec[i];
                const uint32_t old = U.sc[o];
                U.occ[o] = U.occ[o] + (double)old * (tt - U.last[o]);
                U.last[o] = tt;
                U.sc[o] = or_bump(old, rs->supd_delta[i]);
            }
            for (int i = 0; i < rs->niupd; ++i) or_unit_bump(&U, ki, rs->iupd_spec[i], rs->iupd_delta[i], tt);
            for (int i = 0; i < rs->noupd && ko >= 0; ++i) or_unit_bump(&U, ko, rs->oupd_spec[i], rs->oupd_delta[i], tt);
            chi = rs->niupd > 0;
            cho = rs->noupd > 0;
        } else {
            int g = 0, left = sel - npr;
            for (; g < s->nghk; ++g)
                if (s->ghks[g].patch == p && left-- == 0) break;
            const or_ghk* gh = &s->ghks[g];
            const int outer = gh->voconc < 0.0 && ko >= 0;
            const uint32_t n = U.sc[(size_t)j * SS + gh->sspec];
            const uint32_t ci = U.cnt[(size_t)ki * S + gh->ion];
            const double sr = outer ? or_ghk_rate_outer(gh, s->tri_v[m], ci, n, s->ivs[s->tri_inner[m]],
                                                        U.cnt[(size_t)ko * S + gh->ion], s->ivs[s->tri_outer[m]], s->temp)
                                    : or_ghk_rate(gh, s->tri_v[m], ci, n, s->ivs[s->tri_inner[m]], s->temp);
            const int eff = sr >= 0.0;
            if (gh->realflux) {
                or_unit_bump(&U, ki, gh->ion, eff ? -1 : 1, tt);
                if (outer) or_unit_bump(&U, ko, gh->ion, eff ? 1 : -1, tt);
                chi = 1;
                cho = outer;
            }
#pragma omp atomic
            s->echarge[m] += eff ? gh->valence : -gh->valence;
        }
#pragma omp atomic
        s->surf_ext += 1;
        or_unit_refresh(&U, e);
        if (chi) or_unit_refresh_tet(&U, ki);
        if (cho) or_unit_refresh_tet(&U, ko);
    }
    for (int j = 0; j < U.nm; ++j) {
        const int m = U.tris[j];
        for (int i = 0; i < SS; ++i) {
            const uint32_t c = U.sc[(size_t)j * SS + i];
            s->tri_counts[(size_t)i * M + m] = c;
            const double o = U.occ[(size_t)j * SS + i] + (double)c * (T - U.last[(size_t)j * SS + i]);
            s->spec_int[(size_t)i * M + m] += o;
            if (s->nsdiff > 0) {
                const int sd = s->sdiff_slot[i];
                if (sd >= 0) s->tri_occ[(size_t)sd * M + m] = o;
            }
        }
    }
    for (int k = 0; k < U.nt; ++k)
        for (int i = 0; i < S; ++i) {
            s->counts[(size_t)i * s->ntets + U.tets[k]] = U.cnt[(size_t)k * S + i];
            s->utdel[(size_t)U.tets[k] * S + i] = U.tdel[(size_t)k * S + i];
        }
    free(U.loc);
    free(U.loco);
    free(U.cnt);
    free(U.tdel);
    free(U.sc);
    free(U.occ);
    free(U.last);
    free(U.prop);
    free(U.tree);
}

/* Surface diffusion leave of triangle m (TOS:1716-1793, sdiff.cpp:498-560): n = min(pop,
 * window integral / T) with a Bernoulli on its fraction, Binomial(n, min(1, T D G)) leaving,
 * split over the three edges by the conditional selectors (purpose 80 + species stream). */
static void or_tri_leave(or_solver* s, int r, int m, double T, uint64_t w) {
    const int M = s->ntris, SS = s->nsspec;
    for (int sd = 0; sd < s->nsdiff; ++sd) {
        const int sp = s->sdspec[sd];
        uint32_t* o = s->tri_out + ((size_t)sd * M + m) * 4;
        o[0] = o[1] = o[2] = o[3] = 0;
        const double D = s->sdcst[(size_t)s->tri_patch[m] * SS + sp];
        if (!(D > 0.0)) continue;
        const size_t ci = (size_t)sp * M + m;
        const uint32_t pop = s->tri_counts[ci];
        if (pop == 0) continue;
        const float* g = s->sgeo + (size_t)m * 4;
        double t1 = T * (D * (double)g[3]);
        if (t1 >= 1.0) t1 = 1.0;
        double nd = s->tri_occ[(size_t)sd * M + m] / T;
        if (nd > (double)pop) nd = (double)pop;
        const double nint = floor(nd), frc = nd - nint;
        uint32_t mean_n = (uint32_t)nint;
        or_stream st;
        or_stream_init(&st, s->seed, (uint32_t)r, (uint32_t)m, w, 80u + (uint32_t)sp);
        if (frc > 0.0 && u_co(or_u32(&st)) < frc) mean_n += 1u;
        uint32_t Kn = 0;
        if (mean_n <= OR_PM_MAX) {
            if (mean_n > 0 && t1 > 0.0) {
                const double c3[3] = {(double)g[0], (double)g[1], 1.0};
                uint32_t k4[4];
                Kn = or_leave_molecules(&st, mean_n, t1, c3, k4);
                o[0] = k4[0];
                o[1] = k4[1];
                o[2] = k4[2];
            }
        } else {
            Kn = or_binom(&st, mean_n, t1);
            uint32_t rem = Kn;
            o[0] = or_binom(&st, rem, (double)g[0]);
            rem -= o[0];
            o[1] = or_binom(&st, rem, (double)g[1]);
            rem -= o[1];
            o[2] = rem;
        }
        if (Kn > 0) {
            s->tri_counts[ci] = pop - Kn;
#pragma omp atomic
            s->diff_moved += Kn;
        }
    }
}

/* Surface arrivals: each edge slot holds what the neighbour across it sent. */
static void or_tri_enter(or_solver* s, int m) {
    const int M = s->ntris, SS = s->nsspec;
    for (int sd = 0; sd < s->nsdiff; ++sd) {
        const int sp = s->sdspec[sd];
        if (!(s->sdcst[(size_t)s->tri_patch[m] * SS + sp] > 0.0)) continue;
        uint64_t sum = s->tri_counts[(size_t)sp * M + m];
        for (int e = 0; e < 3; ++e) {
            const int nb = s->snbr[(size_t)m * 4 + e];
            if (nb < 0) continue;
            sum += s->tri_out[((size_t)sd * M + (nb >> 2)) * 4 + (nb & 3)];
        }
        s->tri_counts[(size_t)sp * M + m] = (uint32_t)(sum > 0xFFFFFFFFull ? 0xFFFFFFFFull : sum);
    }
}

/* SSA phase (TOS:1565-1588) then diffusion phase (TOS:1633-1712) of tet t. */
static void or_tet_window(or_solver* s, int r, int t, double T, uint64_t w) {
    const int S = s->nspec;
    const int c = s->tcomp[t];
    uint32_t cnt[OR_MAXS];
    /* Occupancy (tet.cpp:318-340 keeps the running integral and the last update time):
     * the integral of a count over [0, T) is c_end T - sum_k (change_k) t_k, so tdel keeps
     * sum_k (change_k) t_k. */
    double tdel[OR_MAXS];
    /* A tet of a merged unit: its SSA ran in or_unit_ssa, which left the counts and the
     * change-time sums. */
    const int merged = s->nunits > 0 && s->tet_unit[t] >= 0;
    for (int i = 0; i < S; ++i) {
        cnt[i] = s->counts[(size_t)i * s->ntets + t];
        tdel[i] = merged ? s->utdel[(size_t)t * S + i] : 0.0;
    }
    const uint32_t clampm = s->clamp[t];
    or_stream st;
    or_stream_init(&st, s->seed, (uint32_t)r, (uint32_t)(t - s->real_begin[r]), w, 0u);
    const double ivs = s->ivs[t];
    const double* K = s->kcst + (size_t)r * s->nreac;

    int rb = -1, re = -1;
    for (int q = 0; q < s->nreac; ++q) {
        if (s->reac[q].comp == c) {
            if (rb < 0) rb = q;
            re = q + 1;
        }
    }
    const int has_tris = s->ntris > 0 && (s->tet_tris[(size_t)t * 4] >= 0);
    if (merged) {
    } else if (has_tris) {
        or_ssa_surf(s, t, T, cnt, tdel, &st, clampm, ivs, K, rb, re);
    } else if (rb >= 0) {
        double tt = 0.0;
        for (;;) {
            double a0 = 0.0;
            for (int q = rb; q < re; ++q) a0 = a0 + or_prop(s, &s->reac[q], cnt, K[q], ivs);
            if (!(a0 > 0.0)) break;
            double dt = -or_log(u_oc(or_u32(&st))) / a0;
            if (tt + dt > T) break;
            tt = tt + dt;
            double target = u_co(or_u32(&st)) * a0;
            double cum = 0.0;
            int sel = -1, lastnz = -1;
            for (int q = rb; q < re; ++q) {
                double p = or_prop(s, &s->reac[q], cnt, K[q], ivs);
                if (p > 0.0) {
                    lastnz = q;
                    cum = cum + p;
                    if (target < cum) {
                        sel = q;
                        break;
                    }
                }
            }
            if (sel < 0) sel = lastnz;
            if (sel < 0) break;
            /* Reac::apply (reac.cpp:235-251) with Tet::setCount occupancy (tet.cpp:318-340). */
            for (int i = 0; i < S; ++i) {
                int32_t d = s->reac[sel].upd[i];
                if (d == 0 || ((clampm >> i) & 1u)) continue;
                tdel[i] = tdel[i] + (double)d * tt;
                cnt[i] = (uint32_t)((int64_t)cnt[i] + d);
            }
#pragma omp atomic
            s->ext[sel] += 1;
        }
    }

    const float* g = s->geo + (size_t)t * 4;
    const double G = (double)g[3];
    const double* Dc = s->dcst + ((size_t)r * s->ncomp + c) * S;
    uint64_t moved = 0;
    for (int i = 0; i < S; ++i) {
        if (!s->has_rule[i]) continue;
        double D = Dc[i];
        if (!(D > 0.0)) continue;
        uint32_t* o = s->outflow + ((size_t)i * s->ntets + t) * 4;
        o[0] = o[1] = o[2] = o[3] = 0;
        uint32_t pop = cnt[i];
        if (pop == 0) continue;
        /* Each (tet, species) leaves on its own stream (purpose 16 + species). */
        or_stream_init(&st, s->seed, (uint32_t)r, (uint32_t)(t - s->real_begin[r]), w, 16u + (uint32_t)i);
        double t1 = T * (D * G);
        float gs[3] = {g[0], g[1], g[2]};
        if (or_has_bnd(s, t)) t1 = T * or_bnd_split(s, t, i, D, gs);
        const double cs[3] = {(double)gs[0], (double)gs[1], (double)gs[2]};
        if (t1 >= 1.0) t1 = 1.0;
        uint32_t mean_n = pop;
        if (tdel[i] != 0.0) {
            double nbar = (double)pop - tdel[i] * (1.0 / T);
            if (nbar > (double)pop) nbar = (double)pop;
            double nint = floor(nbar);
            double frc = nbar - nint;
            mean_n = (uint32_t)nint;
            if (frc > 0.0 && u_co(or_u32(&st)) < frc) mean_n += 1;
        }
        uint32_t Kn, kk[4] = {0, 0, 0, 0};
        if (mean_n <= OR_PM_MAX) {
            if (mean_n == 0 || !(t1 > 0.0)) continue;
            Kn = or_leave_molecules(&st, mean_n, t1, cs, kk);
            if (Kn == 0) continue;
        } else {
            Kn = or_binom(&st, mean_n, t1);
            if (Kn == 0) continue;
            uint32_t rem = Kn;
            for (int f = 0; f < 3; ++f) {
                kk[f] = or_binom(&st, rem, cs[f]);
                rem -= kk[f];
            }
            kk[3] = rem;
        }
        for (int f = 0; f < 4; ++f) o[f] = kk[f];
        if (!((clampm >> i) & 1u)) cnt[i] = pop - Kn;
        moved += Kn;
    }
    for (int i = 0; i < S; ++i) s->counts[(size_t)i * s->ntets + t] = cnt[i];
#pragma omp atomic
    s->diff_moved += moved;
}

/* Arrivals: Tet::incCount on the receiving tet (tet.cpp:342-370), skipped when clamped. */
static void or_tet_enter(or_solver* s, int r, int t) {
    const int c = s->tcomp[t];
    const double* Dc = s->dcst + ((size_t)r * s->ncomp + c) * s->nspec;
    for (int i = 0; i < s->nspec; ++i) {
        if (!s->has_rule[i] || !(Dc[i] > 0.0) || ((s->clamp[t] >> i) & 1u)) continue;
        uint64_t sum = s->counts[(size_t)i * s->ntets + t];
        for (int f = 0; f < 4; ++f) {
            int n = s->nbr[(size_t)t * 4 + f];
            if (n < 0) continue;
            sum += s->outflow[((size_t)i * s->ntets + n) * 4 + s->rface[(size_t)t * 4 + f]];
        }
        /* Boundary faces: what the tet behind sent, when it diffuses species i. */
        for (int f = 0; s->nbnd && f < 4; ++f) {
            const int nb = s->bnbr[(size_t)t * 4 + f];
            if (nb < 0) continue;
            const int n = nb / 4, cn = s->tcomp[n];
            if (cn >= 0 && s->has_rule[i] && s->dcst[((size_t)r * s->ncomp + cn) * s->nspec + i] > 0.0)
                sum += s->outflow[((size_t)i * s->ntets + n) * 4 + nb % 4];
        }
        s->counts[(size_t)i * s->ntets + t] = (uint32_t)sum;
    }
}

/* run(endtime) for every realization (TOS:1507-1527, window recurrence TOS:1550-1558 and
 * the time update at the end of each window TOS:1818-1823). Returns windows run. */
uint64_t or_run(or_solver* s, double endtime) {
    uint64_t total = 0;
    for (int r = 0; r < s->nreal; ++r) {
        int tb = s->real_begin[r], te = s->real_begin[r + 1];
        /* TOS:1513: a run to (almost) the current time only sets the time
         * (util::almost_equal, src/steps/util/collections.hpp:144-148). */
        double d = fabs(s->t[r] - endtime);
        if (d <= 2.220446049250313e-16 * fabs(s->t[r] + endtime) * 4 || d < 2.2250738585072014e-308) {
            s->t[r] = endtime;
            continue;
        }
        while (s->t[r] < endtime) {
            double t = s->t[r], per = s->period[r];
            double T = (t + per > endtime) ? endtime - t : per;
            uint64_t w = s->window[r];
#pragma omp parallel for schedule(dynamic, 1)
            for (int u = 0; u < s->nunits; ++u)
                if (s->u_tets[s->u_tb[u]] >= tb && s->u_tets[s->u_tb[u]] < te) or_unit_ssa(s, r, u, T, w);
#pragma omp parallel for schedule(dynamic, 256)
            for (int tet = tb; tet < te; ++tet)
                if (s->tcomp[tet] >= 0) or_tet_window(s, r, tet, T, w);
#pragma omp parallel for schedule(static)
            for (int m = 0; m < s->ntris * (s->nsdiff > 0); ++m)
                if (s->tri_inner[m] >= tb && s->tri_inner[m] < te) or_tri_leave(s, r, m, T, w);
#pragma omp parallel for schedule(static)
            for (int tet = tb; tet < te; ++tet)
                if (s->tcomp[tet] >= 0) or_tet_enter(s, r, tet);
#pragma omp parallel for schedule(static)
            for (int m = 0; m < s->ntris * (s->nsdiff > 0); ++m)
                if (s->tri_inner[m] >= tb && s->tri_inner[m] < te) or_tri_enter(s, m);
            s->t[r] = (t + per > endtime) ? endtime : t + per;
            s->window[r] = w + 1;
            total += 1;
        }
    }
    return total;
}

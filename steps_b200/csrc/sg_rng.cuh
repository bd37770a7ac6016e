// Counter-based random streams and exact discrete samplers for the
// operator-split SSA step.
//
// Everything here is __host__ __device__ and uses only IEEE-754 operations
// that are correctly rounded on both the GPU and an x86 host (+, -, *, /,
// sqrt, explicit fma, floor).  With FMA contraction disabled on both sides
// (-fmad=false for nvcc device code, -ffp-contract=off for gcc) the same
// counters produce bit-identical samples on CPU and GPU.
//
// Reference behaviour replaced:
//   * src/steps/rng/r123.cpp:43-82      Philox4x32-8 buffered serial stream (key 0,
//                                        seed in the counter) -> one independent
//                                        counter stream per (unit, window).
//   * src/steps/rng/rng.hpp:87-105      getUnfII / getUnfIE / getUnfEE.
//   * src/steps/rng/rng.cpp:512-514     getExp (Ahrens-Dieter in float) -> -log(U)/a0
//                                        with the project log below.
//   * src/steps/rng/rng.cpp:516-527     getBinom (small_binomial / libstdc++) ->
//                                        BINV inversion, inversion from the mode,
//                                        BTRD rejection for very large n p.
#pragma once
#include <stdint.h>
#include <math.h>

#if defined(__CUDACC__)
#define SG_HD __host__ __device__ __forceinline__
#define SG_HD_NOINLINE static __host__ __device__ __noinline__
#else
#define SG_HD static inline
#define SG_HD_NOINLINE static
#endif

// ---------------------------------------------------------------------------
// Philox4x32 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy as 1, 2, 3",
// SC'11), 8 rounds as the reference's generator.  Multipliers and Weyl constants are the
// published ones.
// ---------------------------------------------------------------------------
#define SG_PHILOX_M0 0xD2511F53u
#define SG_PHILOX_M1 0xCD9E8D57u
#define SG_PHILOX_W0 0x9E3779B9u
#define SG_PHILOX_W1 0xBB67AE85u
#define SG_PHILOX_ROUNDS 8  // the reference's R123 generator (src/steps/rng/r123.hpp:76, Philox4x32_R<8>)

struct sg_u32x4 {
    uint32_t x, y, z, w;
};

SG_HD void sg_mulhilo32(uint32_t a, uint32_t b, uint32_t* hi, uint32_t* lo) {
#if defined(__CUDA_ARCH__)
    *hi = __umulhi(a, b);
    *lo = a * b;
#else
    uint64_t p = (uint64_t)a * (uint64_t)b;
    *hi = (uint32_t)(p >> 32);
    *lo = (uint32_t)p;
#endif
}

SG_HD sg_u32x4 sg_philox4x32(sg_u32x4 c, uint32_t k0, uint32_t k1) {
#if defined(__CUDA_ARCH__)
#pragma unroll
#endif
    for (int r = 0; r < SG_PHILOX_ROUNDS; ++r) {
        uint32_t hi0, lo0, hi1, lo1;
        sg_mulhilo32(SG_PHILOX_M0, c.x, &hi0, &lo0);
        sg_mulhilo32(SG_PHILOX_M1, c.z, &hi1, &lo1);
        sg_u32x4 n;
        n.x = hi1 ^ c.y ^ k0;
        n.y = lo1;
        n.z = hi0 ^ c.w ^ k1;
        n.w = lo0;
        c = n;
        k0 += SG_PHILOX_W0;
        k1 += SG_PHILOX_W1;
    }
    return c;
}

// Stream purposes (top byte of counter word w).
#define SG_PURPOSE_WINDOW 0u   // reaction SSA of one unit in one split window
#define SG_PURPOSE_SETUP 1u    // host-side placement of molecules (setters)
#define SG_PURPOSE_EFIELD 2u   // reserved
#define SG_PURPOSE_DIFF 16u    // + species: diffusion leave of one (unit, species) in one window
#define SG_PURPOSE_SDIFF 80u   // + surface species: surface diffusion leave of one (triangle, species)

// One independent stream: counter = (block, unit, window_lo, purpose<<24 | window_hi24),
// key = (seed_lo, seed_hi + realization * W0).  Draw j of the stream is word
// (j mod 4) of Philox(block = j / 4).  Values are consumed through a 4-word
// shift register so that the state stays in registers on the GPU.
struct sg_stream {
    uint32_t k0, k1;
    uint32_t unit, wlo, whi;
    uint32_t block;
    uint32_t b0, b1, b2, b3;
    uint32_t left;
};

SG_HD void sg_stream_init(sg_stream* s, uint64_t seed, uint32_t realization, uint32_t unit,
                          uint64_t window, uint32_t purpose) {
    s->k0 = (uint32_t)seed;
    s->k1 = (uint32_t)(seed >> 32) + realization * SG_PHILOX_W0;
    s->unit = unit;
    s->wlo = (uint32_t)window;
    s->whi = (purpose << 24) | ((uint32_t)(window >> 32) & 0xFFFFFFu);
    s->block = 0;
    s->left = 0;
    s->b0 = s->b1 = s->b2 = s->b3 = 0;
}

// One Philox block of a stream.  With SG_NOINLINE_REFILL the rounds exist once in the
// device code instead of at every draw site (smaller instruction footprint); arguments
// and result pass by value so the caller's stream state stays in registers.
#if defined(__CUDACC__) && defined(SG_NOINLINE_REFILL)
static __host__ __device__ __noinline__
#else
SG_HD
#endif
sg_u32x4 sg_philox_block(uint32_t block, uint32_t unit, uint32_t wlo, uint32_t whi, uint32_t k0,
                         uint32_t k1) {
    sg_u32x4 c;
    c.x = block;
    c.y = unit;
    c.z = wlo;
    c.w = whi;
    return sg_philox4x32(c, k0, k1);
}

SG_HD void sg_stream_refill(sg_stream* s) {
    sg_u32x4 r = sg_philox_block(s->block, s->unit, s->wlo, s->whi, s->k0, s->k1);
    s->block += 1;
    s->b0 = r.x;
    s->b1 = r.y;
    s->b2 = r.z;
    s->b3 = r.w;
    s->left = 4;
}

SG_HD uint32_t sg_next_u32(sg_stream* s) {
    if (s->left == 0) sg_stream_refill(s);
    uint32_t v = s->b0;
    s->b0 = s->b1;
    s->b1 = s->b2;
    s->b2 = s->b3;
    s->left -= 1;
    return v;
}

#define SG_TWO_M32 2.3283064365386963e-10  // 2^-32, exact

// [0,1): x * 2^-32   (reference getUnfIE, rng.hpp:93-96)
SG_HD double sg_u01_co(uint32_t x) { return (double)x * SG_TWO_M32; }
// (0,1]: (x + 1) * 2^-32   (argument of the waiting-time log, never 0)
SG_HD double sg_u01_oc(uint32_t x) { return ((double)x + 1.0) * SG_TWO_M32; }
// (0,1): (x + 0.5) * 2^-32 (reference getUnfEE, rng.hpp:99-102)
SG_HD double sg_u01_oo(uint32_t x) { return ((double)x + 0.5) * SG_TWO_M32; }

// ---------------------------------------------------------------------------
// Natural logarithm written from the mathematics (no libm call, so host and
// device agree bit for bit).  x = m * 2^e with m in [sqrt(1/2), sqrt(2));
// log m = 2 atanh(s), s = (m - 1)/(m + 1), |s| <= 0.1716, expanded as the
// Taylor series 2 s (1 + z/3 + z^2/5 + ... + z^11/23), z = s^2 (truncation
// error below 1e-19 relative).  ln 2 is split into a 32-bit head and a tail
// so that e * ln2_head is exact.
// ---------------------------------------------------------------------------
#define SG_LN2_HEAD 0.6931471803691238
#define SG_LN2_TAIL 1.9082149292705877e-10
#define SG_SQRT2 1.4142135623730951

SG_HD uint64_t sg_f64_bits(double x) {
#if defined(__CUDA_ARCH__)
    return (uint64_t)__double_as_longlong(x);
#else
    union {
        double d;
        uint64_t u;
    } c;
    c.d = x;
    return c.u;
#endif
}

SG_HD double sg_bits_f64(uint64_t b) {
#if defined(__CUDA_ARCH__)
    return __longlong_as_double((long long)b);
#else
    union {
        double d;
        uint64_t u;
    } c;
    c.u = b;
    return c.d;
#endif
}

// Valid for finite x > 0 (callers never pass 0, negatives or non-finite values).
SG_HD double sg_log(double x) {
    uint64_t b = sg_f64_bits(x);
    int e = (int)((b >> 52) & 0x7FF);
    if (e == 0) {  // subnormal: scale by 2^54
        x = x * 18014398509481984.0;
        b = sg_f64_bits(x);
        e = (int)((b >> 52) & 0x7FF) - 54;
    }
    e -= 1023;
    double m = sg_bits_f64((b & 0x000FFFFFFFFFFFFFull) | 0x3FF0000000000000ull);
    if (m > SG_SQRT2) {
        m = m * 0.5;
        e += 1;
    }
    double s = (m - 1.0) / (m + 1.0);
    double z = s * s;
    double p = 1.0 / 23.0;
    p = fma(p, z, 1.0 / 21.0);
    p = fma(p, z, 1.0 / 19.0);
    p = fma(p, z, 1.0 / 17.0);
    p = fma(p, z, 1.0 / 15.0);
    p = fma(p, z, 1.0 / 13.0);
    p = fma(p, z, 1.0 / 11.0);
    p = fma(p, z, 1.0 / 9.0);
    p = fma(p, z, 1.0 / 7.0);
    p = fma(p, z, 1.0 / 5.0);
    p = fma(p, z, 1.0 / 3.0);
    double t = 2.0 * s;
    double lm = fma(t * z, p, t);
    double de = (double)e;
    return fma(de, SG_LN2_HEAD, fma(de, SG_LN2_TAIL, lm));
}

// e^x written from the mathematics: x = k ln2 + r with k = round(x / ln2) and
// |r| <= ln2 / 2 (ln2 split into the head and tail above, so k ln2_head is exact), e^r by
// its Taylor series to r^14 (truncation below 3e-19 relative), then 2^k by the exponent
// bits.  Overflow gives +inf, underflow below 2^-1022 gives 0 (no subnormal results).
SG_HD double sg_exp(double x) {
    if (!(x < 709.78)) return x != x ? x : sg_bits_f64(0x7FF0000000000000ull);
    if (x < -708.39) return 0.0;
    const double k = floor(x * 1.4426950408889634 + 0.5);
    double r = fma(-k, SG_LN2_HEAD, x);
    r = fma(-k, SG_LN2_TAIL, r);
    double p = 1.0 / 87178291200.0;             // 1/14!
    p = fma(p, r, 1.0 / 6227020800.0);          // 1/13!
    p = fma(p, r, 1.0 / 479001600.0);
    p = fma(p, r, 1.0 / 39916800.0);
    p = fma(p, r, 1.0 / 3628800.0);
    p = fma(p, r, 1.0 / 362880.0);
    p = fma(p, r, 1.0 / 40320.0);
    p = fma(p, r, 1.0 / 5040.0);
    p = fma(p, r, 1.0 / 720.0);
    p = fma(p, r, 1.0 / 120.0);
    p = fma(p, r, 1.0 / 24.0);
    p = fma(p, r, 1.0 / 6.0);
    p = fma(p, r, 0.5);
    p = fma(p, r, 1.0);
    p = fma(p, r, 1.0);
    int ki = (int)k;
    if (ki > 1023) {  // e^r > 1 for x near the top of the range: scale in two steps
        p = p * 2.0;
        ki -= 1;
    }
    if (ki < -1022) {
        p = p * 0.5;
        ki += 1;
    }
    return p * sg_bits_f64((uint64_t)(ki + 1023) << 52);
}

// q^n by binary powering (multiplications only).
SG_HD double sg_pow_u(double q, uint32_t n) {
    double r = 1.0;
    double b = q;
    while (n) {
        if (n & 1u) r = r * b;
        b = b * b;
        n >>= 1;
    }
    return r;
}

// ---------------------------------------------------------------------------
// Binomial(n, p) sampling.
//   n * min(p, 1-p) < SG_BINV_CUT : BINV sequential-search inversion
//       (Kachitvichyanukul & Schmeiser, "Binomial random variate generation",
//        CACM 31(2), 1988), one uniform per sample.
//   n * min(p, 1-p) < SG_MODE_CUT : inversion by a search that starts at the mode and
//       alternates up and down (sequential-search inversion over the support taken in
//       order of distance from the mode; Devroye, "Non-Uniform Random Variate
//       Generation", 1986, sections III.2 and X.4), one uniform per sample, about
//       1 + 1.6 sqrt(n p q) pmf steps instead of n p.
//   otherwise                     : BTRD transformed rejection with decomposition
//       (Hormann, "The generation of binomial random variates", J. Statist.
//        Comput. Simul. 46, 1993).
// ---------------------------------------------------------------------------
#define SG_BINV_CUT 24.0
#define SG_MODE_CUT 1000.0
#define SG_BTRD_MAX_ITERS 256
#define SG_RCP_TABLE 128   // 1/x for x < SG_RCP_TABLE, precomputed (same value as 1.0/x)
#define SG_MODE_TABLE 1024 // 1/x and ln x! for x < SG_MODE_TABLE (mode search), same values
#define SG_HALF_LN_2PI 0.91893853320467274

// 1/x, read from a table of correctly rounded reciprocals when one is given.
SG_HD double sg_rcp(const double* tab, uint32_t x) {
    return (tab && x < SG_RCP_TABLE) ? tab[x] : 1.0 / (double)x;
}

// Sequential search from 0: pmf recurrence f(x) = f(x-1) * ((n+1) s / x - s), s = p/q,
// the factor as one fma with 1/x from the reciprocal table.  The search runs on without
// an x < n test: past x = n the factor is rounding-small, and negative from x = n + 2, so
// the loop ends by x = n + 2 at the latest and the result is clamped to n (the value the
// bounded search returns).  With n + 3 < SG_RCP_TABLE the next reciprocal is loaded one
// step ahead, off the multiply chain.
SG_HD uint32_t sg_binv(sg_stream* st, uint32_t n, double p, const double* rcp, double s) {
    double q = 1.0 - p;
    double a = ((double)n + 1.0) * s;
    double r = sg_pow_u(q, n);
    double u = sg_u01_co(sg_next_u32(st));
    uint32_t x = 0;
    if (rcp && n + 3u < (uint32_t)SG_RCP_TABLE) {
        double rc = rcp[1];
        while (u >= r) {
            u = u - r;
            x += 1;
            double m = fma(a, rc, -s);
            rc = rcp[x + 1];
            r = r * m;
            if (!(r > 0.0)) break;  // pmf underflowed past the mass (or x > n)
        }
    } else {
        while (u >= r) {
            u = u - r;
            x += 1;
            r = r * fma(a, sg_rcp(rcp, x), -s);
            if (!(r > 0.0)) break;
        }
    }
    return x < n ? x : n;
}

// Stirling-series remainder fc(k) = ln k! - ((k + 1/2) ln(k + 1) - (k + 1) + ln(2 pi)/2),
// tabulated for k < 10 (values computed from the definition), series beyond.
SG_HD double sg_stirling_fc(uint32_t k) {
    switch (k) {
        case 0: return 0.08106146679532733;
        case 1: return 0.04134069595540946;
        case 2: return 0.027677925684997717;
        case 3: return 0.02079067210376584;
        case 4: return 0.01664469118982126;
        case 5: return 0.013876128823072875;
        case 6: return 0.011896709945893313;
        case 7: return 0.010411265261973668;
        case 8: return 0.00925546218270945;
        case 9: return 0.008330563433359472;
        default: break;
    }
    double k1 = (double)k + 1.0;
    double k1sq = k1 * k1;
    return (1.0 / 12.0 - (1.0 / 360.0 - 1.0 / 1260.0 / k1sq) / k1sq) / k1;
}

// ln k! = (k + 1/2) ln(k + 1) - (k + 1) + ln(2 pi)/2 + fc(k): the Stirling form with the
// remainder above (exact to rounding for every k).
SG_HD double sg_lnfact(uint32_t k) {
    const double k1 = (double)k + 1.0;
    return (k1 - 0.5) * sg_log(k1) - k1 + SG_HALF_LN_2PI + sg_stirling_fc(k);
}

// Table lookups with the same values as the direct forms (tables may be null).
SG_HD double sg_lnfact_t(uint32_t k, const double* lnf) {
    return (lnf && k < (uint32_t)SG_MODE_TABLE) ? lnf[k] : sg_lnfact(k);
}
SG_HD double sg_rcp_l(const double* rcpl, uint32_t x) {
    return (rcpl && x < (uint32_t)SG_MODE_TABLE) ? rcpl[x] : 1.0 / (double)x;
}

// Inversion from the mode for p <= 1/2, s = p / q: the support is searched in the order
// m, m+1, m-1, m+2, m-2, ... (one side alone once the other end is reached), subtracting
// each pmf value from one uniform until it goes negative.  f(m) from the log-factorials;
// the neighbours by the pmf ratios f(x+1)/f(x) = (n+1) s / (x+1) - s and
// f(x-1)/f(x) = x r / (n - x + 1), r = q / p.
SG_HD uint32_t sg_binom_mode(sg_stream* st, uint32_t n, double p, double s, const double* rcpl,
                             const double* lnf) {
    const double q = 1.0 - p;
    const double dn = (double)n;
    uint32_t m = (uint32_t)floor((dn + 1.0) * p);
    if (m > n) m = n;
    const double lf = ((sg_lnfact_t(n, lnf) - sg_lnfact_t(m, lnf)) - sg_lnfact_t(n - m, lnf)) +
                      (double)m * sg_log(p) + (double)(n - m) * sg_log(q);
    const double fm = sg_exp(lf);
    const double a = (dn + 1.0) * s;
    const double r = q / p;
    double u = sg_u01_co(sg_next_u32(st)) - fm;
    if (u < 0.0) return m;
    double fu = fm, fd = fm;
    uint32_t xu = m, xd = m;
    for (;;) {
        const bool cu = xu < n, cd = xd > 0u;
        if (!cu && !cd) return m;  // only when rounding left mass uncovered
        if (cu) {
            fu = fu * fma(a, sg_rcp_l(rcpl, xu + 1u), -s);
            xu += 1u;
            u = u - fu;
            if (u < 0.0) return xu;
        }
        if (cd) {
            fd = fd * ((double)xd * r) * sg_rcp_l(rcpl, n - xd + 1u);
            xd -= 1u;
            u = u - fd;
            if (u < 0.0) return xd;
        }
    }
}

// BTRD for p <= 1/2 and n p >= SG_MODE_CUT.  Candidates outside [0, n] are
// rejected.  The iteration cap is never reached in practice (acceptance rate
// is above 0.8 per round); if it were, the mode is returned.
SG_HD uint32_t sg_btrd(sg_stream* st, uint32_t n, double p) {
    double dn = (double)n;
    double q = 1.0 - p;
    double m = floor((dn + 1.0) * p);
    double r = p / q;
    double nr = (dn + 1.0) * r;
    double npq = dn * p * q;
    double sq = sqrt(npq);
    double b = 1.15 + 2.53 * sq;
    double a = -0.0873 + 0.0248 * b + 0.01 * p;
    double c = dn * p + 0.5;
    double alpha = (2.83 + 5.1 / b) * sq;
    double vr = 0.92 - 4.2 / b;
    double urvr = 0.86 * vr;
    uint32_t mi = (uint32_t)m;
    for (int iter = 0; iter < SG_BTRD_MAX_ITERS; ++iter) {
        double v = sg_u01_co(sg_next_u32(st));
        double u;
        if (v <= urvr) {
            u = v / vr - 0.43;
            double kq = floor((2.0 * a / (0.5 - fabs(u)) + b) * u + c);
            if (kq < 0.0 || kq > dn) continue;
            return (uint32_t)kq;
        }
        if (v >= vr) {
            u = sg_u01_co(sg_next_u32(st)) - 0.5;
        } else {
            u = v / vr - 0.93;
            u = (u < 0.0 ? -0.5 : 0.5) - u;
            v = sg_u01_co(sg_next_u32(st)) * vr;
        }
        double us = 0.5 - fabs(u);
        double kd = floor((2.0 * a / us + b) * u + c);
        if (kd < 0.0 || kd > dn) continue;
        v = v * alpha / (a / (us * us) + b);
        double km = fabs(kd - m);
        uint32_t k = (uint32_t)kd;
        if (km <= 15.0) {
            // Recursive evaluation of f(k)/f(m).
            double f = 1.0;
            if (mi < k) {
                for (uint32_t i = mi + 1; i <= k; ++i) f = f * (nr / (double)i - r);
            } else if (mi > k) {
                for (uint32_t i = k + 1; i <= mi; ++i) v = v * (nr / (double)i - r);
            }
            if (v <= f) return k;
            continue;
        }
        // Squeeze on log f(k)/f(m), then the exact test with Stirling corrections.
        v = sg_log(v);
        double rho = (km / npq) * (((km / 3.0 + 0.625) * km + 1.0 / 6.0) / npq + 0.5);
        double t = -km * km / (2.0 * npq);
        if (v < t - rho) return k;
        if (v > t + rho) continue;
        double nm = dn - m + 1.0;
        double h = (m + 0.5) * sg_log((m + 1.0) / (r * nm)) + sg_stirling_fc(mi) +
                   sg_stirling_fc(n - mi);
        double nk = dn - kd + 1.0;
        double bound = h + (dn + 1.0) * sg_log(nm / nk) + (kd + 0.5) * sg_log(nk * r / (kd + 1.0)) -
                       sg_stirling_fc(k) - sg_stirling_fc(n - k);
        if (v <= bound) return k;
    }
    return mi;
}

// Binomial(n, p) for any p (values <= 0 give 0, >= 1 give n).  For p > 1/2
// the sample is n - Binomial(n, 1 - p) (1 - p is exact there).
// Odds ratio of the smaller tail, pp / (1 - pp) with pp = min(p, 1 - p): the value the
// samplers below use; callers with a fixed p may compute it once.
SG_HD double sg_binom_odds(double p) {
    double pp = (p > 0.5) ? 1.0 - p : p;
    return pp / (1.0 - pp);
}

// Binomial(n, p) with odds = sg_binom_odds(p) supplied by the caller; rcp (SG_RCP_TABLE
// entries), rcpl and lnf (SG_MODE_TABLE entries) are optional tables of 1/x and ln x!.
SG_HD uint32_t sg_binom_o(sg_stream* st, uint32_t n, double p, double odds, const double* rcp,
                          const double* rcpl = nullptr, const double* lnf = nullptr) {
    if (n == 0 || !(p > 0.0)) return 0;
    if (p >= 1.0) return n;
    bool flip = p > 0.5;
    double pp = flip ? 1.0 - p : p;
    const double np = (double)n * pp;
    uint32_t k;
    if (np < SG_BINV_CUT)
        k = sg_binv(st, n, pp, rcp, odds);
    else if (np < SG_MODE_CUT)
        k = sg_binom_mode(st, n, pp, odds, rcpl, lnf);
    else
        k = sg_btrd(st, n, pp);
    return flip ? n - k : k;
}

SG_HD uint32_t sg_binom(sg_stream* st, uint32_t n, double p, const double* rcp = nullptr) {
    if (n == 0 || !(p > 0.0)) return 0;
    if (p >= 1.0) return n;
    return sg_binom_o(st, n, p, sg_binom_odds(p), rcp);
}

/*
 * Deterministic transcendentals for the particle pass.
 *
 * The particle pass must give the same bits on the GPU and on the CPU so its
 * checksum is reproducible and can be checked against a CPU replica. Basic
 * IEEE operations (+ - * / sqrt) are correctly rounded on both sides, but
 * library sin, cos and log differ between CUDA and glibc, so the few
 * transcendentals the spawn uses are written here from their series, using
 * only basic double operations, and rounded to float once at the end.
 * Evaluating in double makes the float result accurate to well under an
 * ulp; using only correctly rounded operations in a fixed order makes it
 * bit-identical wherever it runs, provided the compiler does not contract
 * multiplies and adds into fused operations (nvcc --fmad=false, gcc
 * -ffp-contract=off for every translation unit that needs the bits).
 *
 * Methods:
 *  - log: x = m 2^e with m in [sqrt(1/2), sqrt(2)), log m = 2 atanh(s),
 *    s = (m - 1)/(m + 1), atanh by its odd power series (|s| <= 0.1716, so
 *    terms through s^17 leave a relative error below 1e-16).
 *  - sin, cos: reduction by the nearest multiple of pi/2 with pi/2 split in
 *    two doubles (Cody and Waite 1980, Software Manual for the Elementary
 *    Functions), then the Taylor series of sin and cos on |r| <= pi/4
 *    through r^17 and r^18.
 *  - x^(3/4) and x^(1/4): products of square roots, exact compositions of
 *    correctly rounded operations.
 */
#ifndef GARGANTUA_DETMATH_H
#define GARGANTUA_DETMATH_H

#include <stdint.h>
#include <string.h>
#include <math.h>

#if defined(__CUDACC__)
#define GG_HD __host__ __device__ __forceinline__
#else
#define GG_HD static inline
#endif

GG_HD uint64_t gg_double_bits(double x) {
#if defined(__CUDA_ARCH__)
    return (uint64_t)__double_as_longlong(x);
#else
    uint64_t b;
    memcpy(&b, &x, sizeof b);
    return b;
#endif
}

GG_HD double gg_bits_double(uint64_t b) {
#if defined(__CUDA_ARCH__)
    return __longlong_as_double((long long)b);
#else
    double x;
    memcpy(&x, &b, sizeof x);
    return x;
#endif
}

/* Natural logarithm for finite x > 0 (normal doubles only; every float is a
 * normal double). */
GG_HD double gg_log_d(double x) {
    uint64_t bits = gg_double_bits(x);
    int e = (int)((bits >> 52) & 0x7ff) - 1023;
    double m = gg_bits_double((bits & 0x000fffffffffffffULL) | 0x3ff0000000000000ULL);
    if (m > 1.4142135623730951) {
        m = m * 0.5;
        e = e + 1;
    }
    double s = (m - 1.0) / (m + 1.0);
    double s2 = s * s;
    /* atanh(s) = s (1 + s^2/3 + s^4/5 + ... + s^16/17) */
    double p = 1.0 / 17.0;
    p = p * s2 + 1.0 / 15.0;
    p = p * s2 + 1.0 / 13.0;
    p = p * s2 + 1.0 / 11.0;
    p = p * s2 + 1.0 / 9.0;
    p = p * s2 + 1.0 / 7.0;
    p = p * s2 + 1.0 / 5.0;
    p = p * s2 + 1.0 / 3.0;
    p = p * s2 + 1.0;
    double logm = 2.0 * (s * p);
    /* ln 2 = hi + lo, hi holding 33 significant bits so e * hi is exact. */
    const double ln2_hi = 6.93147180485539138317e-01;
    const double ln2_lo = 7.44061711001239684738e-11;
    double de = (double)e;
    return de * ln2_hi + (de * ln2_lo + logm);
}

/* sin and cos of a double argument of moderate size (|x| < 2^20). */
GG_HD void gg_sincos_d(double x, double* s_out, double* c_out) {
    const double two_over_pi = 6.36619772367581382433e-01;
    /* pi/2 = hi + lo, hi holding 21 significant bits so k * hi is exact. */
    const double pio2_hi = 1.57079601287841796875e+00;
    const double pio2_lo = 3.13916478650481311129e-07;
    double kd = floor(x * two_over_pi + 0.5);
    double r = (x - kd * pio2_hi) - kd * pio2_lo;
    double r2 = r * r;
    /* sin r = r (1 - r^2/3! + r^4/5! - ... + r^16/17!) */
    double ps = 1.0 / 355687428096000.0;          /* 1/17! */
    ps = ps * r2 - 1.0 / 1307674368000.0;         /* 1/15! */
    ps = ps * r2 + 1.0 / 6227020800.0;            /* 1/13! */
    ps = ps * r2 - 1.0 / 39916800.0;              /* 1/11! */
    ps = ps * r2 + 1.0 / 362880.0;                /* 1/9!  */
    ps = ps * r2 - 1.0 / 5040.0;                  /* 1/7!  */
    ps = ps * r2 + 1.0 / 120.0;                   /* 1/5!  */
    ps = ps * r2 - 1.0 / 6.0;                     /* 1/3!  */
    double sr = r + r * (r2 * ps);
    /* cos r = 1 - r^2/2! + r^4/4! - ... + r^18/18! */
    double pc = 1.0 / 6402373705728000.0;         /* 1/18! */
    pc = pc * r2 - 1.0 / 20922789888000.0;        /* 1/16! */
    pc = pc * r2 + 1.0 / 87178291200.0;           /* 1/14! */
    pc = pc * r2 - 1.0 / 479001600.0;             /* 1/12! */
    pc = pc * r2 + 1.0 / 3628800.0;               /* 1/10! */
    pc = pc * r2 - 1.0 / 40320.0;                 /* 1/8!  */
    pc = pc * r2 + 1.0 / 720.0;                   /* 1/6!  */
    pc = pc * r2 - 1.0 / 24.0;                    /* 1/4!  */
    pc = pc * r2 + 0.5;                           /* 1/2!  */
    double cr = 1.0 - r2 * pc;
    int64_t k = (int64_t)kd;
    int q = (int)(k & 3);
    double s, c;
    if (q == 0) { s = sr; c = cr; }
    else if (q == 1) { s = cr; c = -sr; }
    else if (q == 2) { s = -sr; c = -cr; }
    else { s = -cr; c = sr; }
    *s_out = s;
    *c_out = c;
}

GG_HD float gg_logf(float x) { return (float)gg_log_d((double)x); }

GG_HD void gg_sincosf(float x, float* s, float* c) {
    double sd, cd;
    gg_sincos_d((double)x, &sd, &cd);
    *s = (float)sd;
    *c = (float)cd;
}

GG_HD float gg_sinf(float x) { float s, c; gg_sincosf(x, &s, &c); return s; }
GG_HD float gg_cosf(float x) { float s, c; gg_sincosf(x, &s, &c); return c; }

/* x^(3/4) = x^(1/2) x^(1/4) for x >= 0. */
GG_HD float gg_pow34f(float x) {
    float h = sqrtf(x);
    return h * sqrtf(h);
}

/* x^(1/4) for x >= 0. */
GG_HD float gg_pow14f(float x) { return sqrtf(sqrtf(x)); }

/* The thin-disk profile's powers x^(3/4) t^(1/4) (Common.h:49-53) for x, t
 * >= 0, given h = sqrt(x) (which the profile's zero-torque factor has
 * computed already): h (x t)^(1/4), three square roots in all where the
 * separate powers take four. */
GG_HD float gg_disk_powers(float x, float h, float t) { return h * sqrtf(sqrtf(x * t)); }

#endif

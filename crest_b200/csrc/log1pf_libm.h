/*
 * Single-precision log1p with the exact rounding behaviour of the platform
 * libm that the reference's Rust kernels call through f32::ln_1p
 * (src/kernels.rs:81 -> glibc 2.39 log1pf on x86-64 Linux).
 *
 * glibc's log1pf is not correctly rounded (about 0.4% of non-negative inputs
 * differ from the correctly rounded result by one ulp), so a correctly
 * rounded GPU log1p would not reproduce the reference's normalised values.
 * This function follows the published fdlibm method for log1p that glibc's
 * single-precision version uses:
 *
 *   1. reduce 1+x = 2^k (1+f) with sqrt(2)/2 < 1+f < sqrt(2); when k != 0
 *      the rounding error of u = fl(1+x) is carried as c = ((1+x)-u)/u;
 *   2. with s = f/(2+f), log(1+f) = f - (f^2/2 - s (f^2/2 + R(s^2))), R a
 *      degree-7 polynomial in s^2 with fdlibm's Remez coefficients Lp1..Lp7
 *      (the double-precision coefficients rounded to float);
 *   3. log1p(x) = k ln2_hi + (f - (hfsq - (s (hfsq + R) + (k ln2_lo + c)))).
 *
 * Every operation is an IEEE-754 binary32 operation in a fixed order.  On
 * the device the explicit round-to-nearest intrinsics keep nvcc from fusing
 * multiply-adds; host builds must use -ffp-contract=off.  Equality with the
 * platform libm over all 2^32 inputs is checked by tests/test_log1pf.py.
 */
#ifndef CREST_LOG1PF_LIBM_H
#define CREST_LOG1PF_LIBM_H

#include <stdint.h>
#include <string.h>
#ifndef __cplusplus
#include <stdbool.h>
#endif

#if defined(__CUDACC__)
#define CREST_HD __host__ __device__ __forceinline__
#else
#define CREST_HD static inline
#endif

#if defined(__CUDA_ARCH__)
#define L1P_ADD(a, b) __fadd_rn((a), (b))
#define L1P_SUB(a, b) __fsub_rn((a), (b))
#define L1P_MUL(a, b) __fmul_rn((a), (b))
#define L1P_DIV(a, b) __fdiv_rn((a), (b))
CREST_HD uint32_t l1p_bits(float x) { return __float_as_uint(x); }
CREST_HD float l1p_from(uint32_t u) { return __uint_as_float(u); }
#else
#define L1P_ADD(a, b) ((a) + (b))
#define L1P_SUB(a, b) ((a) - (b))
#define L1P_MUL(a, b) ((a) * (b))
#define L1P_DIV(a, b) ((a) / (b))
CREST_HD uint32_t l1p_bits(float x) { uint32_t u; memcpy(&u, &x, 4); return u; }
CREST_HD float l1p_from(uint32_t u) { float x; memcpy(&x, &u, 4); return x; }
#endif

/* Polynomial tail and reconstruction: step 2 and 3 of the method. */
CREST_HD float l1p_reconstruct(float f, int k, float c) {
    const float ln2_hi = l1p_from(0x3f317180u); /* ln2 with 9 trailing zero bits   */
    const float ln2_lo = l1p_from(0x3717f7d1u); /* ln2 - ln2_hi                    */
    const float lp1 = l1p_from(0x3f2aaaabu), lp2 = l1p_from(0x3ecccccdu), lp3 = l1p_from(0x3e924925u),
                lp4 = l1p_from(0x3e638e29u), lp5 = l1p_from(0x3e3a3325u), lp6 = l1p_from(0x3e1cd04fu),
                lp7 = l1p_from(0x3e178897u);
    const float hfsq = L1P_MUL(L1P_MUL(0.5f, f), f);
    const float s = L1P_DIV(f, L1P_ADD(2.0f, f));
    const float z = L1P_MUL(s, s);
    float r = L1P_ADD(lp6, L1P_MUL(z, lp7));
    r = L1P_ADD(lp5, L1P_MUL(z, r));
    r = L1P_ADD(lp4, L1P_MUL(z, r));
    r = L1P_ADD(lp3, L1P_MUL(z, r));
    r = L1P_ADD(lp2, L1P_MUL(z, r));
    r = L1P_ADD(lp1, L1P_MUL(z, r));
    r = L1P_MUL(z, r);
    const float t = L1P_MUL(s, L1P_ADD(hfsq, r));
    if (k == 0) return L1P_SUB(f, L1P_SUB(hfsq, t));
    const float kf = (float)k;
    const float lo = L1P_ADD(L1P_MUL(kf, ln2_lo), c);
    return L1P_SUB(L1P_MUL(kf, ln2_hi), L1P_SUB(L1P_SUB(hfsq, L1P_ADD(t, lo)), f));
}

/* |f| < 2^-20 after reduction: a two-term series replaces the polynomial. */
CREST_HD float l1p_tiny_f(float f, int k, float c) {
    const float ln2_hi = l1p_from(0x3f317180u), ln2_lo = l1p_from(0x3717f7d1u);
    const float kf = (float)k;
    if (f == 0.0f) {
        if (k == 0) return 0.0f;
        return L1P_ADD(L1P_MUL(kf, ln2_hi), L1P_ADD(c, L1P_MUL(kf, ln2_lo)));
    }
    const float hfsq = L1P_MUL(L1P_MUL(0.5f, f), f);
    const float r = L1P_MUL(hfsq, L1P_SUB(1.0f, L1P_MUL(l1p_from(0x3f2aaaabu), f)));
    if (k == 0) return L1P_SUB(f, r);
    return L1P_SUB(L1P_MUL(kf, ln2_hi), L1P_SUB(L1P_SUB(r, L1P_ADD(L1P_MUL(kf, ln2_lo), c)), f));
}

CREST_HD float crest_log1pf(float x) {
    const uint32_t bits = l1p_bits(x);
    const int32_t hx = (int32_t)bits;
    const uint32_t ax = bits & 0x7fffffffu;
    /* NaN and +inf propagate; -1 -> -inf; below -1 -> NaN */
    if (ax > 0x7f800000u) return L1P_ADD(x, x);
    if (hx >= 0x7f800000) return L1P_ADD(x, x);
    /* region where 1+x needs no reduction: -(1-sqrt(2)/2) <= x < sqrt(2)-1 */
    const bool near_zero = (hx < 0x3ed413d7) && (hx > 0 || hx <= (int32_t)0xbe95f61fu);
    if (hx < 0x3ed413d7) {
        if (ax >= 0x3f800000u) {
            if (x == -1.0f) return l1p_from(0xff800000u);
            return l1p_from(0x7fc00000u);
        }
        if (ax < 0x31000000u) { /* |x| < 2^-29 */
            if (ax < 0x24800000u) return x;
            return L1P_SUB(x, L1P_MUL(L1P_MUL(x, x), 0.5f));
        }
    }
    if (near_zero) return l1p_reconstruct(x, 0, 0.0f);
    /* step 1: 1+x = 2^k (1+f) */
    float u, c;
    int32_t hu;
    int k;
    if (hx < 0x5a000000) { /* x < 2^53: keep the rounding error of 1+x */
        u = L1P_ADD(1.0f, x);
        hu = (int32_t)l1p_bits(u);
        k = (hu >> 23) - 127;
        c = (k > 0) ? L1P_SUB(1.0f, L1P_SUB(u, x)) : L1P_SUB(x, L1P_SUB(u, 1.0f));
        c = L1P_DIV(c, u);
    } else {
        u = x;
        hu = (int32_t)l1p_bits(u);
        k = (hu >> 23) - 127;
        c = 0.0f;
    }
    hu &= 0x007fffff;
    int32_t tag;
    if (hu < 0x3504f7) {
        u = l1p_from((uint32_t)hu | 0x3f800000u);
        tag = hu;
    } else {
        k += 1;
        u = l1p_from((uint32_t)hu | 0x3f000000u);
        tag = (0x00800000 - hu) >> 2;
    }
    const float f = L1P_SUB(u, 1.0f);
    if (tag == 0) return l1p_tiny_f(f, k, c);
    return l1p_reconstruct(f, k, c);
}

#endif

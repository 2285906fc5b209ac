// trig.cuh -- the sine and cosine of the SIN and COS ops, single precision.
//
// The reference evaluates SIN/COS with the C library's sinf/cosf
// (src/ISA.h:219-231).  CUDA's own sinf/cosf cost about 30 instructions per
// case and round correctly about 80% of the time between 0.5 and 2^17.
// These are about 20 instructions per case on |x| < 2^17.  They round
// correctly about 85% of the time, stay within 1.56 ulp of the exact value,
// and give the same bits on the host and the device.
//
// Method (own implementation of textbook algorithms):
//  * |x| < 2^17: Cody and Waite's additive reduction (W. J. Cody, W. Waite,
//    "Software Manual for the Elementary Functions", 1980) by multiples of
//    pi/2, held in three floats P1 + P2 + P3.  The quadrant j is the nearest
//    integer to |x| 2/pi, taken from the low bits of a 1.5 * 2^23 + |x| 2/pi
//    sum (no float-to-integer conversion).  With FMA the first step
//    |x| - j P1 is exact.  The reduced argument r in [-pi/4, pi/4] then goes
//    into minimax polynomials r + r^3 S(r^2) and 1 + r^2 C(r^2).  Their
//    coefficients were fitted by the Remez exchange algorithm for relative
//    error (sin: 2^-26.9, cos: 2^-33.8 before rounding the coefficients to
//    float).
//  * |x| >= 2^17, infinities and NaN: Payne and Hanek's reduction (M. Payne,
//    R. Hanek, "Radian reduction for trigonometric functions", SIGNUM
//    Newsletter 18(1), 1983).  The 24-bit significand is multiplied by a
//    96-bit window of the binary expansion of 2/pi in integer arithmetic.
//    That gives |x| 2/pi mod 4 with 62 fraction bits, so the reduced
//    argument is exact to double precision.  Degree-11 and degree-10
//    polynomials (Remez, 2^-46.7 and 2^-43.5) evaluate it in double, and the
//    result is rounded once to float.
//
// sin(-x) = -sin(x) and cos(-x) = cos(x) hold bit for bit: both reduce |x|,
// and sin puts x's sign back at the end (so sin(-0) = -0).  Infinities
// and NaN give the NaN 0x7fffffff, as the device's own arithmetic does.
//
// Every operation is a correctly rounded IEEE operation (explicit
// round-to-nearest intrinsics on the device, no contraction on the host), so
// the host build of this header computes the same bits as the device.  The
// oracle compiles it to state the device's transcendental ops on the CPU.
// The interpreter's product path runs only the device build.
//
// Plain C99 when compiled outside nvcc (the oracle is C).
#ifndef GALOP_TRIG_CUH
#define GALOP_TRIG_CUH

#include <stdint.h>
#include <string.h>
#include <math.h>

#if defined(__CUDACC__)
#define GT_FN __host__ __device__ __forceinline__
#define GT_SLOW static __host__ __device__ __noinline__
#else
#define GT_FN static inline
#define GT_SLOW static
#endif

/* Arguments with |x| below this take the Cody-Waite path. */
#define GALOP_TRIG_FAST_LIMIT 131072.0f

/* pi/2 = P1 + P2 + P3 (each the float nearest to what remains), 2/pi, 1.5 * 2^23. */
#define GT_P1 0x1.921fb6p+0f
#define GT_P2 -0x1.777a5cp-25f
#define GT_P3 -0x1.ee59dap-50f
#define GT_TWO_OVER_PI 0x1.45f306p-1f
#define GT_ROUND 0x1.8p+23f

/* sin r = r + r^3 (S1 + S2 z + S3 z^2), cos r = 1 + z (C1 + C2 z + C3 z^2 + C4 z^3), z = r^2. */
#define GT_S1 -0x1.555554p-3f
#define GT_S2 0x1.110b9ep-7f
#define GT_S3 -0x1.9a728cp-13f
#define GT_C1 -0x1p-1f
#define GT_C2 0x1.55553cp-5f
#define GT_C3 -0x1.6c07d2p-10f
#define GT_C4 0x1.990f5cp-16f

/* Double-precision polynomials of the Payne-Hanek path. */
#define GT_DS1 -0x1.5555555555411p-3
#define GT_DS2 0x1.1111110ef1153p-7
#define GT_DS3 -0x1.a019fbb141d5dp-13
#define GT_DS4 0x1.71d873acf525fp-19
#define GT_DS5 -0x1.a9ae2bf88ab3bp-26
#define GT_DC1 -0x1.ffffffffe7229p-2
#define GT_DC2 0x1.555555447434bp-5
#define GT_DC3 -0x1.6c16b26650f4bp-10
#define GT_DC4 0x1.a00e42d7919d8p-16
#define GT_DC5 -0x1.23b428ab42cafp-22
/* pi/2 x 2^-62: scales the 62-bit fixed-point reduced argument. */
#define GT_PIO2_2M62 0x1.921fb54442d18p-62

GT_FN float gt_mul(float a, float b) {
#if defined(__CUDA_ARCH__)
    return __fmul_rn(a, b);
#else
    return a * b;
#endif
}
GT_FN float gt_sub(float a, float b) {
#if defined(__CUDA_ARCH__)
    return __fsub_rn(a, b);
#else
    return a - b;
#endif
}
GT_FN float gt_fma(float a, float b, float c) {
#if defined(__CUDA_ARCH__)
    return __fmaf_rn(a, b, c);
#else
    return fmaf(a, b, c);
#endif
}
GT_FN double gt_dmul(double a, double b) {
#if defined(__CUDA_ARCH__)
    return __dmul_rn(a, b);
#else
    return a * b;
#endif
}
GT_FN double gt_dfma(double a, double b, double c) {
#if defined(__CUDA_ARCH__)
    return __fma_rn(a, b, c);
#else
    return fma(a, b, c);
#endif
}
GT_FN uint32_t gt_bits(float f) {
#if defined(__CUDA_ARCH__)
    return __float_as_uint(f);
#else
    uint32_t u;
    memcpy(&u, &f, sizeof u);
    return u;
#endif
}
GT_FN float gt_float(uint32_t u) {
#if defined(__CUDA_ARCH__)
    return __uint_as_float(u);
#else
    float f;
    memcpy(&f, &u, sizeof f);
    return f;
#endif
}

/* Bits 1..320 of the binary expansion of 2/pi (2/pi = 0.a2f9836e...h),
   most significant first. */
#define GT_TWO_OVER_PI_BITS                                                                   \
    {0xa2f9836eu, 0x4e441529u, 0xfc2757d1u, 0xf534ddc0u, 0xdb629599u, 0x3c439041u, 0xfe5163abu, \
     0xdebbc561u, 0xb7246e3au, 0x424dd2e0u}
#if defined(__CUDACC__)
static __constant__ uint32_t gt_two_over_pi_dev[10] = GT_TWO_OVER_PI_BITS;
#endif
static const uint32_t gt_two_over_pi_host[10] = GT_TWO_OVER_PI_BITS;

/* Bits a..a+31 of 2/pi (bit k has weight 2^-k; bits k <= 0 are zero), for
   -31 <= a <= 257. */
GT_FN uint32_t gt_two_over_pi_word(int a) {
#if defined(__CUDA_ARCH__)
    const uint32_t* w = gt_two_over_pi_dev;
#else
    const uint32_t* w = gt_two_over_pi_host;
#endif
    if (a < 1) return w[0] >> (1 - a);
    const int i = (a - 1) >> 5, s = (a - 1) & 31;
    return s ? (w[i] << s) | (w[i + 1] >> (32 - s)) : w[i];
}

/* The value with the bits of y and the sign bit toggled where t has it. */
GT_FN float gt_flip(float y, uint32_t t) { return gt_float(gt_bits(y) ^ (t & 0x80000000u)); }

/* Payne-Hanek path: sin (cosine = 0) or cos (cosine = 1) of x with
   |x| >= GALOP_TRIG_FAST_LIMIT, an infinity or NaN. */
GT_SLOW float galop_trig_slow(float x, uint32_t cosine) {
    const uint32_t ux = gt_bits(x) & 0x7fffffffu;
    if (ux >= 0x7f800000u) return gt_float(0x7fffffffu);
    /* |x| = m 2^e with m the 24-bit significand (|x| >= 2^17 is normal) */
    const uint64_t m = (uint64_t)((ux & 0x7fffffu) | 0x800000u);
    const int e = (int)(ux >> 23) - 150;
    /* T = floor(2^(e+94) 2/pi) mod 2^96 = bits e-1 .. e+94 of 2/pi */
    const uint64_t t_hi = gt_two_over_pi_word(e - 1);
    const uint64_t t_mid = gt_two_over_pi_word(e + 31);
    const uint64_t t_lo = gt_two_over_pi_word(e + 63);
    /* m T mod 2^96; its top 64 bits are |x| 2/pi mod 4 with 62 fraction bits */
    const uint64_t p0 = m * t_lo;
    const uint64_t p1 = m * t_mid + (p0 >> 32);
    const uint64_t p2 = m * t_hi + (p1 >> 32);
    const uint64_t f = (p2 << 32) | (p1 & 0xffffffffu);
    /* nearest quadrant and the signed remainder in [-1/2, 1/2) quadrants */
    const uint64_t q = (f + (1ull << 61)) >> 62;
    const int64_t rem = (int64_t)(f - (q << 62));
#if defined(__CUDA_ARCH__)
    const double r = gt_dmul(__ll2double_rn(rem), GT_PIO2_2M62);
#else
    const double r = gt_dmul((double)rem, GT_PIO2_2M62);
#endif
    const double z = gt_dmul(r, r);
    double ps = gt_dfma(gt_dfma(gt_dfma(gt_dfma(GT_DS5, z, GT_DS4), z, GT_DS3), z, GT_DS2), z, GT_DS1);
    const double s = gt_dfma(gt_dmul(r, z), ps, r);
    const double c = gt_dfma(gt_dfma(gt_dfma(gt_dfma(gt_dfma(GT_DC5, z, GT_DC4), z, GT_DC3), z, GT_DC2), z,
                                     GT_DC1), z, 1.0);
    const uint32_t qq = (uint32_t)q + cosine;
#if defined(__CUDA_ARCH__)
    const float y = __double2float_rn((qq & 1u) ? c : s);
#else
    const float y = (float)((qq & 1u) ? c : s);
#endif
    return gt_flip(y, (qq << 30) ^ (cosine ? 0u : gt_bits(x)));
}

/* Cody-Waite path for |x| < GALOP_TRIG_FAST_LIMIT (callers check). */
GT_FN float galop_trig_fast(float x, uint32_t cosine) {
    const float ax = fabsf(x);
    const float jr = gt_fma(ax, GT_TWO_OVER_PI, GT_ROUND);
    const float j = gt_sub(jr, GT_ROUND);
    const uint32_t q = gt_bits(jr) + cosine;
    float r = gt_fma(j, -GT_P1, ax);
    r = gt_fma(j, -GT_P2, r);
    r = gt_fma(j, -GT_P3, r);
    const float z = gt_mul(r, r);
    const float ps = gt_fma(gt_fma(GT_S3, z, GT_S2), z, GT_S1);
    const float s = gt_fma(gt_mul(r, z), ps, r);
    const float c = gt_fma(gt_fma(gt_fma(gt_fma(GT_C4, z, GT_C3), z, GT_C2), z, GT_C1), z, 1.0f);
    return gt_flip((q & 1u) ? c : s, (q << 30) ^ (cosine ? 0u : gt_bits(x)));
}

GT_FN int galop_trig_is_fast(float x) { return fabsf(x) < GALOP_TRIG_FAST_LIMIT; }

/* sin and cos of one float. */
GT_FN float galop_sinf(float x) { return galop_trig_is_fast(x) ? galop_trig_fast(x, 0u) : galop_trig_slow(x, 0u); }
GT_FN float galop_cosf(float x) { return galop_trig_is_fast(x) ? galop_trig_fast(x, 1u) : galop_trig_slow(x, 1u); }

#if defined(__CUDACC__)
/* sin (cosine = 0) or cos (cosine = 1) of a lane's K cases: the Cody-Waite
   path for all K, then Payne-Hanek for the elements that need it, so the
   warp takes the slow path only when one of its lanes has such an argument. */
template <int K>
__device__ __forceinline__ void galop_trig_k(const float (&b)[K], float (&t)[K], uint32_t cosine) {
    bool slow = false;
#pragma unroll
    for (int k = 0; k < K; ++k) {
        t[k] = galop_trig_fast(b[k], cosine);
        slow |= !galop_trig_is_fast(b[k]);
    }
    if (slow) {
#pragma unroll
        for (int k = 0; k < K; ++k)
            if (!galop_trig_is_fast(b[k])) t[k] = galop_trig_slow(b[k], cosine);
    }
}
#endif

#endif /* GALOP_TRIG_CUH */

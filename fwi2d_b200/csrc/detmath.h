// detmath.h — deterministic random numbers and elementary functions shared by
// host and device code, so that the random boundary is bit-identical wherever
// it is generated.
//
// The reference draws its random boundary from cuRAND XORWOW seeded with
// clock64() (src/modeling/modeling.cu:526-531) and from a std::mt19937 seeded
// by std::random_device (modeling.cu:406-407, admin.cpp:146-147), so it is not
// reproducible.  This engine replaces both with a counter-based generator:
//   * SplitMix64 mixing (Steele, Lea & Flood, "Fast splittable pseudorandom
//     number generators", OOPSLA 2014) of (seed, shot, stream, counter);
//   * standard normals by inversion with Wichura's AS 241 (PPND16, Applied
//     Statistics 37(3), 1988), accurate to about 1e-16;
//   * exp and log from Cody-Waite range reduction and Taylor / atanh series,
//     evaluated in double with no fused multiply-add.
// Everything is plain IEEE-754 +,-,*,/ and sqrt, which are correctly rounded
// on x86-64 (SSE2) and on sm_100a, so a translation unit compiled without FMA
// contraction (-ffp-contract=off on the host, -fmad=false on the device)
// gets the same bits on both.
#pragma once
#include <stdint.h>
#include <math.h>

#if defined(__CUDACC__)
#define DM_FN __host__ __device__ __forceinline__
#else
#define DM_FN static inline
#endif

namespace detm {

// Streams of the random-boundary generator.
enum : uint32_t { STREAM_BG_X = 1, STREAM_BG_Z = 2, STREAM_PDS = 3, STREAM_BUMP = 4 };

DM_FN uint64_t mix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// Key of one (seed, shot, stream) sequence; draw number `ctr` of it.
DM_FN uint64_t stream_key(uint64_t seed, uint32_t shot, uint32_t stream) {
    return mix64(mix64(seed) ^ (((uint64_t)shot << 32) | (uint64_t)stream));
}
DM_FN uint64_t draw(uint64_t key, uint64_t ctr) { return mix64(key ^ mix64(ctr)); }

// 24-bit uniform float in [0, 1).
DM_FN float u01f(uint64_t h) { return (float)(uint32_t)(h >> 40) * 5.9604644775390625e-8f; }
// 53-bit uniform double in (0, 1).
DM_FN double u01d_open(uint64_t h) { return ((double)(h >> 11) + 0.5) * 1.1102230246251565e-16; }

DM_FN double bits_to_double(uint64_t b) {
    union { uint64_t u; double d; } v; v.u = b; return v.d;
}
DM_FN uint64_t double_to_bits(double d) {
    union { uint64_t u; double d; } v; v.d = d; return v.u;
}

// Natural log of a positive, finite, normal double.
DM_FN double log_pos(double x) {
    uint64_t b = double_to_bits(x);
    int e = (int)((b >> 52) & 0x7FF) - 1023;
    double m = bits_to_double((b & 0x000FFFFFFFFFFFFFull) | 0x3FF0000000000000ull);  // [1,2)
    if (m > 1.4142135623730951) { m = m * 0.5; e = e + 1; }                             // [sqrt(.5), sqrt(2)]
    double s = (m - 1.0) / (m + 1.0);
    double s2 = s * s;
    // 2*atanh(s) = 2*(s + s^3/3 + s^5/5 + ...), |s| <= 0.1716
    double p = 1.0 / 23.0;
    p = p * s2 + 1.0 / 21.0;
    p = p * s2 + 1.0 / 19.0;
    p = p * s2 + 1.0 / 17.0;
    p = p * s2 + 1.0 / 15.0;
    p = p * s2 + 1.0 / 13.0;
    p = p * s2 + 1.0 / 11.0;
    p = p * s2 + 1.0 / 9.0;
    p = p * s2 + 1.0 / 7.0;
    p = p * s2 + 1.0 / 5.0;
    p = p * s2 + 1.0 / 3.0;
    p = p * s2 + 1.0;
    double lm = 2.0 * s * p;
    const double ln2_hi = 6.93147180369123816490e-01;  // high bits of ln 2
    const double ln2_lo = 1.90821492927058770002e-10;  // ln 2 - ln2_hi
    return ((double)e * ln2_hi + lm) + (double)e * ln2_lo;
}

// exp(x) for x <= 0 (returns 0 below about -708).
DM_FN double exp_nonpos(double x) {
    if (x < -708.0) return 0.0;
    const double inv_ln2 = 1.44269504088896338700e+00;
    const double ln2_hi = 6.93147180369123816490e-01;
    const double ln2_lo = 1.90821492927058770002e-10;
    double kf = x * inv_ln2 + 0.5;
    // floor for kf in [-1100, 1]
    int k = (int)kf;
    if ((double)k > kf) k = k - 1;
    double r = (x - (double)k * ln2_hi) - (double)k * ln2_lo;   // |r| <= ~0.35
    double p = 1.0 / 6227020800.0;            // 1/13!
    p = p * r + 1.0 / 479001600.0;            // 1/12!
    p = p * r + 1.0 / 39916800.0;
    p = p * r + 1.0 / 3628800.0;
    p = p * r + 1.0 / 362880.0;
    p = p * r + 1.0 / 40320.0;
    p = p * r + 1.0 / 5040.0;
    p = p * r + 1.0 / 720.0;
    p = p * r + 1.0 / 120.0;
    p = p * r + 1.0 / 24.0;
    p = p * r + 1.0 / 6.0;
    p = p * r + 0.5;
    p = p * r + 1.0;
    p = p * r + 1.0;
    if (k < -1022) {  // scale in two steps to reach the subnormal range
        p = p * bits_to_double((uint64_t)(k + 600 + 1023) << 52);
        return p * bits_to_double((uint64_t)(-600 + 1023) << 52);
    }
    return p * bits_to_double((uint64_t)(k + 1023) << 52);
}

// expf replacement for the Gaussian bumps: exp evaluated in double, rounded once.
DM_FN float expf_nonpos(float x) { return (float)exp_nonpos((double)x); }

// Inverse of the standard normal CDF, AS 241 PPND16, for p in (0,1).
DM_FN double ppnd16(double p) {
    double q = p - 0.5;
    if ((q < 0 ? -q : q) <= 0.425) {
        double r = 0.180625 - q * q;
        double num = (((((((2.5090809287301226727e+3 * r + 3.3430575583588128105e+4) * r
                     + 6.7265770927008700853e+4) * r + 4.5921953931549871457e+4) * r
                     + 1.3731693765509461125e+4) * r + 1.9715909503065514427e+3) * r
                     + 1.3314166789178437745e+2) * r + 3.3871328727963666080e0);
        double den = (((((((5.2264952788528545610e+3 * r + 2.8729085735721942674e+4) * r
                     + 3.9307895800092710610e+4) * r + 2.1213794301586595867e+4) * r
                     + 5.3941960214247511077e+3) * r + 6.8718700749205790830e+2) * r
                     + 4.2313330701600911252e+1) * r + 1.0);
        return q * num / den;
    }
    double r = q < 0 ? p : 1.0 - p;
    r = sqrt(-log_pos(r));
    double val;
    if (r <= 5.0) {
        r = r - 1.6;
        double num = (((((((7.74545014278341407640e-4 * r + 2.27238449892691845833e-2) * r
                     + 2.41780725177450611770e-1) * r + 1.27045825245236838258e0) * r
                     + 3.64784832476320460504e0) * r + 5.76949722146069140550e0) * r
                     + 4.63033784615654529590e0) * r + 1.42343711074968357734e0);
        double den = (((((((1.05075007164441684324e-9 * r + 5.47593808499534494600e-4) * r
                     + 1.51986665636164571966e-2) * r + 1.48103976427480074590e-1) * r
                     + 6.89767334985100004550e-1) * r + 1.67638483018380384940e0) * r
                     + 2.05319162663775882187e0) * r + 1.0);
        val = num / den;
    } else {
        r = r - 5.0;
        double num = (((((((2.01033439929228813265e-7 * r + 2.71155556874348757815e-5) * r
                     + 1.24266094738807843860e-3) * r + 2.65321895265761230930e-2) * r
                     + 2.96560571828504891230e-1) * r + 1.78482653991729133580e0) * r
                     + 5.46378491116411436990e0) * r + 6.65790464350110377720e0);
        double den = (((((((2.04426310338993978564e-15 * r + 1.42151175831644588870e-7) * r
                     + 1.84631831751005468180e-5) * r + 7.86869131145613259100e-4) * r
                     + 1.48753612908506148525e-2) * r + 1.36929880922735805310e-1) * r
                     + 5.99832206555887937690e-1) * r + 1.0);
        val = num / den;
    }
    return q < 0 ? -val : val;
}

// Standard normal draw `ctr` of a stream, as float.
DM_FN float normalf(uint64_t key, uint64_t ctr) { return (float)ppnd16(u01d_open(draw(key, ctr))); }

}  // namespace detm

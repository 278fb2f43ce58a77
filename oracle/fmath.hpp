// oracle/fmath.hpp -- deterministic exp / log for the oracle (TEST INFRASTRUCTURE ONLY).
//
// The reference calls the platform libm (`f32::exp`, `f32::ln`; glibc on Linux)
// for every transcendental: sigmoid/logit (src/math/mod.rs:183-192), the scale
// decode (mod.rs:72-78), alpha (src/cpu/backward.rs:344,444) and the SSIM
// window (backward.rs:764). libm and CUDA's expf disagree by an ulp on some
// inputs, and an ulp is enough to flip the 3-sigma AABB truncation that decides
// tile lists or the alpha >= 1/255 test. So the oracle and the CUDA kernels
// evaluate the SAME sequence of IEEE-754 operations (explicit fma, single
// roundings, no contraction) and agree bit for bit. Two routines:
//
//  * exp_cr / log_cr: double-precision Cody-Waite reduction (fdlibm's two-part
//    ln2) + Taylor polynomial (degree 13 for exp; log via 2*atanh((m-1)/(m+1))
//    through s^21), rounded once to float. This is correctly rounded except
//    with probability ~1e-8, so it matches glibc's expf wherever glibc is
//    itself correctly rounded. Used per Gaussian (sigmoid, scale, logit, SSIM
//    window, densification).
//  * expf_fast: single-precision Cody-Waite + degree-8 Taylor with a
//    compensated final sum (max error 0.62 ulp, measured). Used per
//    (pixel, splat) pair for alpha = opacity * exp(power).
#pragma once
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>

namespace orc {
namespace fm {

inline float bits_to_float(uint32_t u) { float f; std::memcpy(&f, &u, 4); return f; }
inline uint32_t float_to_bits(float f) { uint32_t u; std::memcpy(&u, &f, 4); return u; }
inline double bits_to_double(uint64_t u) { double f; std::memcpy(&f, &u, 8); return f; }
inline uint64_t double_to_bits(double f) { uint64_t u; std::memcpy(&u, &f, 8); return u; }

constexpr double LN2_HI_D = 6.93147180369123816490e-01;  // 32 significant bits
constexpr double LN2_LO_D = 1.90821492927058770002e-10;
constexpr double INV_LN2_D = 1.44269504088896338700e+00;

// e^x in double for x in [-104, 89] (|k| <= 151 so k*LN2_HI_D is exact).
inline double exp_core_d(double x) {
    const double SHIFT = 6755399441055744.0;  // 1.5 * 2^52
    double j = std::fma(x, INV_LN2_D, SHIFT);
    double k = j - SHIFT;
    double r = std::fma(-k, LN2_HI_D, x);
    r = std::fma(-k, LN2_LO_D, r);
    double p = 1.0 / 6227020800.0;            // 1/13!
    p = std::fma(p, r, 1.0 / 479001600.0);    // 1/12!
    p = std::fma(p, r, 1.0 / 39916800.0);
    p = std::fma(p, r, 1.0 / 3628800.0);
    p = std::fma(p, r, 1.0 / 362880.0);
    p = std::fma(p, r, 1.0 / 40320.0);
    p = std::fma(p, r, 1.0 / 5040.0);
    p = std::fma(p, r, 1.0 / 720.0);
    p = std::fma(p, r, 1.0 / 120.0);
    p = std::fma(p, r, 1.0 / 24.0);
    p = std::fma(p, r, 1.0 / 6.0);
    p = std::fma(p, r, 0.5);
    p = std::fma(p, r, 1.0);
    p = std::fma(p, r, 1.0);
    int ki = (int)k;
    return p * bits_to_double((uint64_t)(ki + 1023) << 52);
}

inline float exp_cr(float x) {
    if (x != x) return x + x;
    if (x > 88.7228394f) return std::numeric_limits<float>::infinity();
    if (x < -103.972084f) return 0.0f;
    return (float)exp_core_d((double)x);
}

// ln(d) in double for a positive, finite d that came from a float (every
// positive float is a normal double).
inline double log_pos_d(double d) {
    uint64_t b = double_to_bits(d);
    int e = (int)((b >> 52) & 0x7ffu) - 1023;
    double m = bits_to_double((b & 0x000fffffffffffffull) | 0x3ff0000000000000ull);  // [1, 2)
    if (m > 1.4142135623730951) { m = m * 0.5; e += 1; }
    double f = m - 1.0;
    double s = f / (2.0 + f);
    double z = s * s;
    double P = 2.0 / 21.0;
    P = std::fma(P, z, 2.0 / 19.0);
    P = std::fma(P, z, 2.0 / 17.0);
    P = std::fma(P, z, 2.0 / 15.0);
    P = std::fma(P, z, 2.0 / 13.0);
    P = std::fma(P, z, 2.0 / 11.0);
    P = std::fma(P, z, 2.0 / 9.0);
    P = std::fma(P, z, 2.0 / 7.0);
    P = std::fma(P, z, 2.0 / 5.0);
    P = std::fma(P, z, 2.0 / 3.0);
    double logm = std::fma(s * z, P, 2.0 * s);
    double ef = (double)e;
    return ef * LN2_HI_D + std::fma(ef, LN2_LO_D, logm);
}

inline float log_cr(float x) {
    if (x != x) return x + x;
    if (x < 0.0f) return std::numeric_limits<float>::quiet_NaN();
    if (x == 0.0f) return -std::numeric_limits<float>::infinity();
    if (x == std::numeric_limits<float>::infinity()) return x;
    return (float)log_pos_d((double)x);
}

// rasterizer.rs:262-269 linear_to_srgb (IEC 61966-2-1). The reference calls
// f32::powf(x, 1.0 / 2.4); here x^y = exp(y ln x) is evaluated in double and
// rounded once (correctly rounded except in rare near-halfway cases).
inline float linear_to_srgb(float x) {
    if (x <= 0.0031308f) return 12.92f * x;
    const float y = 1.0f / 2.4f;
    const float p = (float)exp_core_d((double)y * log_pos_d((double)x));
    return 1.055f * p - 0.055f;
}

// src/io/images.rs:76-82 srgb_to_linear: ((x + 0.055) / 1.055).powf(2.4) evaluated as
// exp(2.4 ln t) in double and rounded once (t > 0.0405 here).
inline float srgb_to_linear(float x) {
    if (x <= 0.04045f) return x / 12.92f;
    const float t = (x + 0.055f) / 1.055f;
    return (float)exp_core_d(2.4 * log_pos_d((double)t));
}

// Rust `f as u8`: truncate toward zero, saturate, NaN -> 0.
inline uint8_t as_u8(float f) {
    if (!(f > 0.0f)) return 0;
    if (f >= 255.0f) return 255;
    return (uint8_t)(int)f;
}

inline float expf_fast(float x) {
    if (x != x) return x + x;
    if (x > 88.7228394f) return std::numeric_limits<float>::infinity();
    if (x < -103.972084f) return 0.0f;
    const float L2E = 1.44269502f;
    const float SHIFT = 12582912.0f;          // 1.5 * 2^23: the fma rounds to an integer
    const float LN2_HI = 0.693145751953125f;  // 0x3F317200, 16 significant bits
    const float LN2_LO = 1.42860677e-06f;     // ln2 - LN2_HI
    float j = std::fma(x, L2E, SHIFT);
    float k = j - SHIFT;
    float rh = std::fma(-k, LN2_HI, x);       // exact
    float rl = -k * LN2_LO;
    float q = 2.48015873e-05f;                // 1/8!
    q = std::fma(q, rh, 1.98412698e-4f);      // 1/7!
    q = std::fma(q, rh, 1.38888889e-3f);      // 1/6!
    q = std::fma(q, rh, 8.33333333e-3f);      // 1/5!
    q = std::fma(q, rh, 4.16666667e-2f);      // 1/4!
    q = std::fma(q, rh, 1.66666667e-1f);      // 1/3!
    q = std::fma(q, rh, 0.5f);                // 1/2!
    float hi = 1.0f + rh;
    float lo = (1.0f - hi) + rh;              // exact error of hi (|rh| < 1)
    float s = rh * rh;
    float tail = std::fma(s, q, lo);          // e^rh = hi + tail
    float ea = hi + tail;
    tail = std::fma(rl, ea, tail);            // e^(rh+rl) ~ e^rh * (1 + rl)
    float p = hi + tail;
    int ki = (int)k;
    if (ki > 127) return (p * bits_to_float(254u << 23)) * bits_to_float((uint32_t)ki << 23);
    if (ki < -126) return (p * bits_to_float(1u << 23)) * bits_to_float((uint32_t)(ki + 253) << 23);
    return p * bits_to_float((uint32_t)(ki + 127) << 23);
}

}  // namespace fm
}  // namespace orc

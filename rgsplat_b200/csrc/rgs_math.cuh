// rgs_math.cuh -- device math shared by every kernel of the training path.
//
// Every expression below that feeds an integer decision (the 3-sigma AABB
// truncation of src/math/projection.rs:138-165, the culls of
// src/cpu/backward.rs:220-250) or a threshold test (alpha >= 1/255, T < 1e-4,
// backward.rs:341-355) is written as the same sequence of IEEE-754 roundings
// the reference evaluates: the translation units are compiled with
// --fmad=false so no a*b+c is fused, and fma is used only where written
// explicitly. The transcendental routines are the library's own (the
// reference calls libm):
//   * rgs_exp_cr / rgs_log_cr: double-precision Cody-Waite reduction with
//     fdlibm's two-part ln2, Taylor polynomial (degree 13 for exp; log through
//     2*atanh(s) up to s^21), one rounding to float. Correctly rounded except
//     with probability ~1e-8, so they agree with glibc's expf/logf wherever
//     those are correctly rounded. Used once per Gaussian.
//   * rgs_expf_fast: single-precision Cody-Waite + degree-8 Taylor with a
//     compensated final sum (max error 0.62 ulp). Used per (pixel, splat).
#pragma once
#include <cstdint>

#define RGS_HD __host__ __device__ __forceinline__

namespace rgs {

__device__ __forceinline__ double exp_core_d(double x) {
    const double LN2_HI = 6.93147180369123816490e-01;
    const double LN2_LO = 1.90821492927058770002e-10;
    const double INV_LN2 = 1.44269504088896338700e+00;
    const double SHIFT = 6755399441055744.0;
    double j = fma(x, INV_LN2, SHIFT);
    double k = j - SHIFT;
    double r = fma(-k, LN2_HI, x);
    r = fma(-k, LN2_LO, r);
    double p = 1.0 / 6227020800.0;
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
    return p * __longlong_as_double((long long)(ki + 1023) << 52);
}

__device__ __forceinline__ float exp_cr(float x) {
    if (x != x) return x + x;
    if (x > 88.7228394f) return __int_as_float(0x7f800000);
    if (x < -103.972084f) return 0.0f;
    return __double2float_rn(exp_core_d((double)x));
}

// ln(d) in double for a positive, finite d that came from a float.
__device__ __forceinline__ double log_pos_d(double d) {
    const double LN2_HI = 6.93147180369123816490e-01;
    const double LN2_LO = 1.90821492927058770002e-10;
    unsigned long long b = (unsigned long long)__double_as_longlong(d);
    int e = (int)((b >> 52) & 0x7ffull) - 1023;
    double m = __longlong_as_double((long long)((b & 0x000fffffffffffffull) | 0x3ff0000000000000ull));
    if (m > 1.4142135623730951) { m = m * 0.5; e += 1; }
    double f = m - 1.0;
    double s = f / (2.0 + f);
    double z = s * s;
    double P = 2.0 / 21.0;
    P = fma(P, z, 2.0 / 19.0);
    P = fma(P, z, 2.0 / 17.0);
    P = fma(P, z, 2.0 / 15.0);
    P = fma(P, z, 2.0 / 13.0);
    P = fma(P, z, 2.0 / 11.0);
    P = fma(P, z, 2.0 / 9.0);
    P = fma(P, z, 2.0 / 7.0);
    P = fma(P, z, 2.0 / 5.0);
    P = fma(P, z, 2.0 / 3.0);
    double logm = fma(s * z, P, 2.0 * s);
    double ef = (double)e;
    return ef * LN2_HI + fma(ef, LN2_LO, logm);
}

__device__ __forceinline__ float log_cr(float x) {
    if (x != x) return x + x;
    if (x < 0.0f) return __int_as_float(0x7fc00000);
    if (x == 0.0f) return __int_as_float(0xff800000);
    if (x == __int_as_float(0x7f800000)) return x;
    return __double2float_rn(log_pos_d((double)x));
}

// linear_to_srgb (src/cpu/rasterizer.rs:262-269, IEC 61966-2-1): powf(x, 1/2.4)
// evaluated as exp(y ln x) in double and rounded once.
__device__ __forceinline__ float linear_to_srgb(float x) {
    if (x <= 0.0031308f) return 12.92f * x;
    const float y = 1.0f / 2.4f;
    const float p = __double2float_rn(exp_core_d((double)y * log_pos_d((double)x)));
    return 1.055f * p - 0.055f;
}

// srgb_to_linear (src/io/images.rs:76-82): ((x + 0.055) / 1.055).powf(2.4)
// evaluated as exp(2.4 ln t) in double and rounded once.
__device__ __forceinline__ float srgb_to_linear(float x) {
    if (x <= 0.04045f) return x / 12.92f;
    const float t = (x + 0.055f) / 1.055f;
    return __double2float_rn(exp_core_d(2.4 * log_pos_d((double)t)));
}

// Rust `f as u8`: truncate toward zero, saturate, NaN -> 0.
__device__ __forceinline__ unsigned char as_u8(float f) {
    if (!(f > 0.0f)) return 0;
    if (f >= 255.0f) return 255;
    return (unsigned char)(int)f;
}

__device__ __forceinline__ float expf_fast(float x) {
    if (x != x) return x + x;
    if (x > 88.7228394f) return __int_as_float(0x7f800000);
    if (x < -103.972084f) return 0.0f;
    const float L2E = 1.44269502f;
    const float SHIFT = 12582912.0f;
    const float LN2_HI = 0.693145751953125f;
    const float LN2_LO = 1.42860677e-06f;
    float j = __fmaf_rn(x, L2E, SHIFT);
    float k = j - SHIFT;
    float rh = __fmaf_rn(-k, LN2_HI, x);
    float rl = -k * LN2_LO;
    float q = 2.48015873e-05f;
    q = __fmaf_rn(q, rh, 1.98412698e-4f);
    q = __fmaf_rn(q, rh, 1.38888889e-3f);
    q = __fmaf_rn(q, rh, 8.33333333e-3f);
    q = __fmaf_rn(q, rh, 4.16666667e-2f);
    q = __fmaf_rn(q, rh, 1.66666667e-1f);
    q = __fmaf_rn(q, rh, 0.5f);
    float hi = 1.0f + rh;
    float lo = (1.0f - hi) + rh;
    float s = rh * rh;
    float tail = __fmaf_rn(s, q, lo);
    float ea = hi + tail;
    tail = __fmaf_rn(rl, ea, tail);
    float p = hi + tail;
    int ki = (int)k;
    if (ki > 127) return (p * __int_as_float(254 << 23)) * __int_as_float(ki << 23);
    if (ki < -126) return (p * __int_as_float(1 << 23)) * __int_as_float((ki + 253) << 23);
    return p * __int_as_float((ki + 127) << 23);
}

// expf_fast restricted to x in [-87, 0] (or NaN), where none of its special
// cases (overflow, underflow, subnormal scaling) can occur: the same
// operations in the same order, so the result is bit-identical to
// expf_fast(x) on that domain. The blend kernels call it only for
// power in [ln(1 / (255 opacity)) - 0.01, 0], a subset of it.
__device__ __forceinline__ float expf_fast_nonpos(float x) {
    const float L2E = 1.44269502f;
    const float SHIFT = 12582912.0f;
    const float LN2_HI = 0.693145751953125f;
    const float LN2_LO = 1.42860677e-06f;
    float j = __fmaf_rn(x, L2E, SHIFT);
    float k = j - SHIFT;
    float rh = __fmaf_rn(-k, LN2_HI, x);
    float rl = -k * LN2_LO;
    float q = 2.48015873e-05f;
    q = __fmaf_rn(q, rh, 1.98412698e-4f);
    q = __fmaf_rn(q, rh, 1.38888889e-3f);
    q = __fmaf_rn(q, rh, 8.33333333e-3f);
    q = __fmaf_rn(q, rh, 4.16666667e-2f);
    q = __fmaf_rn(q, rh, 1.66666667e-1f);
    q = __fmaf_rn(q, rh, 0.5f);
    float hi = 1.0f + rh;
    float lo = (1.0f - hi) + rh;
    float s = rh * rh;
    float tail = __fmaf_rn(s, q, lo);
    float ea = hi + tail;
    tail = __fmaf_rn(rl, ea, tail);
    float p = hi + tail;
    return p * __int_as_float(((int)k + 127) << 23);
}

// ---- two pixels at once: Blackwell's packed f32x2 instructions ------------
// __fadd2_rn / __fmul2_rn / __ffma2_rn round each lane exactly like the scalar
// _rn operation (one issue slot for two lanes), so a sequence of them gives
// each lane the bits the same scalar sequence gives. One caveat, measured: the
// code generator may contract a packed multiply feeding a packed add into a
// packed FMA (one rounding instead of two), even without --fmad. Every such
// add is therefore written as __ffma2_rn(product, one, acc), with `one` =
// {1, 1} taken from a kernel argument, which it cannot fold: x * 1 + acc
// rounds once, exactly like the separate add.
__device__ __forceinline__ float2 bc2(float x) { return make_float2(x, x); }

// expf_fast_nonpos on two lanes: the same operations in the same order per
// lane (a negated operand moves to the exactly representable constant), so
// each lane is bit-identical to the scalar routine. 2^k is assembled from the
// shifted sum j, whose low mantissa bits hold k (bits(j) = bits(SHIFT) + k),
// which is the same power of two the scalar routine builds from (int)k.
__device__ __forceinline__ float2 expf_fast_nonpos2(float2 x, float2 one) {
    const float L2E = 1.44269502f;
    const float SHIFT = 12582912.0f;
    const float LN2_HI = 0.693145751953125f;
    const float LN2_LO = 1.42860677e-06f;
    const float2 j = __ffma2_rn(x, bc2(L2E), bc2(SHIFT));
    const float2 k = __fadd2_rn(j, bc2(-SHIFT));
    const float2 rh = __ffma2_rn(k, bc2(-LN2_HI), x);
    const float2 rl = __fmul2_rn(k, bc2(-LN2_LO));
    float2 q = __ffma2_rn(bc2(2.48015873e-05f), rh, bc2(1.98412698e-4f));
    q = __ffma2_rn(q, rh, bc2(1.38888889e-3f));
    q = __ffma2_rn(q, rh, bc2(8.33333333e-3f));
    q = __ffma2_rn(q, rh, bc2(4.16666667e-2f));
    q = __ffma2_rn(q, rh, bc2(1.66666667e-1f));
    q = __ffma2_rn(q, rh, bc2(0.5f));
    const float2 hi = __fadd2_rn(one, rh);
    const float2 omh = __ffma2_rn(hi, make_float2(-one.x, -one.y), one);  // 1 - hi, rounded once
    const float2 lo = __fadd2_rn(omh, rh);
    const float2 s = __fmul2_rn(rh, rh);
    float2 tail = __ffma2_rn(s, q, lo);
    const float2 ea = __fadd2_rn(hi, tail);
    tail = __ffma2_rn(rl, ea, tail);
    const float2 p = __fadd2_rn(hi, tail);
    const float2 scale = make_float2(__int_as_float((__float_as_int(j.x) - 0x4B3FFF81) << 23),
                                     __int_as_float((__float_as_int(j.y) - 0x4B3FFF81) << 23));
    return __fmul2_rn(p, scale);
}

// e^x for x in [-8, 0] from the special-function unit's base-2 exponential
// (PTX ex2.approx.ftz.f32) of x * log2(e): one multiply and one SFU
// instruction, within a few ulp (relative error below 1e-6 on that range,
// checked against expf_fast_nonpos by a GPU test). For values that only need
// to be close, never for a decision that must match the forward pass.
__device__ __forceinline__ float exp_sfu_nonpos(float x) {
    const float y = x * 1.44269504f;
    float r;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(y));
    return r;
}

// Relative half-width of the band around a threshold inside which an alpha
// formed with exp_sfu_nonpos cannot decide which side the forward's exact
// alpha lies on (4x the tested error bound of exp_sfu_nonpos).
constexpr float SFU_BAND = 4e-6f;

// Rust f32::max / f32::min ignore a NaN operand (fmaxf/fminf do the same);
// f32::clamp propagates NaN.
__device__ __forceinline__ float rclamp(float x, float lo, float hi) {
    if (x < lo) x = lo;
    if (x > hi) x = hi;
    return x;
}

// Rust `f as i32`: truncate toward zero, saturate, NaN -> 0.
__device__ __forceinline__ int as_i32(float f) {
    if (f != f) return 0;
    if (f >= 2147483647.0f) return 2147483647;
    if (f <= -2147483648.0f) return (int)0x80000000;
    return (int)f;
}

__device__ __forceinline__ float sigmoid(float x) { return 1.0f / (1.0f + exp_cr(-x)); }
__device__ __forceinline__ float logit(float p) { return log_cr(p / (1.0f - p)); }

struct M3 {
    float m[3][3];
};

__device__ __forceinline__ M3 mul(const M3& a, const M3& b) {
    M3 c;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) c.m[i][j] = (a.m[i][0] * b.m[0][j] + a.m[i][1] * b.m[1][j]) + a.m[i][2] * b.m[2][j];
    return c;
}
__device__ __forceinline__ M3 tr(const M3& a) {
    M3 c;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) c.m[i][j] = a.m[j][i];
    return c;
}

// quaternion.rs:10-17 followed by quaternion.rs:23-30.
__device__ __forceinline__ void qnormalize(const float q[4], float o[4]) {
    float n = sqrtf(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
    if (n < 1e-12f) { o[0] = 1.0f; o[1] = 0.0f; o[2] = 0.0f; o[3] = 0.0f; }
    else { o[0] = q[0] / n; o[1] = q[1] / n; o[2] = q[2] / n; o[3] = q[3] / n; }
}
__device__ __forceinline__ M3 mat_from_quat(const float q[4]) {
    float w = q[0], x = q[1], y = q[2], z = q[3];
    M3 r;
    r.m[0][0] = 1.0f - 2.0f * (y * y + z * z); r.m[0][1] = 2.0f * (x * y - w * z); r.m[0][2] = 2.0f * (x * z + w * y);
    r.m[1][0] = 2.0f * (x * y + w * z); r.m[1][1] = 1.0f - 2.0f * (x * x + z * z); r.m[1][2] = 2.0f * (y * z - w * x);
    r.m[2][0] = 2.0f * (x * z - w * y); r.m[2][1] = 2.0f * (y * z + w * x); r.m[2][2] = 1.0f - 2.0f * (x * x + y * y);
    return r;
}
__device__ __forceinline__ M3 to_rotation_matrix(const float q[4]) {
    float n[4];
    qnormalize(q, n);
    return mat_from_quat(n);
}
// covariance.rs:16-31: M = R diag(s), Sigma = M M^T.
__device__ __forceinline__ M3 rs_matrix(const float s[3], const float q[4]) {
    M3 r = to_rotation_matrix(q), o;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) o.m[i][j] = r.m[i][j] * s[j];
    return o;
}
__device__ __forceinline__ M3 build_cov3d(const float s[3], const float q[4]) {
    M3 m = rs_matrix(s, q);
    return mul(m, tr(m));
}

// Constants of src/math/sh.rs:9-32, parsed straight to f32 as Rust does.
#define SH_C0 0.28209479177387814f
#define SH_C1 0.4886025119029199f
#define SH_C2_0 1.0925484305920792f
#define SH_C2_1 -1.0925484305920792f
#define SH_C2_2 0.31539156525252005f
#define SH_C2_3 -1.0925484305920792f
#define SH_C2_4 0.5462742152960396f
#define SH_C3_0 -0.5900435899266435f
#define SH_C3_1 2.890611442640554f
#define SH_C3_2 -0.4570457994644658f
#define SH_C3_3 0.3731763325901154f
#define SH_C3_4 -0.4570457994644658f
#define SH_C3_5 1.445305721320277f
#define SH_C3_6 -0.5900435899266435f

// sh.rs:39-61
__device__ __forceinline__ void sh_basis(const float d[3], float b[16]) {
    float x = d[0], y = d[1], z = d[2];
    float xx = x * x, yy = y * y, zz = z * z, xy = x * y, xz = x * z, yz = y * z;
    b[0] = SH_C0;
    b[1] = SH_C1 * -y;
    b[2] = SH_C1 * z;
    b[3] = SH_C1 * -x;
    b[4] = SH_C2_0 * xy;
    b[5] = SH_C2_1 * yz;
    b[6] = SH_C2_2 * (2.0f * zz - xx - yy);
    b[7] = SH_C2_3 * xz;
    b[8] = SH_C2_4 * (xx - yy);
    b[9] = SH_C3_0 * y * (3.0f * xx - yy);
    b[10] = SH_C3_1 * xy * z;
    b[11] = SH_C3_2 * y * (4.0f * zz - xx - yy);
    b[12] = SH_C3_3 * z * (2.0f * zz - 3.0f * xx - 3.0f * yy);
    b[13] = SH_C3_4 * x * (4.0f * zz - xx - yy);
    b[14] = SH_C3_5 * z * (xx - yy);
    b[15] = SH_C3_6 * x * (xx - 3.0f * yy);
}

// sh.rs:122-139: normalize(cam - pos), [0,0,1] when shorter than 1e-8.
__device__ __forceinline__ void view_dir(const float gp[3], const float cp[3], float d[3]) {
    float v0 = cp[0] - gp[0], v1 = cp[1] - gp[1], v2 = cp[2] - gp[2];
    float len = sqrtf(v0 * v0 + v1 * v1 + v2 * v2);
    if (len < 1e-8f) { d[0] = 0.0f; d[1] = 0.0f; d[2] = 1.0f; }
    else { d[0] = v0 / len; d[1] = v1 / len; d[2] = v2 / len; }
}

}  // namespace rgs

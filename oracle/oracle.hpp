// oracle/oracle.hpp -- CPU restatement of rgsplat's differentiable training path.
//
// TEST INFRASTRUCTURE ONLY. This is the checker for the CUDA kernels in
// rgsplat_b200/csrc and the timed CPU baseline of bench.py. Nothing in the
// product links or calls it.
//
// It restates, function by function, the reference Rust crate (rgsplat 0.1.0):
//   src/math/mod.rs         Gaussian3D decoders, Camera::view_matrix, sigmoid/logit
//   src/math/quaternion.rs  normalize, mat_from_quat_components, rotation_jacobian
//   src/math/covariance.rs  rs_matrix, build_cov3d, backprop_cov3d
//   src/math/sh.rs          SH constants, sh_basis, sh_basis_grad, eval_sh_raw
//   src/math/projection.rs  project_covariance, gaussian_aabb_2d
//   src/cpu/backward.rs     project, project_and_bin, forward_pass, backward_pass,
//                           geometry_backprop, photometric_loss_grad, ssim, blur
//   src/pipeline/optimizer.rs  adam_step, densify_and_prune, reset_opacities
//   src/gpu/splat.wgsl + src/gpu/compute.rs + src/gpu/sort.rs  (WGSL projection,
//                           CPU composite) for the GpuRenderer drop-in.
// Templated on the scalar: float is the parity oracle and CPU baseline, double
// is the FP64 oracle used for finite-difference checks.
//
// Deliberate, documented deviations from the Rust source:
//  * Depth sort: `sort_unstable_by(depth)` (backward.rs:191) leaves ties
//    unspecified; the oracle breaks ties by Gaussian index (stable sort of an
//    index-ordered list), i.e. (tile, depth bits, index) order.
//  * exp/log: fmath.hpp (shared IEEE operation sequence with the kernels)
//    instead of libm; `orc_set_libm_math(1)` switches back to libm.
//  * Camera::view_matrix (mod.rs:155-160) inverts c2w in f32 via nalgebra; the
//    oracle inverts in double and rounds to float (same as the CUDA host code).
//  * Gaussian3D::covariance_3d (mod.rs:89-96) goes through nalgebra's
//    UnitQuaternion; the oracle uses quaternion::to_rotation_matrix (normalise,
//    then quaternion.rs:23-30), which is the same rotation up to rounding.
#pragma once
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <vector>

#include "fmath.hpp"

namespace orc {

// ---------------------------------------------------------------------------
// literals: Rust parses `0.99` straight to f32; so does `0.99f` in C++. A
// double literal cast to float could round twice, so pick per type.
// ---------------------------------------------------------------------------
template <class T> struct Lit;
template <> struct Lit<float> { static float v(float f, double) { return f; } };
template <> struct Lit<double> { static double v(float, double d) { return d; } };
#define LIT(x) (Lit<T>::v(x##f, x))

extern int g_libm_math;  // 0: fmath.hpp (default), 1: libm

// Per-Gaussian transcendentals (correctly rounded in practice).
inline float t_exp(float x) { return g_libm_math ? std::exp(x) : fm::exp_cr(x); }
inline double t_exp(double x) { return std::exp(x); }
inline float t_log(float x) { return g_libm_math ? std::log(x) : fm::log_cr(x); }
inline double t_log(double x) { return std::log(x); }
// Per (pixel, splat) alpha = opacity * exp(power).
inline float t_expa(float x) { return g_libm_math ? std::exp(x) : fm::expf_fast(x); }
inline double t_expa(double x) { return std::exp(x); }

// Rust f32::max / f32::min ignore a NaN operand; f32::clamp propagates NaN.
template <class T> inline T rmax(T a, T b) { if (a != a) return b; if (b != b) return a; return a > b ? a : b; }
template <class T> inline T rmin(T a, T b) { if (a != a) return b; if (b != b) return a; return a < b ? a : b; }
template <class T> inline T rclamp(T x, T lo, T hi) { if (x < lo) x = lo; if (x > hi) x = hi; return x; }
// Rust `f as i32`: truncate toward zero, saturate, NaN -> 0 (projection.rs:159-162).
template <class T> inline int32_t as_i32(T f) {
    if (f != f) return 0;
    if (f >= T(2147483647.0)) return INT32_MAX;
    if (f <= T(-2147483648.0)) return INT32_MIN;
    return (int32_t)f;
}
inline int32_t wrap_add(int32_t a, int32_t b) { return (int32_t)((uint32_t)a + (uint32_t)b); }
// Rust `f as i64`: truncate, saturate, NaN -> 0.
template <class T> inline int64_t as_i64(T f) {
    if (f != f) return 0;
    if (f >= T(9223372036854775807.0)) return INT64_MAX;
    if (f <= T(-9223372036854775808.0)) return INT64_MIN;
    return (int64_t)f;
}

constexpr int TILE_SIZE = 16;
constexpr int NP = 59;  // trainable floats per Gaussian (optimizer.rs:71)
constexpr int NG = 60;  // GaussianGrad floats (backward.rs:33-41)

template <class T> struct Gaussian {
    T position[3];
    T opacity_logit;
    T rotation[4];
    T log_scale[3];
    T sh[48];
};
static_assert(sizeof(Gaussian<float>) == 236, "Gaussian3D is 59 f32");

template <class T> struct Grad {
    T d_position[3];
    T d_rotation[4];
    T d_log_scale[3];
    T d_opacity_logit;
    T d_sh[48];
    T screen_grad_norm;
};
static_assert(sizeof(Grad<float>) == 240, "GaussianGrad is 60 f32");

struct CameraIn {  // mirrors Camera (mod.rs:131-145); c2w row-major
    uint32_t width, height;
    float fx, fy, cx, cy;
    float c2w[16];
    float distortion[3];
};

template <class T> struct Cam {
    int w, h;
    T fx, fy, cx, cy;
    T view[4][4];
    T pos[3];
};

// General 4x4 inverse (cofactors) in double.
inline bool invert4(const double m[16], double out[16]) {
    double inv[16];
    inv[0] = m[5] * m[10] * m[15] - m[5] * m[11] * m[14] - m[9] * m[6] * m[15] + m[9] * m[7] * m[14] + m[13] * m[6] * m[11] - m[13] * m[7] * m[10];
    inv[4] = -m[4] * m[10] * m[15] + m[4] * m[11] * m[14] + m[8] * m[6] * m[15] - m[8] * m[7] * m[14] - m[12] * m[6] * m[11] + m[12] * m[7] * m[10];
    inv[8] = m[4] * m[9] * m[15] - m[4] * m[11] * m[13] - m[8] * m[5] * m[15] + m[8] * m[7] * m[13] + m[12] * m[5] * m[11] - m[12] * m[7] * m[9];
    inv[12] = -m[4] * m[9] * m[14] + m[4] * m[10] * m[13] + m[8] * m[5] * m[14] - m[8] * m[6] * m[13] - m[12] * m[5] * m[10] + m[12] * m[6] * m[9];
    inv[1] = -m[1] * m[10] * m[15] + m[1] * m[11] * m[14] + m[9] * m[2] * m[15] - m[9] * m[3] * m[14] - m[13] * m[2] * m[11] + m[13] * m[3] * m[10];
    inv[5] = m[0] * m[10] * m[15] - m[0] * m[11] * m[14] - m[8] * m[2] * m[15] + m[8] * m[3] * m[14] + m[12] * m[2] * m[11] - m[12] * m[3] * m[10];
    inv[9] = -m[0] * m[9] * m[15] + m[0] * m[11] * m[13] + m[8] * m[1] * m[15] - m[8] * m[3] * m[13] - m[12] * m[1] * m[11] + m[12] * m[3] * m[9];
    inv[13] = m[0] * m[9] * m[14] - m[0] * m[10] * m[13] - m[8] * m[1] * m[14] + m[8] * m[2] * m[13] + m[12] * m[1] * m[10] - m[12] * m[2] * m[9];
    inv[2] = m[1] * m[6] * m[15] - m[1] * m[7] * m[14] - m[5] * m[2] * m[15] + m[5] * m[3] * m[14] + m[13] * m[2] * m[7] - m[13] * m[3] * m[6];
    inv[6] = -m[0] * m[6] * m[15] + m[0] * m[7] * m[14] + m[4] * m[2] * m[15] - m[4] * m[3] * m[14] - m[12] * m[2] * m[7] + m[12] * m[3] * m[6];
    inv[10] = m[0] * m[5] * m[15] - m[0] * m[7] * m[13] - m[4] * m[1] * m[15] + m[4] * m[3] * m[13] + m[12] * m[1] * m[7] - m[12] * m[3] * m[5];
    inv[14] = -m[0] * m[5] * m[14] + m[0] * m[6] * m[13] + m[4] * m[1] * m[14] - m[4] * m[2] * m[13] - m[12] * m[1] * m[6] + m[12] * m[2] * m[5];
    inv[3] = -m[1] * m[6] * m[11] + m[1] * m[7] * m[10] + m[5] * m[2] * m[11] - m[5] * m[3] * m[10] - m[9] * m[2] * m[7] + m[9] * m[3] * m[6];
    inv[7] = m[0] * m[6] * m[11] - m[0] * m[7] * m[10] - m[4] * m[2] * m[11] + m[4] * m[3] * m[10] + m[8] * m[2] * m[7] - m[8] * m[3] * m[6];
    inv[11] = -m[0] * m[5] * m[11] + m[0] * m[7] * m[9] + m[4] * m[1] * m[11] - m[4] * m[3] * m[9] - m[8] * m[1] * m[7] + m[8] * m[3] * m[5];
    inv[15] = m[0] * m[5] * m[10] - m[0] * m[6] * m[9] - m[4] * m[1] * m[10] + m[4] * m[2] * m[9] + m[8] * m[1] * m[6] - m[8] * m[2] * m[5];
    double det = m[0] * inv[0] + m[1] * inv[4] + m[2] * inv[8] + m[3] * inv[12];
    if (det == 0.0 || det != det) return false;
    double id = 1.0 / det;
    for (int i = 0; i < 16; ++i) out[i] = inv[i] * id;
    return true;
}

// Camera::view_matrix (mod.rs:155-160) and Camera::position (mod.rs:163-165).
template <class T> inline bool make_cam(const CameraIn& c, Cam<T>& o) {
    double m[16], inv[16];
    for (int i = 0; i < 16; ++i) m[i] = (double)c.c2w[i];
    if (!invert4(m, inv)) return false;
    o.w = (int)c.width; o.h = (int)c.height;
    o.fx = (T)c.fx; o.fy = (T)c.fy; o.cx = (T)c.cx; o.cy = (T)c.cy;
    for (int r = 0; r < 4; ++r)
        for (int k = 0; k < 4; ++k) o.view[r][k] = (T)inv[r * 4 + k];
    o.pos[0] = (T)c.c2w[3]; o.pos[1] = (T)c.c2w[7]; o.pos[2] = (T)c.c2w[11];
    return true;
}

// ---------------------------------------------------------------------------
// math primitives
// ---------------------------------------------------------------------------
template <class T> inline T sigmoid(T x) { return T(1) / (T(1) + t_exp(-x)); }   // mod.rs:183-185
template <class T> inline T logit(T p) { return t_log(p / (T(1) - p)); }          // mod.rs:189-192

template <class T> struct M3 { T m[3][3]; };

template <class T> inline M3<T> mul(const M3<T>& a, const M3<T>& b) {
    M3<T> c;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) c.m[i][j] = (a.m[i][0] * b.m[0][j] + a.m[i][1] * b.m[1][j]) + a.m[i][2] * b.m[2][j];
    return c;
}
template <class T> inline M3<T> tr(const M3<T>& a) {
    M3<T> c;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) c.m[i][j] = a.m[j][i];
    return c;
}

// quaternion.rs:10-17
template <class T> inline void qnormalize(const T q[4], T o[4]) {
    T n = std::sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
    if (n < LIT(1e-12)) { o[0] = 1; o[1] = 0; o[2] = 0; o[3] = 0; }
    else { o[0] = q[0] / n; o[1] = q[1] / n; o[2] = q[2] / n; o[3] = q[3] / n; }
}
// quaternion.rs:23-30
template <class T> inline M3<T> mat_from_quat(const T q[4]) {
    T w = q[0], x = q[1], y = q[2], z = q[3];
    M3<T> r;
    r.m[0][0] = T(1) - T(2) * (y * y + z * z); r.m[0][1] = T(2) * (x * y - w * z); r.m[0][2] = T(2) * (x * z + w * y);
    r.m[1][0] = T(2) * (x * y + w * z); r.m[1][1] = T(1) - T(2) * (x * x + z * z); r.m[1][2] = T(2) * (y * z - w * x);
    r.m[2][0] = T(2) * (x * z - w * y); r.m[2][1] = T(2) * (y * z + w * x); r.m[2][2] = T(1) - T(2) * (x * x + y * y);
    return r;
}
template <class T> inline M3<T> to_rotation_matrix(const T q[4]) { T n[4]; qnormalize(q, n); return mat_from_quat(n); }

// quaternion.rs:45-70
template <class T> inline void rotation_jacobian(const T qin[4], M3<T> d[4]) {
    T q[4]; qnormalize(qin, q);
    T w = q[0], x = q[1], y = q[2], z = q[3];
    T Z = 0;
    d[0] = M3<T>{{{Z, T(-2) * z, T(2) * y}, {T(2) * z, Z, T(-2) * x}, {T(-2) * y, T(2) * x, Z}}};
    d[1] = M3<T>{{{Z, T(2) * y, T(2) * z}, {T(2) * y, T(-4) * x, T(-2) * w}, {T(2) * z, T(2) * w, T(-4) * x}}};
    d[2] = M3<T>{{{T(-4) * y, T(2) * x, T(2) * w}, {T(2) * x, Z, T(2) * z}, {T(-2) * w, T(2) * z, T(-4) * y}}};
    d[3] = M3<T>{{{T(-4) * z, T(-2) * w, T(2) * x}, {T(2) * w, T(-4) * z, T(2) * y}, {T(2) * x, T(2) * y, Z}}};
}

// covariance.rs:16-31 (rs_matrix / build_cov3d) and mod.rs:89-96.
template <class T> inline M3<T> rs_matrix(const T s[3], const T q[4]) {
    M3<T> r = to_rotation_matrix(q), o;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) o.m[i][j] = r.m[i][j] * s[j];
    return o;
}
template <class T> inline M3<T> build_cov3d(const T s[3], const T q[4]) {
    M3<T> m = rs_matrix(s, q);
    return mul(m, tr(m));
}
template <class T> inline void scale_of(const Gaussian<T>& g, T s[3]) {
    s[0] = t_exp(g.log_scale[0]); s[1] = t_exp(g.log_scale[1]); s[2] = t_exp(g.log_scale[2]);
}

// covariance.rs:42-84
template <class T> inline void backprop_cov3d(const T scale[3], const T rot[4], const M3<T>& g, T d_log_scale[3], T d_rot[4]) {
    M3<T> r = to_rotation_matrix(rot);
    M3<T> m = rs_matrix(scale, rot);
    M3<T> gs;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) gs.m[i][j] = g.m[i][j] + g.m[j][i];
    M3<T> dm = mul(gs, m);
    T ds[3];
    M3<T> dr;
    for (int j = 0; j < 3; ++j) {
        T acc = 0;
        for (int i = 0; i < 3; ++i) {
            acc += dm.m[i][j] * r.m[i][j];
            dr.m[i][j] = dm.m[i][j] * scale[j];
        }
        ds[j] = acc;
    }
    for (int j = 0; j < 3; ++j) d_log_scale[j] = ds[j] * scale[j];
    M3<T> jac[4];
    rotation_jacobian(rot, jac);
    for (int k = 0; k < 4; ++k) {
        T s = 0;  // nalgebra sums in column-major storage order
        for (int c = 0; c < 3; ++c)
            for (int rr = 0; rr < 3; ++rr) s += jac[k].m[rr][c] * dr.m[rr][c];
        d_rot[k] = s;
    }
}

// sh.rs:9-32
template <class T> struct SHC {
    static T C0() { return LIT(0.28209479177387814); }
    static T C1() { return LIT(0.4886025119029199); }
    static T C2(int i) {
        switch (i) {
            case 0: return LIT(1.0925484305920792);
            case 1: return LIT(-1.0925484305920792);
            case 2: return LIT(0.31539156525252005);
            case 3: return LIT(-1.0925484305920792);
            default: return LIT(0.5462742152960396);
        }
    }
    static T C3(int i) {
        switch (i) {
            case 0: return LIT(-0.5900435899266435);
            case 1: return LIT(2.890611442640554);
            case 2: return LIT(-0.4570457994644658);
            case 3: return LIT(0.3731763325901154);
            case 4: return LIT(-0.4570457994644658);
            case 5: return LIT(1.445305721320277);
            default: return LIT(-0.5900435899266435);
        }
    }
};

// sh.rs:39-61
template <class T> inline void sh_basis(const T d[3], T b[16]) {
    typedef SHC<T> S;
    T x = d[0], y = d[1], z = d[2];
    T xx = x * x, yy = y * y, zz = z * z, xy = x * y, xz = x * z, yz = y * z;
    b[0] = S::C0();
    b[1] = S::C1() * -y;
    b[2] = S::C1() * z;
    b[3] = S::C1() * -x;
    b[4] = S::C2(0) * xy;
    b[5] = S::C2(1) * yz;
    b[6] = S::C2(2) * (T(2) * zz - xx - yy);
    b[7] = S::C2(3) * xz;
    b[8] = S::C2(4) * (xx - yy);
    b[9] = S::C3(0) * y * (T(3) * xx - yy);
    b[10] = S::C3(1) * xy * z;
    b[11] = S::C3(2) * y * (T(4) * zz - xx - yy);
    b[12] = S::C3(3) * z * (T(2) * zz - T(3) * xx - T(3) * yy);
    b[13] = S::C3(4) * x * (T(4) * zz - xx - yy);
    b[14] = S::C3(5) * z * (xx - yy);
    b[15] = S::C3(6) * x * (xx - T(3) * yy);
}

// sh.rs:68-89
template <class T> inline void sh_basis_grad(const T d[3], T g[16][3]) {
    typedef SHC<T> S;
    T x = d[0], y = d[1], z = d[2];
    T xx = x * x, yy = y * y, zz = z * z;
    T Z = 0;
    T t[16][3] = {
        {Z, Z, Z},
        {Z, -S::C1(), Z},
        {Z, Z, S::C1()},
        {-S::C1(), Z, Z},
        {S::C2(0) * y, S::C2(0) * x, Z},
        {Z, S::C2(1) * z, S::C2(1) * y},
        {S::C2(2) * T(-2) * x, S::C2(2) * T(-2) * y, S::C2(2) * T(4) * z},
        {S::C2(3) * z, Z, S::C2(3) * x},
        {S::C2(4) * T(2) * x, S::C2(4) * T(-2) * y, Z},
        {S::C3(0) * T(6) * x * y, S::C3(0) * T(3) * (xx - yy), Z},
        {S::C3(1) * y * z, S::C3(1) * x * z, S::C3(1) * x * y},
        {S::C3(2) * T(-2) * x * y, S::C3(2) * (T(4) * zz - xx - T(3) * yy), S::C3(2) * T(8) * y * z},
        {S::C3(3) * T(-6) * x * z, S::C3(3) * T(-6) * y * z, S::C3(3) * (T(6) * zz - T(3) * xx - T(3) * yy)},
        {S::C3(4) * (T(4) * zz - T(3) * xx - yy), S::C3(4) * T(-2) * x * y, S::C3(4) * T(8) * x * z},
        {S::C3(5) * T(2) * x * z, S::C3(5) * T(-2) * y * z, S::C3(5) * (xx - yy)},
        {S::C3(6) * T(3) * (xx - yy), S::C3(6) * T(-6) * x * y, Z},
    };
    std::memcpy(g, t, sizeof(t));
}

// sh.rs:93-104
template <class T> inline void eval_sh_raw(const T* c, const T b[16], T out[3]) {
    for (int ch = 0; ch < 3; ++ch) {
        T acc = 0;
        for (int k = 0; k < 16; ++k) acc += b[k] * c[ch * 16 + k];
        out[ch] = T(0.5) + acc;
    }
}
// sh.rs:122-139
template <class T> inline void view_dir(const T gp[3], const T cp[3], T d[3]) {
    T v[3] = {cp[0] - gp[0], cp[1] - gp[1], cp[2] - gp[2]};
    T len = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    if (len < LIT(1e-8)) { d[0] = 0; d[1] = 0; d[2] = 1; }
    else { d[0] = v[0] / len; d[1] = v[1] / len; d[2] = v[2] / len; }
}

template <class T> inline void view_mul(const Cam<T>& c, const T p[3], T o[3]) {
    for (int i = 0; i < 3; ++i)
        o[i] = ((c.view[i][0] * p[0] + c.view[i][1] * p[1]) + c.view[i][2] * p[2]) + c.view[i][3] * T(1);
}
template <class T> inline M3<T> view3(const Cam<T>& c) {
    M3<T> w;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) w.m[i][j] = c.view[i][j];
    return w;
}

// projection.rs:24-69 -> (a, b, c) of the low-passed 2D covariance.
template <class T> inline void project_covariance(const M3<T>& sig, const T pos[3], const Cam<T>& cam, T abc[3]) {
    T pc[3]; view_mul(cam, pos, pc);
    T tx = pc[0], ty = pc[1], tz = rmax(pc[2], LIT(0.001));
    T fx = cam.fx, fy = cam.fy, Z = 0;
    M3<T> j = {{{fx / tz, Z, -fx * tx / (tz * tz)}, {Z, fy / tz, -fy * ty / (tz * tz)}, {Z, Z, Z}}};
    M3<T> t = mul(j, view3(cam));
    M3<T> s2 = mul(mul(t, sig), tr(t));
    abc[0] = s2.m[0][0] + LIT(0.3);
    abc[1] = s2.m[0][1];
    abc[2] = s2.m[1][1] + LIT(0.3);
}

// projection.rs:138-165 with n_sigma = 3 (the only caller, backward.rs:261).
template <class T> inline bool aabb_2d(T mx, T my, const T abc[3], int w, int h, int32_t box[4]) {
    T a = abc[0], b = abc[1], c = abc[2];
    T mid = (a + c) * T(0.5);
    T disc = std::sqrt((a - c) * (a - c) * T(0.25) + b * b);
    T l1 = rmax(mid + disc, T(0));
    T l2 = rmax(mid - disc, T(0));
    T r = T(3) * rmax(std::sqrt(l1), std::sqrt(l2));
    int32_t x0 = std::max(as_i32(mx - r), 0);
    int32_t y0 = std::max(as_i32(my - r), 0);
    int32_t x1 = std::min(wrap_add(as_i32(mx + r), 1), (int32_t)w);
    int32_t y1 = std::min(wrap_add(as_i32(my + r), 1), (int32_t)h);
    if (x0 >= x1 || y0 >= y1) return false;
    box[0] = x0; box[1] = y0; box[2] = x1; box[3] = y1;
    return true;
}

// backward.rs:74-90
template <class T> struct Splat {
    int gi;
    T sx, sy;
    T conic[3];
    T cov2d[3];
    T color[3];
    T raw_color[3];
    T opacity;
    T depth;
    T basis[16];
    T pcam[3];
    int32_t tx0, ty0, tx1, ty1;
};

template <class T> struct Consts {
    static T alpha_threshold() { return T(1) / T(255); }
    static T transmittance_stop() { return LIT(1e-4); }
    static T max_alpha() { return LIT(0.99); }
};

// backward.rs:210-280
template <class T> inline bool project(const Gaussian<T>& g, int gi, const Cam<T>& cam, Splat<T>& s) {
    T opacity = sigmoid(g.opacity_logit);
    if (opacity < Consts<T>::alpha_threshold()) return false;
    T pc[3]; view_mul(cam, g.position, pc);
    T tz = pc[2];
    if (tz <= LIT(0.001)) return false;
    T sx = cam.fx * pc[0] / tz + cam.cx;
    T sy = cam.fy * pc[1] / tz + cam.cy;
    T margin = T(128);
    if (sx < -margin || sx > (T)cam.w + margin || sy < -margin || sy > (T)cam.h + margin) return false;
    T sc[3]; scale_of(g, sc);
    M3<T> sig = build_cov3d(sc, g.rotation);
    T abc[3]; project_covariance(sig, g.position, cam, abc);
    T a = abc[0], b = abc[1], c = abc[2];
    T det = a * c - b * b;
    if (std::fabs(det) < LIT(1e-8)) return false;
    T inv_det = T(1) / det;
    T d[3]; view_dir(g.position, cam.pos, d);
    sh_basis(d, s.basis);
    eval_sh_raw(g.sh, s.basis, s.raw_color);
    int32_t box[4];
    if (!aabb_2d(sx, sy, abc, cam.w, cam.h, box)) return false;
    s.gi = gi; s.sx = sx; s.sy = sy;
    s.conic[0] = c * inv_det; s.conic[1] = -b * inv_det; s.conic[2] = a * inv_det;
    s.cov2d[0] = a; s.cov2d[1] = b; s.cov2d[2] = c;
    for (int ch = 0; ch < 3; ++ch) s.color[ch] = rclamp(s.raw_color[ch], T(0), T(1));
    s.opacity = opacity;
    s.depth = tz;
    s.pcam[0] = pc[0]; s.pcam[1] = pc[1]; s.pcam[2] = pc[2];
    s.tx0 = box[0] / TILE_SIZE; s.ty0 = box[1] / TILE_SIZE;
    s.tx1 = (box[2] + TILE_SIZE - 1) / TILE_SIZE; s.ty1 = (box[3] + TILE_SIZE - 1) / TILE_SIZE;
    return true;
}

enum { ORC_OK = 0, ORC_EINVAL = -1, ORC_ENAN = -2, ORC_ESIZE = -3 };

template <class T> struct Binned {
    std::vector<Splat<T>> splats;            // depth-sorted
    std::vector<std::vector<int>> tile_lists;  // indices into splats
    int ntx = 0, nty = 0;
};

// backward.rs:172-208
template <class T> inline int project_and_bin(const Gaussian<T>* gs, size_t n, const Cam<T>& cam, Binned<T>& out) {
    int w = cam.w, h = cam.h;
    out.ntx = (w + TILE_SIZE - 1) / TILE_SIZE;
    out.nty = (h + TILE_SIZE - 1) / TILE_SIZE;
    std::vector<Splat<T>> all(n);
    std::vector<char> vis(n, 0);
#pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)n; ++i) vis[i] = project(gs[i], (int)i, cam, all[i]) ? 1 : 0;
    out.splats.clear();
    for (size_t i = 0; i < n; ++i)
        if (vis[i]) out.splats.push_back(all[i]);
    for (auto& s : out.splats)
        if (s.depth != s.depth) return ORC_ENAN;  // the reference panics here (backward.rs:191)
    std::stable_sort(out.splats.begin(), out.splats.end(), [](const Splat<T>& a, const Splat<T>& b) { return a.depth < b.depth; });
    out.tile_lists.assign((size_t)out.ntx * out.nty, std::vector<int>());
    for (size_t idx = 0; idx < out.splats.size(); ++idx) {
        const Splat<T>& s = out.splats[idx];
        int tx0 = std::max(s.tx0, 0), ty0 = std::max(s.ty0, 0);
        int tx1 = std::min(s.tx1, out.ntx), ty1 = std::min(s.ty1, out.nty);
        for (int ty = ty0; ty < ty1; ++ty)
            for (int tx = tx0; tx < tx1; ++tx) out.tile_lists[(size_t)ty * out.ntx + tx].push_back((int)idx);
    }
    return ORC_OK;
}

// backward.rs:296-385
template <class T> inline void forward_pass(const Binned<T>& B, int w, int h, const T bg[3], T* rendered, T* final_t, int32_t* last_contrib) {
    const T ATH = Consts<T>::alpha_threshold(), TST = Consts<T>::transmittance_stop(), MA = Consts<T>::max_alpha();
    for (long p = 0; p < (long)w * h; ++p) {
        rendered[p * 3] = 0; rendered[p * 3 + 1] = 0; rendered[p * 3 + 2] = 0;
        final_t[p] = 1; last_contrib[p] = -1;
    }
#pragma omp parallel for schedule(dynamic, 4)
    for (long ti = 0; ti < (long)B.tile_lists.size(); ++ti) {
        const std::vector<int>& L = B.tile_lists[ti];
        if (L.empty()) continue;
        int tx = (int)(ti % B.ntx), ty = (int)(ti / B.ntx);
        int px0 = tx * TILE_SIZE, py0 = ty * TILE_SIZE;
        int px1 = std::min(px0 + TILE_SIZE, w), py1 = std::min(py0 + TILE_SIZE, h);
        for (int py = py0; py < py1; ++py)
            for (int px = px0; px < px1; ++px) {
                T t = 1, col[3] = {0, 0, 0};
                int32_t last = -1;
                for (size_t li = 0; li < L.size(); ++li) {
                    const Splat<T>& s = B.splats[L[li]];
                    T dx = (T)px + T(0.5) - s.sx;
                    T dy = (T)py + T(0.5) - s.sy;
                    T a = s.conic[0], b = s.conic[1], c = s.conic[2];
                    T power = T(-0.5) * (a * dx * dx + T(2) * b * dx * dy + c * dy * dy);
                    if (power > T(0)) continue;
                    T alpha = rmin(s.opacity * t_expa(power), MA);
                    if (alpha < ATH) continue;
                    T weight = alpha * t;
                    col[0] += s.color[0] * weight;
                    col[1] += s.color[1] * weight;
                    col[2] += s.color[2] * weight;
                    t *= T(1) - alpha;
                    last = (int32_t)li;
                    if (t < TST) break;
                }
                long pix = (long)py * w + px;
                rendered[pix * 3] = col[0] + t * bg[0];
                rendered[pix * 3 + 1] = col[1] + t * bg[1];
                rendered[pix * 3 + 2] = col[2] + t * bg[2];
                final_t[pix] = t;
                last_contrib[pix] = last;
            }
    }
}

template <class T> struct Acc {  // backward.rs:92-99
    T color[3];
    T opacity;
    T conic[3];
    T sx, sy;
};

// backward.rs:391-512
template <class T> inline void backward_pass(const Binned<T>& B, int w, int h, const T bg[3], const T* final_t, const int32_t* last_contrib, const T* dl_dpix, std::vector<Acc<T>>& merged) {
    const T ATH = Consts<T>::alpha_threshold(), MA = Consts<T>::max_alpha();
    size_t nt = B.tile_lists.size();
    std::vector<std::vector<Acc<T>>> per_tile(nt);
#pragma omp parallel for schedule(dynamic, 4)
    for (long ti = 0; ti < (long)nt; ++ti) {
        const std::vector<int>& L = B.tile_lists[ti];
        if (L.empty()) continue;
        int tx = (int)(ti % B.ntx), ty = (int)(ti / B.ntx);
        int px0 = tx * TILE_SIZE, py0 = ty * TILE_SIZE;
        int px1 = std::min(px0 + TILE_SIZE, w), py1 = std::min(py0 + TILE_SIZE, h);
        std::vector<Acc<T>>& local = per_tile[ti];
        local.assign(L.size(), Acc<T>{{0, 0, 0}, 0, {0, 0, 0}, 0, 0});
        for (int py = py0; py < py1; ++py)
            for (int px = px0; px < px1; ++px) {
                long pix = (long)py * w + px;
                int32_t lc = last_contrib[pix];
                if (lc < 0) continue;
                T dl[3] = {dl_dpix[pix * 3], dl_dpix[pix * 3 + 1], dl_dpix[pix * 3 + 2]};
                T t = final_t[pix];
                T behind[3] = {t * bg[0], t * bg[1], t * bg[2]};
                for (long li = lc; li >= 0; --li) {
                    const Splat<T>& s = B.splats[L[li]];
                    T dx = (T)px + T(0.5) - s.sx;
                    T dy = (T)py + T(0.5) - s.sy;
                    T a = s.conic[0], b = s.conic[1], c = s.conic[2];
                    T power = T(-0.5) * (a * dx * dx + T(2) * b * dx * dy + c * dy * dy);
                    if (power > T(0)) continue;
                    T g_exp = t_expa(power);
                    T alpha_raw = s.opacity * g_exp;
                    T alpha = rmin(alpha_raw, MA);
                    if (alpha < ATH) continue;
                    t /= T(1) - alpha;
                    T weight = alpha * t;
                    Acc<T>& g = local[li];
                    g.color[0] += dl[0] * weight;
                    g.color[1] += dl[1] * weight;
                    g.color[2] += dl[2] * weight;
                    T inv_1ma = T(1) / (T(1) - alpha);
                    T dl_dalpha = 0;
                    for (int ch = 0; ch < 3; ++ch) dl_dalpha += dl[ch] * (t * s.color[ch] - behind[ch] * inv_1ma);
                    T dalpha_draw = alpha_raw > MA ? T(0) : T(1);
                    T dl_draw = dl_dalpha * dalpha_draw;
                    g.opacity += dl_draw * g_exp;
                    T dl_dpower = dl_draw * s.opacity * g_exp;
                    g.conic[0] += dl_dpower * (T(-0.5) * dx * dx);
                    g.conic[1] += dl_dpower * (-dx * dy);
                    g.conic[2] += dl_dpower * (T(-0.5) * dy * dy);
                    g.sx += dl_dpower * (a * dx + b * dy);
                    g.sy += dl_dpower * (b * dx + c * dy);
                    behind[0] += weight * s.color[0];
                    behind[1] += weight * s.color[1];
                    behind[2] += weight * s.color[2];
                }
            }
    }
    merged.assign(B.splats.size(), Acc<T>{{0, 0, 0}, 0, {0, 0, 0}, 0, 0});
    for (size_t ti = 0; ti < nt; ++ti) {
        const std::vector<int>& L = B.tile_lists[ti];
        const std::vector<Acc<T>>& local = per_tile[ti];
        for (size_t li = 0; li < local.size(); ++li) {
            Acc<T>& m = merged[L[li]];
            const Acc<T>& a = local[li];
            for (int ch = 0; ch < 3; ++ch) { m.color[ch] += a.color[ch]; m.conic[ch] += a.conic[ch]; }
            m.opacity += a.opacity;
            m.sx += a.sx;
            m.sy += a.sy;
        }
    }
}

// backward.rs:518-638
template <class T> inline void geometry_backprop(const Splat<T>& s, const Acc<T>& acc, const Gaussian<T>& g, const Cam<T>& cam, Grad<T>& out) {
    std::memset(&out, 0, sizeof(out));
    T op = s.opacity;
    out.d_opacity_logit = acc.opacity * op * (T(1) - op);
    T masked[3];
    for (int ch = 0; ch < 3; ++ch) masked[ch] = (s.raw_color[ch] > T(0) && s.raw_color[ch] < T(1)) ? acc.color[ch] : T(0);
    for (int ch = 0; ch < 3; ++ch)
        for (int k = 0; k < 16; ++k) out.d_sh[ch * 16 + k] = masked[ch] * s.basis[k];

    T ga = acc.conic[0], gb = acc.conic[1], gc = acc.conic[2];
    T a2 = s.cov2d[0], b2 = s.cov2d[1], c2 = s.cov2d[2];
    T det = a2 * c2 - b2 * b2;
    T det2 = det * det;
    T dl_da = (-ga * c2 * c2 + gb * b2 * c2 - gc * b2 * b2) / det2;
    T dl_db = (T(2) * ga * b2 * c2 - gb * (det + T(2) * b2 * b2) + T(2) * gc * a2 * b2) / det2;
    T dl_dc = (-ga * b2 * b2 + gb * a2 * b2 - gc * a2 * a2) / det2;

    T fx = cam.fx, fy = cam.fy, Z = 0;
    T tx = s.pcam[0], ty = s.pcam[1], tz = s.pcam[2];
    M3<T> V = view3(cam);
    M3<T> j = {{{fx / tz, Z, -fx * tx / (tz * tz)}, {Z, fy / tz, -fy * ty / (tz * tz)}, {Z, Z, Z}}};
    M3<T> t_mat = mul(j, V);
    T sc[3]; scale_of(g, sc);
    M3<T> sigma3d = build_cov3d(sc, g.rotation);
    M3<T> gcov = {{{dl_da, T(0.5) * dl_db, Z}, {T(0.5) * dl_db, dl_dc, Z}, {Z, Z, Z}}};
    M3<T> dsig = mul(mul(tr(t_mat), gcov), t_mat);
    backprop_cov3d(sc, g.rotation, dsig, out.d_log_scale, out.d_rotation);

    T dp[3] = {acc.sx * fx / tz, acc.sy * fy / tz, acc.sx * (-fx * tx / (tz * tz)) + acc.sy * (-fy * ty / (tz * tz))};
    M3<T> dj[3] = {
        {{{Z, Z, -fx / (tz * tz)}, {Z, Z, Z}, {Z, Z, Z}}},
        {{{Z, Z, Z}, {Z, Z, -fy / (tz * tz)}, {Z, Z, Z}}},
        {{{-fx / (tz * tz), Z, T(2) * fx * tx / (tz * tz * tz)}, {Z, -fy / (tz * tz), T(2) * fy * ty / (tz * tz * tz)}, {Z, Z, Z}}},
    };
    M3<T> sig_tt = mul(sigma3d, tr(t_mat));
    M3<T> ts = mul(t_mat, sigma3d);
    for (int k = 0; k < 3; ++k) {
        M3<T> dt = mul(dj[k], V);
        M3<T> p1 = mul(dt, sig_tt), p2 = mul(ts, tr(dt));
        T d00 = p1.m[0][0] + p2.m[0][0], d01 = p1.m[0][1] + p2.m[0][1], d11 = p1.m[1][1] + p2.m[1][1];
        T contrib = dl_da * d00 + dl_db * d01 + dl_dc * d11;
        dp[k] += contrib;
    }
    T dpos[3];
    for (int i = 0; i < 3; ++i) dpos[i] = (V.m[0][i] * dp[0] + V.m[1][i] * dp[1]) + V.m[2][i] * dp[2];

    T u[3] = {cam.pos[0] - g.position[0], cam.pos[1] - g.position[1], cam.pos[2] - g.position[2]};
    T len = std::sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
    if (len > LIT(1e-8)) {
        T dir[3] = {u[0] / len, u[1] / len, u[2] / len};
        T db[16][3];
        sh_basis_grad(dir, db);
        T dd[3] = {0, 0, 0};
        for (int k = 0; k < 16; ++k) {
            T dbk = masked[0] * g.sh[k] + masked[1] * g.sh[16 + k] + masked[2] * g.sh[32 + k];
            for (int i = 0; i < 3; ++i) dd[i] += dbk * db[k][i];
        }
        T dot = dir[0] * dd[0] + dir[1] * dd[1] + dir[2] * dd[2];
        for (int i = 0; i < 3; ++i) {
            T proj = dd[i] - dir[i] * dot;
            dpos[i] += -(proj / len);
        }
    }
    for (int i = 0; i < 3; ++i) out.d_position[i] = dpos[i];
    out.screen_grad_norm = std::sqrt(acc.sx * acc.sx + acc.sy * acc.sy);
}

// backward.rs:759-772
template <class T> inline std::vector<T> gaussian_kernel_1d(int radius, T sigma) {
    std::vector<T> k(2 * radius + 1);
    T sum = 0;
    for (size_t i = 0; i < k.size(); ++i) {
        T d = (T)(int)i - (T)radius;
        T v = t_exp(T(-0.5) * d * d / (sigma * sigma));
        k[i] = v;
        sum += v;
    }
    for (auto& v : k) v /= sum;
    return k;
}

// backward.rs:776-807 (zero padding)
template <class T> inline void blur(const T* src, int w, int h, const std::vector<T>& k, T* out) {
    int radius = (int)(k.size() / 2);
    std::vector<T> tmp((size_t)w * h);
    for (int y = 0; y < h; ++y)
        for (int x = 0; x < w; ++x) {
            T acc = 0;
            for (int ki = 0; ki < (int)k.size(); ++ki) {
                int sx = x + ki - radius;
                if (sx >= 0 && sx < w) acc += k[ki] * src[(size_t)y * w + sx];
            }
            tmp[(size_t)y * w + x] = acc;
        }
    for (int y = 0; y < h; ++y)
        for (int x = 0; x < w; ++x) {
            T acc = 0;
            for (int ki = 0; ki < (int)k.size(); ++ki) {
                int sy = y + ki - radius;
                if (sy >= 0 && sy < h) acc += k[ki] * tmp[(size_t)sy * w + x];
            }
            out[(size_t)y * w + x] = acc;
        }
}

// backward.rs:697-756; returns sum of SSIM and writes d(sum)/dx.
template <class T> inline T ssim_channel(const T* x, const T* y, int w, int h, const std::vector<T>& k, T* grad) {
    const T C1 = LIT(0.01) * LIT(0.01);
    const T C2 = LIT(0.03) * LIT(0.03);
    size_t n = (size_t)w * h;
    std::vector<T> mu_x(n), mu_y(n), xx(n), yy(n), xy(n), mu_xx(n), mu_yy(n), mu_xy(n);
    blur(x, w, h, k, mu_x.data());
    blur(y, w, h, k, mu_y.data());
    for (size_t p = 0; p < n; ++p) { xx[p] = x[p] * x[p]; yy[p] = y[p] * y[p]; xy[p] = x[p] * y[p]; }
    blur(xx.data(), w, h, k, mu_xx.data());
    blur(yy.data(), w, h, k, mu_yy.data());
    blur(xy.data(), w, h, k, mu_xy.data());
    T ssim_sum = 0;
    std::vector<T> pm(n), qm(n), rm(n), qmu(n), rmu(n);
    for (size_t p = 0; p < n; ++p) {
        T mx = mu_x[p], my = mu_y[p];
        T sx2 = mu_xx[p] - mx * mx;
        T sy2 = mu_yy[p] - my * my;
        T sxy = mu_xy[p] - mx * my;
        T a1 = T(2) * mx * my + C1;
        T a2 = T(2) * sxy + C2;
        T b1 = mx * mx + my * my + C1;
        T b2 = sx2 + sy2 + C2;
        T num = a1 * a2;
        T den = b1 * b2;
        ssim_sum += num / den;
        T inv_den = T(1) / den;
        T p_coef = inv_den * (T(2) * my * a2) - (num / (den * den)) * (T(2) * mx * b2);
        T q_coef = inv_den * (T(2) * a1);
        T r_coef = -(num / (den * den)) * b1;
        pm[p] = p_coef; qm[p] = q_coef; rm[p] = r_coef;
        qmu[p] = q_coef * my; rmu[p] = r_coef * mx;
    }
    std::vector<T> bp(n), bq(n), br(n), bqmu(n), brmu(n);
    blur(pm.data(), w, h, k, bp.data());
    blur(qm.data(), w, h, k, bq.data());
    blur(rm.data(), w, h, k, br.data());
    blur(qmu.data(), w, h, k, bqmu.data());
    blur(rmu.data(), w, h, k, brmu.data());
    for (size_t p = 0; p < n; ++p) grad[p] = bp[p] + y[p] * bq[p] - bqmu[p] + T(2) * x[p] * br[p] - T(2) * brmu[p];
    return ssim_sum;
}

// backward.rs:646-693
template <class T> inline T photometric_loss_grad(const T* rendered, const T* target_rgba, int w, int h, T lambda, T* dl) {
    size_t n = (size_t)w * h;
    T m_total = (T)(n * 3);
    std::vector<T> x[3], y[3];
    for (int ch = 0; ch < 3; ++ch) { x[ch].resize(n); y[ch].resize(n); }
    for (size_t p = 0; p < n; ++p)
        for (int ch = 0; ch < 3; ++ch) { x[ch][p] = rendered[p * 3 + ch]; y[ch][p] = target_rgba[p * 4 + ch]; }
    T l1 = 0;
    for (size_t p = 0; p < n; ++p)
        for (int ch = 0; ch < 3; ++ch) {
            T d = rendered[p * 3 + ch] - target_rgba[p * 4 + ch];
            l1 += std::fabs(d);
            // Rust signum: +1 for +0.0 and positives, -1 for -0.0 and negatives, NaN for NaN.
            T sg = (d != d) ? d : std::copysign(T(1), d);
            dl[p * 3 + ch] = (T(1) - lambda) * sg / m_total;
        }
    l1 = l1 / m_total;
    std::vector<T> kernel = gaussian_kernel_1d<T>(5, LIT(1.5));
    T ssim_sum = 0;
    std::vector<T> g(n);
    for (int ch = 0; ch < 3; ++ch) {
        T s = ssim_channel(x[ch].data(), y[ch].data(), w, h, kernel, g.data());
        ssim_sum += s;
        for (size_t p = 0; p < n; ++p) dl[p * 3 + ch] += -lambda * g[p] / m_total;
    }
    T ssim_mean = ssim_sum / m_total;
    return (T(1) - lambda) * l1 + lambda * (T(1) - ssim_mean);
}

template <class T> struct DebugOut {
    T* rendered;        // w*h*3
    T* final_t;         // w*h
    int32_t* last;      // w*h
    T* dl_dpix;         // w*h*3
    T* acc;             // n*9 per Gaussian (color3, opacity, conic3, sx, sy)
};

// backward.rs:107-149
template <class T> inline int render_and_backward(const Gaussian<T>* gs, size_t n, const Cam<T>& cam, const T* target, const T bg[3], T lambda, T* loss_out, Grad<T>* grads, const DebugOut<T>* dbg) {
    int w = cam.w, h = cam.h;
    Binned<T> B;
    int rc = project_and_bin(gs, n, cam, B);
    if (rc) return rc;
    size_t P = (size_t)w * h;
    std::vector<T> rendered(P * 3), final_t(P);
    std::vector<int32_t> last(P);
    forward_pass(B, w, h, bg, rendered.data(), final_t.data(), last.data());
    std::vector<T> dl(P * 3);
    T loss = photometric_loss_grad(rendered.data(), target, w, h, lambda, dl.data());
    std::vector<Acc<T>> sg;
    backward_pass(B, w, h, bg, final_t.data(), last.data(), dl.data(), sg);
    if (grads) {
        std::memset(grads, 0, sizeof(Grad<T>) * n);
        for (size_t si = 0; si < B.splats.size(); ++si) {
            const Splat<T>& s = B.splats[si];
            geometry_backprop(s, sg[si], gs[s.gi], cam, grads[s.gi]);
        }
    }
    if (dbg) {
        if (dbg->rendered) std::memcpy(dbg->rendered, rendered.data(), P * 3 * sizeof(T));
        if (dbg->final_t) std::memcpy(dbg->final_t, final_t.data(), P * sizeof(T));
        if (dbg->last) std::memcpy(dbg->last, last.data(), P * sizeof(int32_t));
        if (dbg->dl_dpix) std::memcpy(dbg->dl_dpix, dl.data(), P * 3 * sizeof(T));
        if (dbg->acc) {
            std::memset(dbg->acc, 0, n * 9 * sizeof(T));
            for (size_t si = 0; si < B.splats.size(); ++si) {
                T* a = dbg->acc + (size_t)B.splats[si].gi * 9;
                const Acc<T>& s = sg[si];
                a[0] = s.color[0]; a[1] = s.color[1]; a[2] = s.color[2]; a[3] = s.opacity;
                a[4] = s.conic[0]; a[5] = s.conic[1]; a[6] = s.conic[2]; a[7] = s.sx; a[8] = s.sy;
            }
        }
    }
    if (loss_out) *loss_out = loss;
    return ORC_OK;
}

// cpu::rasterize, src/cpu/rasterizer.rs:72-192: the same projection, depth
// order and 16x16 tile lists as the training path (project_gaussian,
// rasterizer.rs:198-257, repeats backward.rs's project), composited per pixel
// from a colour that STARTS at bg (tile_buf init, :133) with the weighted
// splat colours added and no bg * T term; alpha = 1 - T (:179). A pixel stops
// taking splats once T < 1e-4 (:147). Tiles no splat touches keep (0, 0, 0, 0).
template <class T> inline int rasterize(const Gaussian<T>* gs, size_t n, const Cam<T>& cam, const T bg[3], T* rgba) {
    Binned<T> B;
    int rc = project_and_bin(gs, n, cam, B);
    if (rc) return rc;
    const int w = cam.w, h = cam.h;
    const T ATH = Consts<T>::alpha_threshold(), TST = Consts<T>::transmittance_stop(), MA = Consts<T>::max_alpha();
    std::fill(rgba, rgba + (size_t)w * h * 4, T(0));
#pragma omp parallel for schedule(dynamic, 4)
    for (long ti = 0; ti < (long)B.tile_lists.size(); ++ti) {
        const std::vector<int>& L = B.tile_lists[ti];
        if (L.empty()) continue;
        int tx = (int)(ti % B.ntx), ty = (int)(ti / B.ntx);
        int px0 = tx * TILE_SIZE, py0 = ty * TILE_SIZE;
        int px1 = std::min(px0 + TILE_SIZE, w), py1 = std::min(py0 + TILE_SIZE, h);
        for (int py = py0; py < py1; ++py)
            for (int px = px0; px < px1; ++px) {
                T t = 1, col[3] = {bg[0], bg[1], bg[2]};
                for (size_t li = 0; li < L.size(); ++li) {
                    if (t < TST) break;
                    const Splat<T>& s = B.splats[L[li]];
                    T dx = (T)px + T(0.5) - s.sx;
                    T dy = (T)py + T(0.5) - s.sy;
                    T a = s.conic[0], b = s.conic[1], c = s.conic[2];
                    T power = T(-0.5) * (a * dx * dx + T(2) * b * dx * dy + c * dy * dy);
                    if (power > T(0)) continue;
                    T alpha = rmin(s.opacity * t_expa(power), MA);
                    if (alpha < ATH) continue;
                    T weight = alpha * t;
                    col[0] += s.color[0] * weight;
                    col[1] += s.color[1] * weight;
                    col[2] += s.color[2] * weight;
                    t *= T(1) - alpha;
                }
                size_t pix = (size_t)py * w + px;
                rgba[pix * 4] = col[0];
                rgba[pix * 4 + 1] = col[1];
                rgba[pix * 4 + 2] = col[2];
                rgba[pix * 4 + 3] = T(1) - t;
            }
    }
    return ORC_OK;
}

// Framebuffer::to_u8_srgb, rasterizer.rs:38-48: RGB through linear_to_srgb,
// alpha linear, each clamped to [0, 1], scaled by 255 and cast as u8.
inline void to_u8_srgb(const float* rgba, size_t n_values, uint8_t* out) {
    for (size_t i = 0; i < n_values; ++i) {
        const float v = rclamp(rgba[i], 0.0f, 1.0f);
        out[i] = i % 4 == 3 ? fm::as_u8(v * 255.0f) : fm::as_u8(fm::linear_to_srgb(v) * 255.0f);
    }
}

// backward.rs:152-166
template <class T> inline int render_color(const Gaussian<T>* gs, size_t n, const Cam<T>& cam, const T bg[3], T* rgb, T* final_t_out, int32_t* last_out) {
    Binned<T> B;
    int rc = project_and_bin(gs, n, cam, B);
    if (rc) return rc;
    size_t P = (size_t)cam.w * cam.h;
    std::vector<T> ft(P);
    std::vector<int32_t> lc(P);
    forward_pass(B, cam.w, cam.h, bg, rgb, ft.data(), lc.data());
    if (final_t_out) std::memcpy(final_t_out, ft.data(), P * sizeof(T));
    if (last_out) std::memcpy(last_out, lc.data(), P * sizeof(int32_t));
    return ORC_OK;
}

// ---------------------------------------------------------------------------
// optimizer.rs
// ---------------------------------------------------------------------------
struct TrainCfgIn {  // mirrors TrainConfig (optimizer.rs:22-40)
    uint64_t num_iterations;
    float lr_position, lr_rotation, lr_scale, lr_opacity, lr_sh_dc, lr_sh_rest;
    float beta1, beta2, eps;
    uint64_t densify_from_iter, densify_until_iter;
    float densify_grad_threshold;
    uint64_t opacity_reset_iter;
    float prune_opacity_thresh;
    uint64_t max_gaussians;
};

// compiler-rt __powisf2 (LLVM's lowering of f32::powi): binary exponentiation.
template <class T> inline T powi(T a, int b) {
    bool recip = b < 0;
    T r = 1;
    while (true) {
        if (b & 1) r *= a;
        b /= 2;
        if (b == 0) break;
        a *= a;
    }
    return recip ? T(1) / r : r;
}

// optimizer.rs:175-184 (flat index order of flatten_grad, :165-173)
template <class T> inline void learning_rates(const TrainCfgIn& c, T lr[NP]) {
    int i = 0;
    for (int k = 0; k < 3; ++k) lr[i++] = (T)c.lr_position;
    for (int k = 0; k < 4; ++k) lr[i++] = (T)c.lr_rotation;
    for (int k = 0; k < 3; ++k) lr[i++] = (T)c.lr_scale;
    lr[i++] = (T)c.lr_opacity;
    for (int k = 0; k < 3; ++k) lr[i++] = (T)c.lr_sh_dc;
    for (int k = 0; k < 45; ++k) lr[i++] = (T)c.lr_sh_rest;
}

// flat index j of flatten_grad -> float offset inside the Gaussian3D record
// (apply_update_to_gaussian, optimizer.rs:186-195).
inline int flat_to_record(int j) {
    if (j < 3) return j;            // position
    if (j < 7) return 4 + (j - 3);  // rotation
    if (j < 10) return 8 + (j - 7); // log_scale
    if (j == 10) return 3;          // opacity_logit
    return 11 + (j - 11);           // sh
}

// optimizer.rs:116-163. m1/m2 hold at least n*59 floats, grad_accum/denom n.
template <class T> inline void adam_step(Gaussian<T>* gs, size_t n, const Grad<T>* grads, T* m1, T* m2, T* grad_accum, uint32_t* grad_denom, uint64_t* t, const TrainCfgIn& cfg) {
    *t += 1;
    T b1 = (T)cfg.beta1, b2 = (T)cfg.beta2, eps = (T)cfg.eps;
    T bc1 = T(1) - powi(b1, (int)*t);
    T bc2 = T(1) - powi(b2, (int)*t);
    T lrs[NP];
    learning_rates(cfg, lrs);
#pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)n; ++i) {
        const T* gr = (const T*)&grads[i];  // flatten_grad order == Grad field order
        T* rec = (T*)&gs[i];
        T* a = m1 + (size_t)i * NP;
        T* v = m2 + (size_t)i * NP;
        for (int j = 0; j < NP; ++j) {
            T gj = gr[j];
            a[j] = b1 * a[j] + (T(1) - b1) * gj;
            v[j] = b2 * v[j] + (T(1) - b2) * gj * gj;
            T m1h = a[j] / bc1;
            T m2h = v[j] / bc2;
            T upd = lrs[j] * m1h / (std::sqrt(m2h) + eps);
            rec[flat_to_record(j)] -= upd;
        }
        grad_accum[i] += grads[i].screen_grad_norm;
        grad_denom[i] += 1;
    }
#pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)n; ++i) {
        T* q = gs[i].rotation;
        T nrm = std::sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
        if (nrm > LIT(1e-8)) { q[0] /= nrm; q[1] /= nrm; q[2] /= nrm; q[3] /= nrm; }
    }
}

// optimizer.rs:274-301 (the major axis uses the normalised-quaternion rotation)
template <class T> inline void split_gaussian(const Gaussian<T>& g, Gaussian<T> out[2]) {
    T s[3]; scale_of(g, s);
    M3<T> r = to_rotation_matrix(g.rotation);
    T ax[3] = {r.m[0][0] * s[0], r.m[1][0] * s[0], r.m[2][0] * s[0]};
    T nrm = std::sqrt(ax[0] * ax[0] + ax[1] * ax[1] + ax[2] * ax[2]);
    T off[3] = {ax[0] / nrm * s[0], ax[1] / nrm * s[0], ax[2] / nrm * s[0]};
    out[0] = g; out[1] = g;
    for (int i = 0; i < 3; ++i) { out[0].position[i] += off[i]; out[1].position[i] -= off[i]; }
    const T SQRT_2 = LIT(1.4142135623730951);
    T ns = t_log(rmax(s[0] / SQRT_2, LIT(1e-6)));
    out[0].log_scale[0] = ns; out[1].log_scale[0] = ns;
    T no = rclamp(sigmoid(g.opacity_logit) * LIT(0.8), LIT(1e-6), LIT(0.999));
    T nl = logit(no);
    out[0].opacity_logit = nl; out[1].opacity_logit = nl;
}

// optimizer.rs:303-311
template <class T> inline Gaussian<T> clone_gaussian(const Gaussian<T>& g, T grad_strength) {
    Gaussian<T> c = g;
    T jitter = grad_strength * LIT(0.01);
    c.position[0] += jitter;
    c.position[1] += jitter;
    return c;
}

// optimizer.rs:206-272. Returns the new count; `out` must hold 3*n Gaussians.
// Adam moments are not touched (AdamState::resize only grows, optimizer.rs:97-105).
template <class T> inline size_t densify_and_prune(const Gaussian<T>* gs, size_t n, Gaussian<T>* out, const T* grad_accum, const uint32_t* grad_denom, const TrainCfgIn& cfg, T extent) {
    std::vector<Gaussian<T>> to_add;
    std::vector<char> remove(n, 0);
    std::vector<T> avg(n);
    for (size_t i = 0; i < n; ++i) avg[i] = grad_denom[i] > 0 ? grad_accum[i] / (T)grad_denom[i] : T(0);
    for (size_t i = 0; i < n; ++i) {
        const Gaussian<T>& g = gs[i];
        T alpha = sigmoid(g.opacity_logit);
        T s[3]; scale_of(g, s);
        T ms = rmax(rmax(s[0], s[1]), s[2]);
        if (alpha < (T)cfg.prune_opacity_thresh || ms > LIT(0.1) * extent) { remove[i] = 1; continue; }
        if (avg[i] >= (T)cfg.densify_grad_threshold && n + to_add.size() < cfg.max_gaussians) {
            if (ms > LIT(0.01) * extent) {
                remove[i] = 1;
                Gaussian<T> ch[2];
                split_gaussian(g, ch);
                to_add.push_back(ch[0]);
                to_add.push_back(ch[1]);
            } else {
                to_add.push_back(clone_gaussian(g, avg[i]));
            }
        }
    }
    size_t k = 0;
    for (size_t i = 0; i < n; ++i)
        if (!remove[i]) out[k++] = gs[i];
    for (auto& g : to_add) out[k++] = g;
    return k;
}

// optimizer.rs:314-319
template <class T> inline void reset_opacities(Gaussian<T>* gs, size_t n) {
#pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)n; ++i) gs[i].opacity_logit = logit(rmin(LIT(0.01), sigmoid(gs[i].opacity_logit)));
}

// pipeline/mod.rs:299-313
template <class T> inline T estimate_scene_extent(const Gaussian<T>* gs, size_t n) {
    if (n == 0) return T(1);
    T mn[3] = {std::numeric_limits<T>::max(), std::numeric_limits<T>::max(), std::numeric_limits<T>::max()};
    T mx[3] = {std::numeric_limits<T>::lowest(), std::numeric_limits<T>::lowest(), std::numeric_limits<T>::lowest()};
    for (size_t i = 0; i < n; ++i)
        for (int k = 0; k < 3; ++k) { mn[k] = rmin(mn[k], gs[i].position[k]); mx[k] = rmax(mx[k], gs[i].position[k]); }
    T dx = mx[0] - mn[0], dy = mx[1] - mn[1], dz = mx[2] - mn[2];
    return std::sqrt(dx * dx + dy * dy + dz * dz);
}

// ---------------------------------------------------------------------------
// WGSL projection (src/gpu/splat.wgsl:57-191) and CPU composite
// (src/gpu/compute.rs:243-296, src/gpu/sort.rs:10-17).
// WGSL `mat3x3(a, b, c)` takes columns; the matrices below are written as
// [row][col] after that transposition.
// ---------------------------------------------------------------------------
struct SplatInfo2D { float sx, sy, conic_a, conic_b, conic_c, color_r, color_g, color_b, alpha, depth; };

inline void project_wgsl(const Gaussian<float>& g, const Cam<float>& cam, SplatInfo2D& o, uint32_t& key) {
    std::memset(&o, 0, sizeof(o));
    float pc[3]; view_mul(cam, g.position, pc);
    float tz = pc[2];
    if (tz <= 0.001f) { key = 0xFFFFFFFFu; return; }
    float alpha = 1.0f / (1.0f + t_exp(-g.opacity_logit));
    if (alpha < 1.0f / 255.0f) { key = 0xFFFFFFFFu; return; }
    float sx = cam.fx * pc[0] / tz + cam.cx;
    float sy = cam.fy * pc[1] / tz + cam.cy;
    // quat_to_mat3 (no normalisation); columns as written in the shader
    float w = g.rotation[0], x = g.rotation[1], y = g.rotation[2], z = g.rotation[3];
    M3<float> R;
    R.m[0][0] = 1.0f - 2.0f * (y * y + z * z); R.m[1][0] = 2.0f * (x * y + w * z); R.m[2][0] = 2.0f * (x * z - w * y);
    R.m[0][1] = 2.0f * (x * y - w * z); R.m[1][1] = 1.0f - 2.0f * (x * x + z * z); R.m[2][1] = 2.0f * (y * z + w * x);
    R.m[0][2] = 2.0f * (x * z + w * y); R.m[1][2] = 2.0f * (y * z - w * x); R.m[2][2] = 1.0f - 2.0f * (x * x + y * y);
    float s[3] = {t_exp(g.log_scale[0]), t_exp(g.log_scale[1]), t_exp(g.log_scale[2])};
    M3<float> S = {{{s[0], 0, 0}, {0, s[1], 0}, {0, 0, s[2]}}};
    M3<float> RS = mul(R, S);
    M3<float> sig = mul(RS, tr(RS));
    float tx = pc[0], ty = pc[1];
    float fx = cam.fx, fy = cam.fy;
    // J = mat3x3(col0 = (fx/tz, 0, -fx*tx/tz^2), col1 = (0, fy/tz, -fy*ty/tz^2), col2 = 0)
    M3<float> J = {{{fx / tz, 0, 0}, {0, fy / tz, 0}, {-fx * tx / (tz * tz), -fy * ty / (tz * tz), 0}}};
    M3<float> W = view3(cam);
    M3<float> T_ = mul(J, W);
    M3<float> s2 = mul(mul(T_, sig), tr(T_));
    float a = s2.m[0][0] + 0.3f;
    float b = s2.m[1][0];  // sigma2d[0][1]: column 0, row 1
    float c = s2.m[1][1] + 0.3f;
    float det = a * c - b * b;
    if (std::fabs(det) < 1e-8f) { key = 0xFFFFFFFFu; return; }
    float inv_det = 1.0f / det;
    const float C0 = 0.28209479177387814f;
    o.sx = sx; o.sy = sy;
    o.conic_a = c * inv_det; o.conic_b = -b * inv_det; o.conic_c = a * inv_det;
    o.color_r = rclamp(0.5f + g.sh[0] * C0, 0.0f, 1.0f);
    o.color_g = rclamp(0.5f + g.sh[16] * C0, 0.0f, 1.0f);
    o.color_b = rclamp(0.5f + g.sh[32] * C0, 0.0f, 1.0f);
    o.alpha = alpha;
    o.depth = tz;
    uint32_t bits; std::memcpy(&bits, &tz, 4);
    key = ~bits;
}

inline void composite(const SplatInfo2D* sp, size_t n, int w, int h, const float bg[3], float* color) {
    std::vector<int> order;
    for (size_t i = 0; i < n; ++i)
        if (sp[i].alpha >= 1.0f / 255.0f && sp[i].depth > 0.0f) order.push_back((int)i);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return sp[a].depth < sp[b].depth; });
    std::vector<float> trans((size_t)w * h, 1.0f);
    for (size_t p = 0; p < (size_t)w * h * 3; ++p) color[p] = 0.0f;
    for (int i : order) {
        const SplatInfo2D& s = sp[i];
        float a = s.conic_a, b = s.conic_b, c = s.conic_c;
        float mid = 0.5f * (a + c);
        float disc = std::sqrt(0.25f * (a - c) * (a - c) + b * b);
        float lmin = rmax(mid - disc, 1e-6f);
        float rad = 3.0f * std::sqrt(1.0f / lmin);
        int64_t x0 = as_i64(rmax(std::floor(s.sx - rad), 0.0f));
        int64_t y0 = as_i64(rmax(std::floor(s.sy - rad), 0.0f));
        int64_t x1 = std::min(std::max(as_i64(std::ceil(s.sx + rad)), (int64_t)0), (int64_t)w);
        int64_t y1 = std::min(std::max(as_i64(std::ceil(s.sy + rad)), (int64_t)0), (int64_t)h);
        for (int64_t py = y0; py < y1; ++py)
            for (int64_t px = x0; px < x1; ++px) {
                size_t pix = (size_t)py * w + px;
                float t = trans[pix];
                if (t < 1e-4f) continue;
                float dx = (float)px + 0.5f - s.sx;
                float dy = (float)py + 0.5f - s.sy;
                float power = -0.5f * (a * dx * dx + 2.0f * b * dx * dy + c * dy * dy);
                if (power > 0.0f) continue;
                float alpha = rmin(s.alpha * t_expa(power), 0.99f);
                if (alpha < 1.0f / 255.0f) continue;
                float weight = alpha * t;
                color[pix * 3] += s.color_r * weight;
                color[pix * 3 + 1] += s.color_g * weight;
                color[pix * 3 + 2] += s.color_b * weight;
                trans[pix] = t * (1.0f - alpha);
            }
    }
    for (size_t pix = 0; pix < (size_t)w * h; ++pix) {
        float t = trans[pix];
        color[pix * 3] += t * bg[0];
        color[pix * 3 + 1] += t * bg[1];
        color[pix * 3 + 2] += t * bg[2];
    }
}

#undef LIT
}  // namespace orc

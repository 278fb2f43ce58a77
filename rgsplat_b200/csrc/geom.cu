// geom.cu -- geometry backward (blend accumulators -> GaussianGrad), Adam, and
// the fused geometry-backward + Adam of the batched training step.
//
// Geometry follows src/cpu/backward.rs:518-638 (`geometry_backprop`) with
// src/math/covariance.rs:42-84 (`backprop_cov3d`), src/math/quaternion.rs:45-70
// (`rotation_jacobian`) and src/math/sh.rs:68-89 (`sh_basis_grad`); Adam
// follows src/pipeline/optimizer.rs:116-163 (dense over all N, bias corrected,
// per-parameter learning rates, quaternion renormalisation, densification
// statistics grad_accum += screen_grad_norm, grad_denom += 1 per view).
//
// Two kernels, so neither holds the whole 59-float gradient and the geometry
// temporaries at once (register pressure, not FLOPs, bounds this stage; both
// are latency-bound, so their register budgets are capped for occupancy:
// 8 and 6 CTAs of 128 threads per SM, measured 7 % faster than uncapped):
//  (A) one thread per visible (view, Gaussian) slot: camera-space mean, the
//      projection Jacobian, the 2D-covariance and conic back-prop, the 3D
//      covariance gradient dSigma = T^T G T, the mean gradient including the
//      SH view-direction term, the clamp mask of the colour gradient. It writes
//      64 bytes per slot.
//  (B) one thread per Gaussian: sums its views in view order, back-props the
//      summed dSigma once (backprop_cov3d is linear in dSigma), forms
//      d opacity_logit, streams the SH gradient plane by plane
//      (sum_v mask_v * basis_v, with the basis recomputed from the view
//      direction) and either applies Adam plane by plane (fused step: the
//      gradient never reaches HBM) or writes/accumulates the gradient planes.
// The projected quantities are recomputed from the parameters in project.cu's
// order; the clamp mask uses the projected colour (clamp(raw) lies strictly
// inside (0, 1) exactly when raw does).
#include "rgs_internal.cuh"
#include "rgs_math.cuh"

namespace rgs {

__device__ __forceinline__ void cam_mul_g(const DevCam& c, const float p[3], float o[3]) {
#pragma unroll
    for (int i = 0; i < 3; ++i)
        o[i] = ((c.view[i * 4 + 0] * p[0] + c.view[i * 4 + 1] * p[1]) + c.view[i * 4 + 2] * p[2]) + c.view[i * 4 + 3] * 1.0f;
}

// sh.rs:68-89
__device__ __forceinline__ void sh_basis_grad(const float d[3], float g[16][3]) {
    float x = d[0], y = d[1], z = d[2];
    float xx = x * x, yy = y * y, zz = z * z;
    g[0][0] = 0.0f; g[0][1] = 0.0f; g[0][2] = 0.0f;
    g[1][0] = 0.0f; g[1][1] = -SH_C1; g[1][2] = 0.0f;
    g[2][0] = 0.0f; g[2][1] = 0.0f; g[2][2] = SH_C1;
    g[3][0] = -SH_C1; g[3][1] = 0.0f; g[3][2] = 0.0f;
    g[4][0] = SH_C2_0 * y; g[4][1] = SH_C2_0 * x; g[4][2] = 0.0f;
    g[5][0] = 0.0f; g[5][1] = SH_C2_1 * z; g[5][2] = SH_C2_1 * y;
    g[6][0] = SH_C2_2 * -2.0f * x; g[6][1] = SH_C2_2 * -2.0f * y; g[6][2] = SH_C2_2 * 4.0f * z;
    g[7][0] = SH_C2_3 * z; g[7][1] = 0.0f; g[7][2] = SH_C2_3 * x;
    g[8][0] = SH_C2_4 * 2.0f * x; g[8][1] = SH_C2_4 * -2.0f * y; g[8][2] = 0.0f;
    g[9][0] = SH_C3_0 * 6.0f * x * y; g[9][1] = SH_C3_0 * 3.0f * (xx - yy); g[9][2] = 0.0f;
    g[10][0] = SH_C3_1 * y * z; g[10][1] = SH_C3_1 * x * z; g[10][2] = SH_C3_1 * x * y;
    g[11][0] = SH_C3_2 * -2.0f * x * y; g[11][1] = SH_C3_2 * (4.0f * zz - xx - 3.0f * yy); g[11][2] = SH_C3_2 * 8.0f * y * z;
    g[12][0] = SH_C3_3 * -6.0f * x * z; g[12][1] = SH_C3_3 * -6.0f * y * z; g[12][2] = SH_C3_3 * (6.0f * zz - 3.0f * xx - 3.0f * yy);
    g[13][0] = SH_C3_4 * (4.0f * zz - 3.0f * xx - yy); g[13][1] = SH_C3_4 * -2.0f * x * y; g[13][2] = SH_C3_4 * 8.0f * x * z;
    g[14][0] = SH_C3_5 * 2.0f * x * z; g[14][1] = SH_C3_5 * -2.0f * y * z; g[14][2] = SH_C3_5 * (xx - yy);
    g[15][0] = SH_C3_6 * 3.0f * (xx - yy); g[15][1] = SH_C3_6 * -6.0f * x * y; g[15][2] = 0.0f;
}

__device__ __forceinline__ float lane_of(const float4& v, int l) { return l == 0 ? v.x : l == 1 ? v.y : l == 2 ? v.z : v.w; }

// ---------------------------------------------------------------------------
// (A) per (view, Gaussian) slot
//   gv[0][s] = (d position xyz, d opacity (before the sigmoid factor))
//   gv[1][s] = (dSigma00, dSigma01, dSigma02, dSigma11)
//   gv[2][s] = (dSigma12, dSigma22, screen_grad_norm, mask * dcolor r)
//   gv[3][s] = (mask * dcolor g, mask * dcolor b, 0, 0)
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(128, 8) k_geom_view(const float4* __restrict__ params, int n, int cap, const DevCam* __restrict__ cams,
                                                   int nviews, const uint32_t* __restrict__ cnt, const float4* __restrict__ acc,
                                                   const float4* __restrict__ rec, const float4* __restrict__ gcache,
                                                   float4* __restrict__ gv) {
    const size_t S = (size_t)n * nviews;
    // chunk-major grid (as k_project): the per-Gaussian reads of the nviews
    // consecutive blocks are shared through L2
    const int v = (int)(blockIdx.x % (unsigned)nviews);
    const int i = (int)((blockIdx.x / (unsigned)nviews) * blockDim.x + threadIdx.x);
    if (i >= n) return;
    const size_t s = (size_t)v * n + i;
    if (cnt[s] == 0) return;
    const DevCam& c = cams[v];
    const float4 a0 = acc[s], a1 = acc[S + s], a2 = acc[2 * S + s];
    const float4 col = rec[2 * S + s];
    const float4 p0 = params[i];
    const float pos[3] = {p0.x, p0.y, p0.z};
    // the 3D covariance of the projection (project.cu k_gauss_cache, this step)
    const float4 g0 = gcache[i], g1 = gcache[(size_t)cap + i];
    const M3 sig = {{{g0.y, g0.z, g0.w}, {g0.z, g1.x, g1.y}, {g0.w, g1.y, g1.z}}};
    float pc[3];
    cam_mul_g(c, pos, pc);
    const float fx = c.fx, fy = c.fy;
    M3 V;
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int k = 0; k < 3; ++k) V.m[r][k] = c.view[r * 4 + k];
    // projection.rs:24-69 (the projection clamps tz; visible splats have tz > 0.001)
    const float tx = pc[0], ty = pc[1], tz = pc[2];
    const float tzc = fmaxf(tz, 0.001f);
    float a2d, b2d, c2d;
    {
        // one reciprocal per denominator (gradients are held to 1e-3 relative,
        // so the quotients need not round as the reference's divisions)
        const float itc = 1.0f / tzc, itc2 = itc * itc;
        M3 j = {{{fx * itc, 0.0f, -fx * tx * itc2}, {0.0f, fy * itc, -fy * ty * itc2}, {0.0f, 0.0f, 0.0f}}};
        M3 t = mul(j, V);
        M3 s2 = mul(mul(t, sig), tr(t));
        a2d = s2.m[0][0] + 0.3f;
        b2d = s2.m[0][1];
        c2d = s2.m[1][1] + 0.3f;
    }
    // conic -> 2D covariance (backward.rs:546-554)
    const float ga = a1.x, gb = a1.y, gc = a1.z;
    const float det = a2d * c2d - b2d * b2d;
    const float idet2 = 1.0f / (det * det);
    const float dl_da = (-ga * c2d * c2d + gb * b2d * c2d - gc * b2d * b2d) * idet2;
    const float dl_db = (2.0f * ga * b2d * c2d - gb * (det + 2.0f * b2d * b2d) + 2.0f * gc * a2d * b2d) * idet2;
    const float dl_dc = (-ga * b2d * b2d + gb * a2d * b2d - gc * a2d * a2d) * idet2;
    // T = J W, rows u0, u1 (row 2 of J is zero) (backward.rs:556-564)
    const float itz = 1.0f / tz, itz2 = itz * itz, itz3 = itz2 * itz;
    const float j00 = fx * itz, j02 = -fx * tx * itz2, j11 = fy * itz, j12 = -fy * ty * itz2;
    float u0[3], u1[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        u0[k] = j00 * V.m[0][k] + j02 * V.m[2][k];
        u1[k] = j11 * V.m[1][k] + j12 * V.m[2][k];
    }
    // dSigma3D = T^T G T with G = [[dl_da, dl_db/2], [dl_db/2, dl_dc]] (backward.rs:567-573)
    const float hb = 0.5f * dl_db;
    float r0[3], r1[3];  // G T rows
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        r0[k] = dl_da * u0[k] + hb * u1[k];
        r1[k] = hb * u0[k] + dl_dc * u1[k];
    }
    float dS[6];  // 00, 01, 02, 11, 12, 22
    dS[0] = u0[0] * r0[0] + u1[0] * r1[0];
    dS[1] = u0[0] * r0[1] + u1[0] * r1[1];
    dS[2] = u0[0] * r0[2] + u1[0] * r1[2];
    dS[3] = u0[1] * r0[1] + u1[1] * r1[1];
    dS[4] = u0[1] * r0[2] + u1[1] * r1[2];
    dS[5] = u0[2] * r0[2] + u1[2] * r1[2];
    // mean through (sx, sy) and through J(pcam) (backward.rs:578-605)
    const float asx = a1.w, asy = a2.x;
    float dp[3] = {asx * j00, asy * j11, asx * j02 + asy * j12};
    {
        // Sigma u0, Sigma u1, Sigma w2 with w2 = row 2 of W
        float su0[3], su1[3], sw2[3];
#pragma unroll
        for (int r = 0; r < 3; ++r) {
            su0[r] = sig.m[r][0] * u0[0] + sig.m[r][1] * u0[1] + sig.m[r][2] * u0[2];
            su1[r] = sig.m[r][0] * u1[0] + sig.m[r][1] * u1[1] + sig.m[r][2] * u1[2];
            sw2[r] = sig.m[r][0] * V.m[2][0] + sig.m[r][1] * V.m[2][1] + sig.m[r][2] * V.m[2][2];
        }
        // d/dtx: dT row 0 = -fx/tz^2 w2
        const float ax = -fx * itz2;
        const float w2su0 = V.m[2][0] * su0[0] + V.m[2][1] * su0[1] + V.m[2][2] * su0[2];
        const float w2su1 = V.m[2][0] * su1[0] + V.m[2][1] * su1[1] + V.m[2][2] * su1[2];
        dp[0] += dl_da * (2.0f * ax * w2su0) + dl_db * (ax * w2su1);
        // d/dty: dT row 1 = -fy/tz^2 w2
        const float ay = -fy * itz2;
        const float u0sw2 = u0[0] * sw2[0] + u0[1] * sw2[1] + u0[2] * sw2[2];
        dp[1] += dl_db * (ay * u0sw2) + dl_dc * (2.0f * ay * w2su1);
        // d/dtz: dT row 0 = -fx/tz^2 W0 + 2 fx tx/tz^3 W2, row 1 = -fy/tz^2 W1 + 2 fy ty/tz^3 W2
        float g0[3], g1[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            g0[k] = ax * V.m[0][k] + (2.0f * fx * tx * itz3) * V.m[2][k];
            g1[k] = ay * V.m[1][k] + (2.0f * fy * ty * itz3) * V.m[2][k];
        }
        const float g0su0 = g0[0] * su0[0] + g0[1] * su0[1] + g0[2] * su0[2];
        const float g0su1 = g0[0] * su1[0] + g0[1] * su1[1] + g0[2] * su1[2];
        const float g1su0 = g1[0] * su0[0] + g1[1] * su0[1] + g1[2] * su0[2];
        const float g1su1 = g1[0] * su1[0] + g1[1] * su1[1] + g1[2] * su1[2];
        dp[2] += dl_da * (2.0f * g0su0) + dl_db * (g0su1 + g1su0) + dl_dc * (2.0f * g1su1);
    }
    float dpos[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) dpos[k] = (V.m[0][k] * dp[0] + V.m[1][k] * dp[1]) + V.m[2][k] * dp[2];
    // colour mask and the SH view-direction term (backward.rs:535-539, 610-632)
    const float mr = (col.x > 0.0f && col.x < 1.0f) ? a0.x : 0.0f;
    const float mg = (col.y > 0.0f && col.y < 1.0f) ? a0.y : 0.0f;
    const float mb = (col.z > 0.0f && col.z < 1.0f) ? a0.z : 0.0f;
    const float ux = c.pos[0] - pos[0], uy = c.pos[1] - pos[1], uz = c.pos[2] - pos[2];
    const float len = sqrtf(ux * ux + uy * uy + uz * uz);
    if (len > 1e-8f && (mr != 0.0f || mg != 0.0f || mb != 0.0f)) {
        const float ilen = 1.0f / len;
        const float dir[3] = {ux * ilen, uy * ilen, uz * ilen};
        float db[16][3];
        sh_basis_grad(dir, db);
        float dd0 = 0.0f, dd1 = 0.0f, dd2 = 0.0f;
#pragma unroll
        for (int kq = 0; kq < 4; ++kq) {
            const float4 cr = params[(size_t)(3 + kq) * cap + i];
            const float4 cg = params[(size_t)(7 + kq) * cap + i];
            const float4 cb = params[(size_t)(11 + kq) * cap + i];
#pragma unroll
            for (int l = 0; l < 4; ++l) {
                const int k = kq * 4 + l;
                const float dbk = mr * lane_of(cr, l) + mg * lane_of(cg, l) + mb * lane_of(cb, l);
                dd0 += dbk * db[k][0];
                dd1 += dbk * db[k][1];
                dd2 += dbk * db[k][2];
            }
        }
        const float dot = dir[0] * dd0 + dir[1] * dd1 + dir[2] * dd2;
        dpos[0] += -((dd0 - dir[0] * dot) * ilen);
        dpos[1] += -((dd1 - dir[1] * dot) * ilen);
        dpos[2] += -((dd2 - dir[2] * dot) * ilen);
    }
    gv[s] = make_float4(dpos[0], dpos[1], dpos[2], a0.w);
    gv[S + s] = make_float4(dS[0], dS[1], dS[2], dS[3]);
    gv[2 * S + s] = make_float4(dS[4], dS[5], sqrtf(asx * asx + asy * asy), mr);
    gv[3 * S + s] = make_float4(mg, mb, 0.0f, 0.0f);
}

// optimizer.rs:142-147 for one element.
__device__ __forceinline__ float adam_lane(float p, float g, float& m1, float& m2, float lr, const AdamArgs& a, float bc1,
                                           float bc2) {
    m1 = a.b1 * m1 + a.one_minus_b1 * g;
    m2 = a.b2 * m2 + a.one_minus_b2 * g * g;
    float m1h = m1 / bc1;
    float m2h = m2 / bc2;
    float upd = lr * m1h / (sqrtf(m2h) + a.eps);
    return p - upd;
}

// Adam on plane p of Gaussian i (lanes 0..3; plane 2 has only three).
// One plane's update with its moments already loaded (m1, m2 updated in place).
__device__ __forceinline__ float4 adam_update(int p, float4 pv, float4 g, float4& m1, float4& m2, const AdamArgs& a, float bc1,
                                              float bc2) {
    const float* lr = a.lr + p * 4;
    pv.x = adam_lane(pv.x, g.x, m1.x, m2.x, lr[0], a, bc1, bc2);
    pv.y = adam_lane(pv.y, g.y, m1.y, m2.y, lr[1], a, bc1, bc2);
    pv.z = adam_lane(pv.z, g.z, m1.z, m2.z, lr[2], a, bc1, bc2);
    if (p != 2) pv.w = adam_lane(pv.w, g.w, m1.w, m2.w, lr[3], a, bc1, bc2);
    if (p == 1) {
        // renormalise the quaternion (optimizer.rs:155-162)
        float nrm = sqrtf(pv.x * pv.x + pv.y * pv.y + pv.z * pv.z + pv.w * pv.w);
        if (nrm > 1e-8f) { pv.x /= nrm; pv.y /= nrm; pv.z /= nrm; pv.w /= nrm; }
    }
    return pv;
}

__device__ __forceinline__ float4 adam_plane(int p, int i, int cap, float4 pv, float4 g, const AdamArgs& a, float bc1, float bc2) {
    const size_t om = (size_t)p * a.mstride + i;
    float4 m1 = a.m1[om], m2 = a.m2[om];
    pv = adam_update(p, pv, g, m1, m2, a, bc1, bc2);
    a.m1[om] = m1;
    a.m2[om] = m2;
    (void)cap;
    return pv;
}

// (B) per Gaussian. MODE 0: write the gradient planes (accumulate if asked);
// MODE 1: apply Adam. PART 0 does both halves; PART 1 only the SH planes
// (3..14) and PART 2 only the geometry planes (0..2) with grad_accum/denom,
// each with fewer registers, so more warps per SM hide the memory latency.
// PART 1 must run before PART 2: it reads the position that PART 2's Adam
// step rewrites.
template <int MODE, int PART = 0>
__global__ void __launch_bounds__(128, PART == 2 ? 8 : 6) k_geom_gauss(const float4* __restrict__ params_in, int n, int cap,
                                                    const DevCam* __restrict__ cams, int nviews, const uint32_t* __restrict__ cnt,
                                                    const float4* __restrict__ gv, float4* __restrict__ grads, int accumulate,
                                                    AdamArgs a) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (MODE == 1 && a.skip_flag && *a.skip_flag) return;
    const size_t S = (size_t)n * nviews;
    float bc1 = 0.0f, bc2 = 0.0f;
    if (MODE == 1) {
        bc1 = a.bc_dev ? a.bc_dev[0] : a.bc1;
        bc2 = a.bc_dev ? a.bc_dev[1] : a.bc2;
    }
    const float4* params = MODE == 1 ? a.params : params_in;
    const float4 p0 = params[i];
    const float pos[3] = {p0.x, p0.y, p0.z};
    if (PART != 2) {
    // ---- SH planes: sum_v mask_v[ch] * basis_v (the basis once per view, all
    // 48 sums in registers), then Adam / store per plane
    float shg[3][16];
#pragma unroll
    for (int ch = 0; ch < 3; ++ch)
#pragma unroll
        for (int k = 0; k < 16; ++k) shg[ch][k] = 0.0f;
    for (int v = 0; v < nviews; ++v) {
        const size_t s = (size_t)v * n + i;
        if (cnt[s] == 0) continue;
        const float4 m2 = gv[2 * S + s], m3 = gv[3 * S + s];
        const float mk[3] = {m2.w, m3.x, m3.y};
        if (mk[0] == 0.0f && mk[1] == 0.0f && mk[2] == 0.0f) continue;
        float d[3], basis[16];
        view_dir(pos, cams[v].pos, d);
        sh_basis(d, basis);
#pragma unroll
        for (int ch = 0; ch < 3; ++ch)
#pragma unroll
            for (int k = 0; k < 16; ++k) shg[ch][k] += mk[ch] * basis[k];
    }
#pragma unroll
    for (int ch = 0; ch < 3; ++ch) {
#pragma unroll
        for (int kq = 0; kq < 4; ++kq) {
            const int p = 3 + ch * 4 + kq;
            const size_t o = (size_t)p * cap + i;
            float4 g = make_float4(shg[ch][kq * 4 + 0], shg[ch][kq * 4 + 1], shg[ch][kq * 4 + 2], shg[ch][kq * 4 + 3]);
            if (MODE == 1) {
                a.params[o] = adam_plane(p, i, cap, a.params[o], g, a, bc1, bc2);
            } else {
                if (accumulate) {
                    const float4 old = grads[o];
                    g.x += old.x; g.y += old.y; g.z += old.z; g.w += old.w;
                }
                grads[o] = g;
            }
        }
    }
    }
    if (PART == 1) return;
    // ---- geometry: sums over views
    float dpos[3] = {0.0f, 0.0f, 0.0f}, dop = 0.0f, dS[6] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f}, screen = 0.0f;
    for (int v = 0; v < nviews; ++v) {
        const size_t s = (size_t)v * n + i;
        if (cnt[s] == 0) continue;
        const float4 x0 = gv[s], x1 = gv[S + s], x2 = gv[2 * S + s];
        dpos[0] += x0.x; dpos[1] += x0.y; dpos[2] += x0.z; dop += x0.w;
        dS[0] += x1.x; dS[1] += x1.y; dS[2] += x1.z; dS[3] += x1.w;
        dS[4] += x2.x; dS[5] += x2.y; screen += x2.z;
    }
    const float4 p1 = params[(size_t)cap + i], p2 = params[2 * (size_t)cap + i];
    const float q[4] = {p1.x, p1.y, p1.z, p1.w};
    const float sc[3] = {exp_cr(p2.x), exp_cr(p2.y), exp_cr(p2.z)};
    const float op = sigmoid(p0.w);
    float d_ls[3] = {0.0f, 0.0f, 0.0f}, d_rot[4] = {0.0f, 0.0f, 0.0f, 0.0f};
    {
        // backprop_cov3d (covariance.rs:42-84) with dL/dSigma = sum over views
        const M3 g = {{{dS[0], dS[1], dS[2]}, {dS[1], dS[3], dS[4]}, {dS[2], dS[4], dS[5]}}};
        const M3 r = to_rotation_matrix(q);
        const M3 m = rs_matrix(sc, q);
        M3 gs;
#pragma unroll
        for (int x = 0; x < 3; ++x)
#pragma unroll
            for (int y = 0; y < 3; ++y) gs.m[x][y] = g.m[x][y] + g.m[y][x];
        const M3 dm = mul(gs, m);
        M3 dr;
#pragma unroll
        for (int jj = 0; jj < 3; ++jj) {
            float accs = 0.0f;
#pragma unroll
            for (int ii = 0; ii < 3; ++ii) {
                accs += dm.m[ii][jj] * r.m[ii][jj];
                dr.m[ii][jj] = dm.m[ii][jj] * sc[jj];
            }
            d_ls[jj] = accs * sc[jj];
        }
        float qn[4];
        qnormalize(q, qn);
        const float w = qn[0], x = qn[1], y = qn[2], z = qn[3];
        // sum over (row, col) of dR/dq_k * dL/dR (quaternion.rs:45-70), column-major order
        d_rot[0] = (2.0f * z * dr.m[1][0] - 2.0f * y * dr.m[2][0]) + (-2.0f * z * dr.m[0][1] + 2.0f * x * dr.m[2][1]) +
                   (2.0f * y * dr.m[0][2] - 2.0f * x * dr.m[1][2]);
        d_rot[1] = (2.0f * y * dr.m[1][0] + 2.0f * z * dr.m[2][0]) + (2.0f * y * dr.m[0][1] - 4.0f * x * dr.m[1][1] + 2.0f * w * dr.m[2][1]) +
                   (2.0f * z * dr.m[0][2] - 2.0f * w * dr.m[1][2] - 4.0f * x * dr.m[2][2]);
        d_rot[2] = (-4.0f * y * dr.m[0][0] + 2.0f * x * dr.m[1][0] - 2.0f * w * dr.m[2][0]) + (2.0f * x * dr.m[0][1] + 2.0f * z * dr.m[2][1]) +
                   (2.0f * w * dr.m[0][2] + 2.0f * z * dr.m[1][2] - 4.0f * y * dr.m[2][2]);
        d_rot[3] = (-4.0f * z * dr.m[0][0] + 2.0f * w * dr.m[1][0] + 2.0f * x * dr.m[2][0]) +
                   (-2.0f * w * dr.m[0][1] - 4.0f * z * dr.m[1][1] + 2.0f * y * dr.m[2][1]) + (2.0f * x * dr.m[0][2] + 2.0f * y * dr.m[1][2]);
    }
    const float4 g0 = make_float4(dpos[0], dpos[1], dpos[2], dop * op * (1.0f - op));
    const float4 g1 = make_float4(d_rot[0], d_rot[1], d_rot[2], d_rot[3]);
    const float4 g2 = make_float4(d_ls[0], d_ls[1], d_ls[2], screen);
    if (MODE == 1) {
        a.params[i] = adam_plane(0, i, cap, p0, g0, a, bc1, bc2);
        a.params[(size_t)cap + i] = adam_plane(1, i, cap, p1, g1, a, bc1, bc2);
        a.params[2 * (size_t)cap + i] = adam_plane(2, i, cap, p2, g2, a, bc1, bc2);
        a.grad_accum[i] += screen;
        a.grad_denom[i] += a.denom_inc;
    } else {
        const float4 gs3[3] = {g0, g1, g2};
#pragma unroll
        for (int p = 0; p < 3; ++p) {
            float4 g = gs3[p];
            const size_t o = (size_t)p * cap + i;
            if (accumulate) {
                const float4 old = grads[o];
                g.x += old.x; g.y += old.y; g.z += old.z; g.w += old.w;
            }
            grads[o] = g;
        }
    }
}

// The SH half of the fused geometry + Adam pass, one colour channel per grid
// row (blockIdx.y): sum over views of mask_v[ch] * basis_v (the views in the
// same order as k_geom_gauss<1, 1>, which adds the same products; a view whose
// mask is zero for this channel adds only zeros there), then Adam on the
// channel's four SH planes. Sixteen sums per thread instead of forty-eight,
// so more warps stay resident in this latency-bound pass. Runs before the
// geometry half, which rewrites the position it reads.
// The SH half of the per-Gaussian step: block row ch handles colour channel
// ch's 16 coefficients (planes 3 + 4 ch .. 6 + 4 ch). The per-view slot
// counts and clamp masks are loaded VIEW_GROUP views at a time before any is
// used, so the thread waits on two round trips to memory per group instead
// of two per view; the sums run in view order as before. (Loading all four
// planes' parameters and moments before the first store as well needed 104
// registers and ran slower at the lower occupancy; two planes at a time ran
// slower too, at 74 registers and 6 CTAs per SM or 64 with spills at 8; and
// one thread per plane, twelve per Gaussian each repeating the view loop,
// took 1.2 against 0.93 ms for the stage.)
constexpr int VIEW_GROUP = 8;
__global__ void __launch_bounds__(128, 8) k_geom_sh(int n, int cap, const DevCam* __restrict__ cams, int nviews,
                                                   const uint32_t* __restrict__ cnt, const float4* __restrict__ gv, AdamArgs a) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (a.skip_flag && *a.skip_flag) return;
    const int ch = (int)blockIdx.y;
    const size_t S = (size_t)n * nviews;
    const float bc1 = a.bc_dev ? a.bc_dev[0] : a.bc1;
    const float bc2 = a.bc_dev ? a.bc_dev[1] : a.bc2;
    const float4 p0 = a.params[i];
    const float pos[3] = {p0.x, p0.y, p0.z};
    const float* mplane = reinterpret_cast<const float*>(gv + (ch == 0 ? 2 : 3) * S);
    const int mlane = ch == 0 ? 3 : ch - 1;
    float shg[16];
#pragma unroll
    for (int k = 0; k < 16; ++k) shg[k] = 0.0f;
    for (int v0 = 0; v0 < nviews; v0 += VIEW_GROUP) {
        uint32_t c8[VIEW_GROUP];
        float m8[VIEW_GROUP];
#pragma unroll
        for (int k = 0; k < VIEW_GROUP; ++k) c8[k] = v0 + k < nviews ? cnt[(size_t)(v0 + k) * n + i] : 0u;
#pragma unroll
        for (int k = 0; k < VIEW_GROUP; ++k) m8[k] = c8[k] ? mplane[((size_t)(v0 + k) * n + i) * 4 + mlane] : 0.0f;
#pragma unroll
        for (int k = 0; k < VIEW_GROUP; ++k) {
            if (m8[k] == 0.0f) continue;
            float d[3], basis[16];
            view_dir(pos, cams[v0 + k].pos, d);
            sh_basis(d, basis);
#pragma unroll
            for (int q = 0; q < 16; ++q) shg[q] += m8[k] * basis[q];
        }
    }
#pragma unroll
    for (int kq = 0; kq < 4; ++kq) {
        const int p = 3 + ch * 4 + kq;
        const size_t o = (size_t)p * cap + i;
        const float4 g = make_float4(shg[kq * 4 + 0], shg[kq * 4 + 1], shg[kq * 4 + 2], shg[kq * 4 + 3]);
        a.params[o] = adam_plane(p, i, cap, a.params[o], g, a, bc1, bc2);
    }
}

static void launch_geom_view(const float4* params, int n, int cap, const DevCam* cams, int nviews, const uint32_t* cnt,
                             const float4* acc, const float4* rec, const float4* gcache, float4* gv, cudaStream_t st) {
    size_t S = (size_t)n * nviews;
    if (S == 0) return;
    k_geom_view<<<(unsigned)(((size_t)n + 127) / 128 * (size_t)nviews), 128, 0, st>>>(params, n, cap, cams, nviews, cnt, acc, rec, gcache, gv);
}

void launch_geometry(const float4* params, int n, int cap, const DevCam* cams, int nviews, const uint32_t* cnt, const float4* acc,
                     const float4* rec, const float4* gcache, float4* gv, float4* grads, int accumulate, cudaStream_t st) {
    if (n <= 0) return;
    launch_geom_view(params, n, cap, cams, nviews, cnt, acc, rec, gcache, gv, st);
    AdamArgs a{};
    k_geom_gauss<0><<<(n + 127) / 128, 128, 0, st>>>(params, n, cap, cams, nviews, cnt, gv, grads, accumulate, a);
}

void launch_geometry_adam(const DevCam* cams, int nviews, int n, int cap, const uint32_t* cnt, const float4* acc, const float4* rec,
                          const float4* gcache, float4* gv, const AdamArgs& a, cudaStream_t st) {
    if (n <= 0) return;
    launch_geom_view(a.params, n, cap, cams, nviews, cnt, acc, rec, gcache, gv, st);
    k_geom_sh<<<dim3((unsigned)((n + 127) / 128), 3), 128, 0, st>>>(n, cap, cams, nviews, cnt, gv, a);
    k_geom_gauss<1, 2><<<(n + 127) / 128, 128, 0, st>>>(nullptr, n, cap, cams, nviews, cnt, gv, nullptr, 0, a);
}

__global__ void __launch_bounds__(256) k_adam(int n, int cap, const float4* __restrict__ grads, AdamArgs a) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (a.skip_flag && *a.skip_flag) return;
    const float bc1 = a.bc_dev ? a.bc_dev[0] : a.bc1;
    const float bc2 = a.bc_dev ? a.bc_dev[1] : a.bc2;
#pragma unroll 1
    for (int p = 0; p < NPL; ++p) {
        const size_t o = (size_t)p * cap + i;
        a.params[o] = adam_plane(p, i, cap, a.params[o], grads[o], a, bc1, bc2);
    }
    a.grad_accum[i] += grads[2 * (size_t)cap + i].w;
    a.grad_denom[i] += a.denom_inc;
}

void launch_adam(int n, int cap, const float4* grads, const AdamArgs& a, cudaStream_t st) {
    if (n <= 0) return;
    k_adam<<<(n + 255) / 256, 256, 0, st>>>(n, cap, grads, a);
}

// optimizer.rs:314-319: logit(min(0.01, sigmoid(logit))).
__global__ void k_reset_opacities(float4* __restrict__ params, int n) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float4 p = params[i];
    p.w = logit(fminf(0.01f, sigmoid(p.w)));
    params[i] = p;
}

void launch_reset_opacities(float4* params, int n, int cap, cudaStream_t st) {
    (void)cap;
    if (n <= 0) return;
    k_reset_opacities<<<(n + 255) / 256, 256, 0, st>>>(params, n);
}

}  // namespace rgs

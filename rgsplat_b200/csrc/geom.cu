// geom.cu -- geometry backward (splat accumulators -> GaussianGrad), Adam, and
// the fused geometry-backward + Adam kernel of the batched training step.
//
// Geometry follows src/cpu/backward.rs:518-638 (`geometry_backprop`) with
// src/math/covariance.rs:42-84 (`backprop_cov3d`), src/math/quaternion.rs:45-70
// (`rotation_jacobian`) and src/math/sh.rs:68-89 (`sh_basis_grad`). The
// projected quantities it needs (camera-space mean, low-passed 2D covariance,
// raw SH colour and basis) are recomputed from the parameters in the same
// order as project.cu instead of being stored per splat.
// Adam follows src/pipeline/optimizer.rs:116-163: dense over all N, bias
// corrected, per-parameter learning rates, quaternion renormalisation, and the
// densification statistics grad_accum += screen_grad_norm, grad_denom += 1 per
// view.
//
// One thread per Gaussian; every parameter plane is a coalesced float4 stream.
// The fused kernel reads the parameters and moments once, sums the per-view
// gradients in registers, and writes parameters and moments once: the
// gradient never touches HBM.
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

// Per-Gaussian gradient accumulators (sum over the views of a batch).
struct GradAcc {
    float pos[3], rot[4], ls[3], op, screen;
    float sh[48];
};

// Adds one view's contribution of Gaussian i (whose slot accumulators are
// a0 = (dcolor, dopacity), a1 = (dconic, dsx), a2.x = dsy) to g.
__device__ __forceinline__ void geometry_one(const float4* __restrict__ params, int cap, int i, const DevCam& c,
                                             float4 a0, float4 a1, float4 a2, GradAcc& g) {
    float4 p0 = params[i];
    float4 p1 = params[(size_t)cap + i];
    float4 p2 = params[2 * (size_t)cap + i];
    float pos[3] = {p0.x, p0.y, p0.z};
    float q[4] = {p1.x, p1.y, p1.z, p1.w};
    float sc[3] = {exp_cr(p2.x), exp_cr(p2.y), exp_cr(p2.z)};
    float op = sigmoid(p0.w);
    float pc[3];
    cam_mul_g(c, pos, pc);
    const float fx = c.fx, fy = c.fy;
    M3 V;
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int k = 0; k < 3; ++k) V.m[r][k] = c.view[r * 4 + k];
    M3 sigma3d = build_cov3d(sc, q);
    // 2D covariance exactly as in projection (projection.rs:24-69)
    float a2d, b2d, c2d;
    {
        float tzc = fmaxf(pc[2], 0.001f);
        M3 j = {{{fx / tzc, 0.0f, -fx * pc[0] / (tzc * tzc)}, {0.0f, fy / tzc, -fy * pc[1] / (tzc * tzc)}, {0.0f, 0.0f, 0.0f}}};
        M3 t = mul(j, V);
        M3 s2 = mul(mul(t, sigma3d), tr(t));
        a2d = s2.m[0][0] + 0.3f;
        b2d = s2.m[0][1];
        c2d = s2.m[1][1] + 0.3f;
    }
    // opacity (backward.rs:529-531)
    g.op += a0.w * op * (1.0f - op);
    // SH (backward.rs:533-544): masked by the [0, 1] clamp of the raw colour
    float d[3], basis[16];
    view_dir(pos, c.pos, d);
    sh_basis(d, basis);
    float masked[3];
    float acol[3] = {a0.x, a0.y, a0.z};
#pragma unroll
    for (int ch = 0; ch < 3; ++ch) {
        float acc = 0.0f;
#pragma unroll
        for (int kq = 0; kq < 4; ++kq) {
            float4 v = params[(size_t)(3 + ch * 4 + kq) * cap + i];
            acc += basis[kq * 4 + 0] * v.x;
            acc += basis[kq * 4 + 1] * v.y;
            acc += basis[kq * 4 + 2] * v.z;
            acc += basis[kq * 4 + 3] * v.w;
        }
        float raw = 0.5f + acc;
        masked[ch] = (raw > 0.0f && raw < 1.0f) ? acol[ch] : 0.0f;
#pragma unroll
        for (int k = 0; k < 16; ++k) g.sh[ch * 16 + k] += masked[ch] * basis[k];
    }
    // conic -> 2D covariance (backward.rs:546-554)
    float ga = a1.x, gb = a1.y, gc = a1.z;
    float det = a2d * c2d - b2d * b2d;
    float det2 = det * det;
    float dl_da = (-ga * c2d * c2d + gb * b2d * c2d - gc * b2d * b2d) / det2;
    float dl_db = (2.0f * ga * b2d * c2d - gb * (det + 2.0f * b2d * b2d) + 2.0f * gc * a2d * b2d) / det2;
    float dl_dc = (-ga * b2d * b2d + gb * a2d * b2d - gc * a2d * a2d) / det2;
    // 2D covariance -> 3D covariance (backward.rs:556-576)
    float tx = pc[0], ty = pc[1], tz = pc[2];
    M3 j = {{{fx / tz, 0.0f, -fx * tx / (tz * tz)}, {0.0f, fy / tz, -fy * ty / (tz * tz)}, {0.0f, 0.0f, 0.0f}}};
    M3 t_mat = mul(j, V);
    M3 gcov = {{{dl_da, 0.5f * dl_db, 0.0f}, {0.5f * dl_db, dl_dc, 0.0f}, {0.0f, 0.0f, 0.0f}}};
    M3 dsig = mul(mul(tr(t_mat), gcov), t_mat);
    {
        // covariance.rs:42-84
        M3 r = to_rotation_matrix(q);
        M3 m = rs_matrix(sc, q);
        M3 gs;
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int b = 0; b < 3; ++b) gs.m[a][b] = dsig.m[a][b] + dsig.m[b][a];
        M3 dm = mul(gs, m);
        M3 dr;
#pragma unroll
        for (int jj = 0; jj < 3; ++jj) {
            float acc = 0.0f;
#pragma unroll
            for (int ii = 0; ii < 3; ++ii) {
                acc += dm.m[ii][jj] * r.m[ii][jj];
                dr.m[ii][jj] = dm.m[ii][jj] * sc[jj];
            }
            g.ls[jj] += acc * sc[jj];
        }
        float qn[4];
        qnormalize(q, qn);
        float w = qn[0], x = qn[1], y = qn[2], z = qn[3];
        M3 jac[4] = {
            {{{0.0f, -2.0f * z, 2.0f * y}, {2.0f * z, 0.0f, -2.0f * x}, {-2.0f * y, 2.0f * x, 0.0f}}},
            {{{0.0f, 2.0f * y, 2.0f * z}, {2.0f * y, -4.0f * x, -2.0f * w}, {2.0f * z, 2.0f * w, -4.0f * x}}},
            {{{-4.0f * y, 2.0f * x, 2.0f * w}, {2.0f * x, 0.0f, 2.0f * z}, {-2.0f * w, 2.0f * z, -4.0f * y}}},
            {{{-4.0f * z, -2.0f * w, 2.0f * x}, {2.0f * w, -4.0f * z, 2.0f * y}, {2.0f * x, 2.0f * y, 0.0f}}},
        };
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            float s = 0.0f;
#pragma unroll
            for (int cc = 0; cc < 3; ++cc)
#pragma unroll
                for (int rr = 0; rr < 3; ++rr) s += jac[k].m[rr][cc] * dr.m[rr][cc];
            g.rot[k] += s;
        }
    }
    // mean (backward.rs:578-608)
    float asx = a1.w, asy = a2.x;
    float dp[3] = {asx * fx / tz, asy * fy / tz, asx * (-fx * tx / (tz * tz)) + asy * (-fy * ty / (tz * tz))};
    {
        M3 dj[3] = {
            {{{0.0f, 0.0f, -fx / (tz * tz)}, {0.0f, 0.0f, 0.0f}, {0.0f, 0.0f, 0.0f}}},
            {{{0.0f, 0.0f, 0.0f}, {0.0f, 0.0f, -fy / (tz * tz)}, {0.0f, 0.0f, 0.0f}}},
            {{{-fx / (tz * tz), 0.0f, 2.0f * fx * tx / (tz * tz * tz)}, {0.0f, -fy / (tz * tz), 2.0f * fy * ty / (tz * tz * tz)}, {0.0f, 0.0f, 0.0f}}},
        };
        M3 sig_tt = mul(sigma3d, tr(t_mat));
        M3 ts = mul(t_mat, sigma3d);
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            M3 dt = mul(dj[k], V);
            M3 p1m = mul(dt, sig_tt), p2m = mul(ts, tr(dt));
            float d00 = p1m.m[0][0] + p2m.m[0][0], d01 = p1m.m[0][1] + p2m.m[0][1], d11 = p1m.m[1][1] + p2m.m[1][1];
            dp[k] += dl_da * d00 + dl_db * d01 + dl_dc * d11;
        }
    }
    float dpos[3];
#pragma unroll
    for (int ii = 0; ii < 3; ++ii) dpos[ii] = (V.m[0][ii] * dp[0] + V.m[1][ii] * dp[1]) + V.m[2][ii] * dp[2];
    // SH view direction (backward.rs:610-632)
    float u0 = c.pos[0] - pos[0], u1 = c.pos[1] - pos[1], u2 = c.pos[2] - pos[2];
    float len = sqrtf(u0 * u0 + u1 * u1 + u2 * u2);
    if (len > 1e-8f) {
        float dir[3] = {u0 / len, u1 / len, u2 / len};
        float db[16][3];
        sh_basis_grad(dir, db);
        float dd0 = 0.0f, dd1 = 0.0f, dd2 = 0.0f;
#pragma unroll
        for (int k = 0; k < 16; ++k) {
            int pk = 3 + k / 4, lk = k % 4;
            float4 cr = params[(size_t)pk * cap + i];
            float4 cg = params[(size_t)(pk + 4) * cap + i];
            float4 cb = params[(size_t)(pk + 8) * cap + i];
            float sr = lk == 0 ? cr.x : lk == 1 ? cr.y : lk == 2 ? cr.z : cr.w;
            float sg = lk == 0 ? cg.x : lk == 1 ? cg.y : lk == 2 ? cg.z : cg.w;
            float sb = lk == 0 ? cb.x : lk == 1 ? cb.y : lk == 2 ? cb.z : cb.w;
            float dbk = masked[0] * sr + masked[1] * sg + masked[2] * sb;
            dd0 += dbk * db[k][0];
            dd1 += dbk * db[k][1];
            dd2 += dbk * db[k][2];
        }
        float dot = dir[0] * dd0 + dir[1] * dd1 + dir[2] * dd2;
        dpos[0] += -((dd0 - dir[0] * dot) / len);
        dpos[1] += -((dd1 - dir[1] * dot) / len);
        dpos[2] += -((dd2 - dir[2] * dot) / len);
    }
    g.pos[0] += dpos[0];
    g.pos[1] += dpos[1];
    g.pos[2] += dpos[2];
    g.screen += sqrtf(asx * asx + asy * asy);
}

__device__ __forceinline__ void zero_acc(GradAcc& g) {
#pragma unroll
    for (int k = 0; k < 3; ++k) { g.pos[k] = 0.0f; g.ls[k] = 0.0f; }
#pragma unroll
    for (int k = 0; k < 4; ++k) g.rot[k] = 0.0f;
#pragma unroll
    for (int k = 0; k < 48; ++k) g.sh[k] = 0.0f;
    g.op = 0.0f;
    g.screen = 0.0f;
}

__device__ __forceinline__ void gather_views(const float4* __restrict__ params, int n, int cap, int i, const DevCam* __restrict__ cams,
                                             int nviews, const uint32_t* __restrict__ cnt, const float4* __restrict__ acc,
                                             GradAcc& g) {
    size_t S = (size_t)n * nviews;
    for (int v = 0; v < nviews; ++v) {
        size_t s = (size_t)v * n + i;
        if (cnt[s] == 0) continue;
        float4 a0 = acc[s], a1 = acc[S + s], a2 = acc[2 * S + s];
        geometry_one(params, cap, i, cams[v], a0, a1, a2, g);
    }
}

// Plane p of the gradient (same layout as the parameters).
__device__ __forceinline__ float4 grad_plane(const GradAcc& g, int p) {
    if (p == 0) return make_float4(g.pos[0], g.pos[1], g.pos[2], g.op);
    if (p == 1) return make_float4(g.rot[0], g.rot[1], g.rot[2], g.rot[3]);
    if (p == 2) return make_float4(g.ls[0], g.ls[1], g.ls[2], g.screen);
    int b = (p - 3) * 4;
    return make_float4(g.sh[b], g.sh[b + 1], g.sh[b + 2], g.sh[b + 3]);
}

__global__ void __launch_bounds__(128) k_geometry(const float4* __restrict__ params, int n, int cap, const DevCam* __restrict__ cams,
                                                  int nviews, const uint32_t* __restrict__ cnt, const float4* __restrict__ acc,
                                                  float4* __restrict__ grads, int accumulate) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    GradAcc g;
    zero_acc(g);
    gather_views(params, n, cap, i, cams, nviews, cnt, acc, g);
#pragma unroll
    for (int p = 0; p < NPL; ++p) {
        float4 v = grad_plane(g, p);
        float4* dst = grads + (size_t)p * cap + i;
        if (accumulate) {
            float4 o = *dst;
            v.x += o.x; v.y += o.y; v.z += o.z; v.w += o.w;
        }
        *dst = v;
    }
}

void launch_geometry(const float4* params, int n, int cap, const DevCam* cams, int nviews, const uint32_t* cnt, const float4* acc,
                     float4* grads, int accumulate, cudaStream_t st) {
    if (n <= 0) return;
    k_geometry<<<(n + 127) / 128, 128, 0, st>>>(params, n, cap, cams, nviews, cnt, acc, grads, accumulate);
}

// optimizer.rs:138-162 for one Gaussian, given its 15 gradient planes.
__device__ __forceinline__ float adam_lane(float p, float g, float& m1, float& m2, float lr, const AdamArgs& a, float bc1,
                                           float bc2) {
    m1 = a.b1 * m1 + a.one_minus_b1 * g;
    m2 = a.b2 * m2 + a.one_minus_b2 * g * g;
    float m1h = m1 / bc1;
    float m2h = m2 / bc2;
    float upd = lr * m1h / (sqrtf(m2h) + a.eps);
    return p - upd;
}

template <class GradFn>
__device__ __forceinline__ void adam_gaussian(int i, int cap, const AdamArgs& a, GradFn gf, float screen) {
    const float bc1 = a.bc_dev ? a.bc_dev[0] : a.bc1;
    const float bc2 = a.bc_dev ? a.bc_dev[1] : a.bc2;
#pragma unroll
    for (int p = 0; p < NPL; ++p) {
        size_t o = (size_t)p * cap + i;
        size_t om = (size_t)p * a.mstride + i;
        float4 pv = a.params[o], g = gf(p), m1 = a.m1[om], m2 = a.m2[om];
        const float* lr = a.lr + p * 4;
        pv.x = adam_lane(pv.x, g.x, m1.x, m2.x, lr[0], a, bc1, bc2);
        pv.y = adam_lane(pv.y, g.y, m1.y, m2.y, lr[1], a, bc1, bc2);
        pv.z = adam_lane(pv.z, g.z, m1.z, m2.z, lr[2], a, bc1, bc2);
        if (p != 2) pv.w = adam_lane(pv.w, g.w, m1.w, m2.w, lr[3], a, bc1, bc2);
        if (p == 1) {
            float nrm = sqrtf(pv.x * pv.x + pv.y * pv.y + pv.z * pv.z + pv.w * pv.w);
            if (nrm > 1e-8f) { pv.x /= nrm; pv.y /= nrm; pv.z /= nrm; pv.w /= nrm; }
        }
        a.params[o] = pv;
        a.m1[om] = m1;
        a.m2[om] = m2;
    }
    a.grad_accum[i] += screen;
    a.grad_denom[i] += a.denom_inc;
}

__global__ void __launch_bounds__(128) k_geometry_adam(const DevCam* __restrict__ cams, int nviews, int n, int cap,
                                                       const uint32_t* __restrict__ cnt, const float4* __restrict__ acc, AdamArgs a) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (a.skip_flag && *a.skip_flag) return;
    GradAcc g;
    zero_acc(g);
    gather_views(a.params, n, cap, i, cams, nviews, cnt, acc, g);
    adam_gaussian(i, cap, a, [&](int p) { return grad_plane(g, p); }, g.screen);
}

void launch_geometry_adam(const DevCam* cams, int nviews, int n, int cap, const uint32_t* cnt, const float4* acc, const AdamArgs& a,
                          cudaStream_t st) {
    if (n <= 0) return;
    k_geometry_adam<<<(n + 127) / 128, 128, 0, st>>>(cams, nviews, n, cap, cnt, acc, a);
}

__global__ void __launch_bounds__(256) k_adam(int n, int cap, const float4* __restrict__ grads, AdamArgs a) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (a.skip_flag && *a.skip_flag) return;
    float screen = grads[2 * (size_t)cap + i].w;
    adam_gaussian(i, cap, a, [&](int p) { return grads[(size_t)p * cap + i]; }, screen);
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

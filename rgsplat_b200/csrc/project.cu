// project.cu -- per-(view, Gaussian) projection: culls, EWA covariance, SH
// colour, 3-sigma AABB and CTA-tile count. One thread per slot.
//
// Follows src/cpu/backward.rs:210-280 (`project`), src/math/projection.rs:24-69
// (`project_covariance`) and :138-165 (`gaussian_aabb_2d`), src/math/sh.rs, and
// src/math/mod.rs:66-96. The arithmetic is written in the reference's
// evaluation order and compiled without FMA contraction, so the tile rectangle
// (an integer decision) matches the CPU restatement bit for bit.
#include "rgs_internal.cuh"
#include "rgs_math.cuh"
#include "tiles.cuh"

namespace rgs {

__device__ __forceinline__ void cam_mul(const DevCam& c, const float p[3], float o[3]) {
#pragma unroll
    for (int i = 0; i < 3; ++i)
        o[i] = ((c.view[i * 4 + 0] * p[0] + c.view[i * 4 + 1] * p[1]) + c.view[i * 4 + 2] * p[2]) + c.view[i * 4 + 3] * 1.0f;
}

// projection.rs:24-69; returns (a, b, c) of the low-passed 2D covariance.
__device__ __forceinline__ void project_cov(const M3& sig, const float pc[3], const DevCam& c, float abc[3]) {
    float tx = pc[0], ty = pc[1], tz = fmaxf(pc[2], 0.001f);
    float fx = c.fx, fy = c.fy;
    M3 j = {{{fx / tz, 0.0f, -fx * tx / (tz * tz)}, {0.0f, fy / tz, -fy * ty / (tz * tz)}, {0.0f, 0.0f, 0.0f}}};
    M3 w;
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int k = 0; k < 3; ++k) w.m[r][k] = c.view[r * 4 + k];
    M3 t = mul(j, w);
    M3 s2 = mul(mul(t, sig), tr(t));
    abc[0] = s2.m[0][0] + 0.3f;
    abc[1] = s2.m[0][1];
    abc[2] = s2.m[1][1] + 0.3f;
}

// projection.rs:138-165 with n_sigma = 3. Release-mode Rust wraps `i32 + 1`.
__device__ __forceinline__ bool aabb_2d(float mx, float my, const float abc[3], int w, int h, int box[4]) {
    float a = abc[0], b = abc[1], c = abc[2];
    float mid = (a + c) * 0.5f;
    float disc = sqrtf((a - c) * (a - c) * 0.25f + b * b);
    float l1 = fmaxf(mid + disc, 0.0f);
    float l2 = fmaxf(mid - disc, 0.0f);
    float r = 3.0f * fmaxf(sqrtf(l1), sqrtf(l2));
    int x0 = max(as_i32(mx - r), 0);
    int y0 = max(as_i32(my - r), 0);
    int x1 = min((int)((unsigned)as_i32(mx + r) + 1u), w);
    int y1 = min((int)((unsigned)as_i32(my + r) + 1u), h);
    if (x0 >= x1 || y0 >= y1) return false;
    box[0] = x0; box[1] = y0; box[2] = x1; box[3] = y1;
    return true;
}

struct Projected {
    float sx, sy, opacity, depth;
    float conic[3];
    float color[3];
    float raw[3];
    int box[4];
};

// The view-independent terms of a Gaussian's projection: sigmoid of the
// opacity logit and the 3D covariance M M^T from exp(log-scales) and the
// normalised quaternion. M M^T forms entry (i, j) and (j, i) from the same
// products in the same order, so its six distinct entries hold it exactly.
__device__ __forceinline__ M3 gauss_sigma(const float4* __restrict__ params, int cap, int i) {
    const float4 p1 = params[(size_t)cap + i], p2 = params[2 * (size_t)cap + i];
    const float q[4] = {p1.x, p1.y, p1.z, p1.w};
    const float sc[3] = {exp_cr(p2.x), exp_cr(p2.y), exp_cr(p2.z)};
    return build_cov3d(sc, q);
}

__device__ __forceinline__ M3 cached_sigma(const float4* __restrict__ gcache, int cap, int i) {
    const float4 c0 = gcache[i], c1 = gcache[(size_t)cap + i];
    return M3{{{c0.y, c0.z, c0.w}, {c0.z, c1.x, c1.y}, {c0.w, c1.y, c1.z}}};
}

// One thread per Gaussian, once per step: gcache[i] = (opacity, S00, S01,
// S02), gcache[cap + i] = (S11, S12, S22, 0), so the per-view projection and
// geometry read them instead of evaluating four exponentials and the
// covariance once per view.
__global__ void __launch_bounds__(256) k_gauss_cache(const float4* __restrict__ params, int n, int cap,
                                                     float4* __restrict__ gcache) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float opacity = sigmoid(params[i].w);
    const M3 sig = gauss_sigma(params, cap, i);
    gcache[i] = make_float4(opacity, sig.m[0][0], sig.m[0][1], sig.m[0][2]);
    gcache[(size_t)cap + i] = make_float4(sig.m[1][1], sig.m[1][2], sig.m[2][2], 0.0f);
}

void launch_gauss_cache(const float4* params, int n, int cap, float4* gcache, cudaStream_t st) {
    if (n > 0) k_gauss_cache<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(params, n, cap, gcache);
}

// backward.rs:210-280. Returns false when the Gaussian is culled. With a
// non-null gcache (k_gauss_cache of the same parameters) the opacity and the
// 3D covariance are read from it.
template <bool FULL>
__device__ __forceinline__ bool project_one(const float4* __restrict__ params, int cap, int i, const DevCam& c, Projected& o,
                                            const float4* __restrict__ gcache = nullptr) {
    float4 p0 = params[i];
    float opacity = gcache ? gcache[i].x : sigmoid(p0.w);
    if (opacity < 1.0f / 255.0f) return false;
    float pos[3] = {p0.x, p0.y, p0.z};
    float pc[3];
    cam_mul(c, pos, pc);
    float tz = pc[2];
    if (tz <= 0.001f) return false;
    float sx = c.fx * pc[0] / tz + c.cx;
    float sy = c.fy * pc[1] / tz + c.cy;
    const float margin = 128.0f;
    if (sx < -margin || sx > (float)c.width + margin || sy < -margin || sy > (float)c.height + margin) return false;
    const M3 sig = gcache ? cached_sigma(gcache, cap, i) : gauss_sigma(params, cap, i);
    float abc[3];
    project_cov(sig, pc, c, abc);
    float a = abc[0], b = abc[1], cc = abc[2];
    float det = a * cc - b * b;
    if (fabsf(det) < 1e-8f) return false;
    float inv_det = 1.0f / det;
    if (FULL) {
        float d[3], basis[16];
        view_dir(pos, c.pos, d);
        sh_basis(d, basis);
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
            o.raw[ch] = 0.5f + acc;
            o.color[ch] = rclamp(o.raw[ch], 0.0f, 1.0f);
        }
    }
    if (!aabb_2d(sx, sy, abc, c.width, c.height, o.box)) return false;
    o.sx = sx;
    o.sy = sy;
    o.opacity = opacity;
    o.depth = tz;
    o.conic[0] = cc * inv_det;
    o.conic[1] = -b * inv_det;
    o.conic[2] = a * inv_det;
    return true;
}

// Five 256-thread CTAs per SM (register budget capped at 48: a few spilled
// words cost less than the extra warps hide; measured 9 % faster). About 40 %
// of the slots are culled early, so a warp runs on about half its lanes; a
// split into a cull pass that lists the survivors and a full pass over them
// on whole warps measured slower (0.72 against 0.60 ms: the extra pass over
// every slot cost 0.19 ms and the full pass saved only 0.07).
__global__ void __launch_bounds__(256, 5) k_project(const float4* __restrict__ params, int n, int cap,
                                                 const DevCam* __restrict__ cams, int nviews, int tile_w,
                                                 int tile_h, float4* __restrict__ rec, uint32_t* __restrict__ cnt,
                                                 uint2* __restrict__ tdesc, uint32_t* __restrict__ dkey,
                                                 uint32_t* __restrict__ ids, int prune, uint32_t* __restrict__ visible,
                                                 const float4* __restrict__ gcache, uint4* __restrict__ spans) {
    // chunk-major grid: the nviews consecutive blocks project the same 256
    // Gaussians into every view, so the per-Gaussian reads (SH, position,
    // cached terms) of all but the first view come from L2
    const size_t S = (size_t)n * nviews;
    const int v = (int)(blockIdx.x % (unsigned)nviews);
    const int i = (int)((blockIdx.x / (unsigned)nviews) * blockDim.x + threadIdx.x);
    if (i >= n) return;
    const size_t s = (size_t)v * n + i;
    const DevCam& c = cams[v];
    ids[s] = (uint32_t)s;
    Projected o;
    if (!project_one<true>(params, cap, i, c, o, gcache)) {
        cnt[s] = 0;
        tdesc[s] = make_uint2(0u, 0u);
        dkey[s] = 0xFFFFFFFFu;
        return;
    }
    // Reference tile rectangle (backward.rs:275-278), expressed in pixels so
    // that any CTA tile shape can test membership per pixel.
    int rtx0 = o.box[0] / REF_TILE, rty0 = o.box[1] / REF_TILE;
    int rtx1 = (o.box[2] + REF_TILE - 1) / REF_TILE, rty1 = (o.box[3] + REF_TILE - 1) / REF_TILE;
    int x0 = rtx0 * REF_TILE, y0 = rty0 * REF_TILE;
    int x1 = min(rtx1 * REF_TILE, c.width), y1 = min(rty1 * REF_TILE, c.height);
    int ctx0 = x0 / tile_w, cty0 = y0 / tile_h;
    int ctx1 = (x1 + tile_w - 1) / tile_w, cty1 = (y1 + tile_h - 1) / tile_h;
    rec[s] = make_float4(o.sx, o.sy, o.opacity, o.depth);
    rec[S + s] = make_float4(o.conic[0], o.conic[1], o.conic[2], __uint_as_float((uint32_t)x0 | ((uint32_t)x1 << 16)));
    rec[2 * S + s] = make_float4(o.color[0], o.color[1], o.color[2], __uint_as_float((uint32_t)y0 | ((uint32_t)y1 << 16)));
    uint32_t count = (uint32_t)((ctx1 - ctx0) * (cty1 - cty0));
    if (prune) {
        // only the tiles of each row's kept span (tiles.cuh); rectangles of
        // at most SPAN_ROWS rows and 15 columns keep their spans packed for
        // the tile lists (byte r: first kept column - ctx0 | count << 4)
        const SpanSetup u = span_setup(o.sx, o.sy, o.conic[0], o.conic[1], o.conic[2], power_floor(o.opacity));
        const bool pack = ctx1 - ctx0 <= 15 && cty1 - cty0 <= SPAN_ROWS;
        unsigned long long lo = 0, hi = 0;
        count = 0;
        for (int ty = cty0; ty < cty1; ++ty) {
            int c0, c1;
            kept_cols(u, ty, tile_w, tile_h, c.height, ctx0, ctx1, c0, c1);
            count += (uint32_t)(c1 - c0);
            const unsigned long long b = (uint32_t)(c0 - ctx0) | ((uint32_t)(c1 - c0) << 4);
            const int r = ty - cty0;
            if (pack) {
                if (r < 8) lo |= b << (8 * r);
                else hi |= b << (8 * (r - 8));
            }
        }
        spans[2 * s] = pack ? make_uint4((uint32_t)lo, (uint32_t)(lo >> 32), (uint32_t)hi, (uint32_t)(hi >> 32))
                            : make_uint4(SPANS_NONE, SPANS_NONE, SPANS_NONE, SPANS_NONE);
    }
    cnt[s] = count;
    if (count) {
        // slots with tile pairs, one atomic per group of converged lanes
        const unsigned m = __activemask();
        if ((threadIdx.x & 31) == __ffs(m) - 1) atomicAdd(visible, (uint32_t)__popc(m));
    }
    const uint2 td = make_uint2((uint32_t)(c.tile_base + cty0 * c.tiles_x + ctx0),
                                (uint32_t)(ctx1 - ctx0) | ((uint32_t)(cty1 - cty0) << 16));
    tdesc[s] = td;
    // with prune, the tile rectangle again beside the spans: the tile-list
    // masks gather one 32-byte record per entry
    if (prune) spans[2 * s + 1] = make_uint4(td.x, td.y, 0u, 0u);
    dkey[s] = __float_as_uint(o.depth);
}

void launch_project(const float4* params, int n, int cap, const DevCam* cams, int nviews, int tile_w, int tile_h,
                    float4* rec, uint32_t* cnt, uint2* tdesc, uint32_t* dkey, uint32_t* ids, int prune, uint32_t* visible,
                    float4* gcache, uint4* spans, cudaStream_t st) {
    size_t S = (size_t)n * nviews;
    if (S == 0) return;
    launch_gauss_cache(params, n, cap, gcache, st);
    unsigned blocks = (unsigned)(((size_t)n + 255) / 256 * (size_t)nviews);
    k_project<<<blocks, 256, 0, st>>>(params, n, cap, cams, nviews, tile_w, tile_h, rec, cnt, tdesc, dkey, ids, prune, visible,
                                      gcache, spans);
}

// ---------------------------------------------------------------------------
// GpuRenderer::project drop-in (src/gpu/compute.rs:140-207, splat.wgsl:119-191):
// one SplatInfo2D (40 B) and one u32 depth key per Gaussian, culled entries all
// zero with key 0xFFFFFFFF. cpu_math = 0 reproduces the shader's arithmetic
// (DC-only colour, no normalisation of q, J built column-major, i.e. the
// transpose of the CPU path's J); cpu_math = 1 returns the CPU path's splat
// (full degree-3 SH, all culls of backward.rs:210-280).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_project_wgsl(const float4* __restrict__ params, int n, int cap,
                                                      const DevCam* __restrict__ cam, int cpu_math,
                                                      float* __restrict__ out, uint32_t* __restrict__ keys) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const DevCam& c = *cam;
    float* o = out + (size_t)i * 10;
#pragma unroll
    for (int k = 0; k < 10; ++k) o[k] = 0.0f;
    if (cpu_math) {
        Projected p;
        if (!project_one<true>(params, cap, i, c, p)) { keys[i] = 0xFFFFFFFFu; return; }
        o[0] = p.sx; o[1] = p.sy; o[2] = p.conic[0]; o[3] = p.conic[1]; o[4] = p.conic[2];
        o[5] = p.color[0]; o[6] = p.color[1]; o[7] = p.color[2]; o[8] = p.opacity; o[9] = p.depth;
        keys[i] = ~__float_as_uint(p.depth);
        return;
    }
    float4 p0 = params[i];
    float pos[3] = {p0.x, p0.y, p0.z};
    float pc[3];
    cam_mul(c, pos, pc);
    float tz = pc[2];
    if (tz <= 0.001f) { keys[i] = 0xFFFFFFFFu; return; }
    float alpha = 1.0f / (1.0f + exp_cr(-p0.w));
    if (alpha < 1.0f / 255.0f) { keys[i] = 0xFFFFFFFFu; return; }
    float sx = c.fx * pc[0] / tz + c.cx;
    float sy = c.fy * pc[1] / tz + c.cy;
    float4 p1 = params[(size_t)cap + i];
    float4 p2 = params[2 * (size_t)cap + i];
    float w = p1.x, x = p1.y, y = p1.z, z = p1.w;
    M3 R;
    R.m[0][0] = 1.0f - 2.0f * (y * y + z * z); R.m[1][0] = 2.0f * (x * y + w * z); R.m[2][0] = 2.0f * (x * z - w * y);
    R.m[0][1] = 2.0f * (x * y - w * z); R.m[1][1] = 1.0f - 2.0f * (x * x + z * z); R.m[2][1] = 2.0f * (y * z + w * x);
    R.m[0][2] = 2.0f * (x * z + w * y); R.m[1][2] = 2.0f * (y * z - w * x); R.m[2][2] = 1.0f - 2.0f * (x * x + y * y);
    float s0 = exp_cr(p2.x), s1 = exp_cr(p2.y), s2 = exp_cr(p2.z);
    M3 S = {{{s0, 0.0f, 0.0f}, {0.0f, s1, 0.0f}, {0.0f, 0.0f, s2}}};
    M3 RS = mul(R, S);
    M3 sig = mul(RS, tr(RS));
    float tx = pc[0], ty = pc[1], fx = c.fx, fy = c.fy;
    M3 J = {{{fx / tz, 0.0f, 0.0f}, {0.0f, fy / tz, 0.0f}, {-fx * tx / (tz * tz), -fy * ty / (tz * tz), 0.0f}}};
    M3 W;
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int k = 0; k < 3; ++k) W.m[r][k] = c.view[r * 4 + k];
    M3 T = mul(J, W);
    M3 s2m = mul(mul(T, sig), tr(T));
    float a = s2m.m[0][0] + 0.3f;
    float b = s2m.m[1][0];
    float cc = s2m.m[1][1] + 0.3f;
    float det = a * cc - b * b;
    if (fabsf(det) < 1e-8f) { keys[i] = 0xFFFFFFFFu; return; }
    float inv_det = 1.0f / det;
    float4 sh0 = params[3 * (size_t)cap + i];
    float4 sh4 = params[7 * (size_t)cap + i];
    float4 sh8 = params[11 * (size_t)cap + i];
    o[0] = sx; o[1] = sy;
    o[2] = cc * inv_det; o[3] = -b * inv_det; o[4] = a * inv_det;
    o[5] = rclamp(0.5f + sh0.x * SH_C0, 0.0f, 1.0f);
    o[6] = rclamp(0.5f + sh4.x * SH_C0, 0.0f, 1.0f);
    o[7] = rclamp(0.5f + sh8.x * SH_C0, 0.0f, 1.0f);
    o[8] = alpha;
    o[9] = tz;
    keys[i] = ~__float_as_uint(tz);
}

void launch_project_wgsl(const float4* params, int n, int cap, const DevCam* cam, int cpu_math, float* splats10,
                         uint32_t* keys, cudaStream_t st) {
    if (n <= 0) return;
    k_project_wgsl<<<(n + 255) / 256, 256, 0, st>>>(params, n, cap, cam, cpu_math, splats10, keys);
}

// GpuRenderer::render's CPU compositor (src/gpu/compute.rs:243-296, with
// depth_order of src/gpu/sort.rs:10-17) expressed as splat records for the
// tile pipeline: a splat is drawn iff alpha >= 1/255 and depth > 0, over the
// pixel box floor(s - r) .. ceil(s + r) with r = 3 / sqrt(lambda_min(conic)).
// The blend kernel then tests each pixel against that box (RECT mode).
__global__ void __launch_bounds__(256) k_composite_prepare(const float* __restrict__ sp, int n, const DevCam* __restrict__ cam,
                                                           int tile_w, int tile_h, float4* __restrict__ rec,
                                                           uint32_t* __restrict__ cnt, uint2* __restrict__ tdesc,
                                                           uint32_t* __restrict__ dkey, uint32_t* __restrict__ ids) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    ids[i] = (uint32_t)i;
    const float* s = sp + (size_t)i * 10;
    const int w = cam->width, h = cam->height;
    cnt[i] = 0;
    tdesc[i] = make_uint2(0u, 0u);
    dkey[i] = 0xFFFFFFFFu;
    if (!(s[8] >= 1.0f / 255.0f && s[9] > 0.0f)) return;
    float a = s[2], b = s[3], c = s[4];
    float mid = 0.5f * (a + c);
    float disc = sqrtf(0.25f * (a - c) * (a - c) + b * b);
    float lmin = fmaxf(mid - disc, 1e-6f);
    float rad = 3.0f * sqrtf(1.0f / lmin);
    // Rust `as usize` / `as i64` saturate and map NaN to 0
    float fx0 = fmaxf(floorf(s[0] - rad), 0.0f), fy0 = fmaxf(floorf(s[1] - rad), 0.0f);
    float fx1 = ceilf(s[0] + rad), fy1 = ceilf(s[1] + rad);
    int x0 = fx0 != fx0 ? 0 : (fx0 >= (float)w ? w : (int)fx0);
    int y0 = fy0 != fy0 ? 0 : (fy0 >= (float)h ? h : (int)fy0);
    int x1 = fx1 != fx1 ? 0 : (fx1 <= 0.0f ? 0 : (fx1 >= (float)w ? w : (int)fx1));
    int y1 = fy1 != fy1 ? 0 : (fy1 <= 0.0f ? 0 : (fy1 >= (float)h ? h : (int)fy1));
    if (x0 >= x1 || y0 >= y1) return;
    int ctx0 = x0 / tile_w, cty0 = y0 / tile_h;
    int ctx1 = (x1 + tile_w - 1) / tile_w, cty1 = (y1 + tile_h - 1) / tile_h;
    rec[i] = make_float4(s[0], s[1], s[8], s[9]);
    rec[(size_t)n + i] = make_float4(a, b, c, __uint_as_float((uint32_t)x0 | ((uint32_t)x1 << 16)));
    rec[2 * (size_t)n + i] = make_float4(s[5], s[6], s[7], __uint_as_float((uint32_t)y0 | ((uint32_t)y1 << 16)));
    cnt[i] = (uint32_t)((ctx1 - ctx0) * (cty1 - cty0));
    tdesc[i] = make_uint2((uint32_t)(cam->tile_base + cty0 * cam->tiles_x + ctx0),
                          (uint32_t)(ctx1 - ctx0) | ((uint32_t)(cty1 - cty0) << 16));
    dkey[i] = __float_as_uint(s[9]);
}

void launch_composite_prepare(const float* splats10, int n, const DevCam* cam, int tile_w, int tile_h, float4* rec,
                              uint32_t* cnt, uint2* tdesc, uint32_t* dkey, uint32_t* ids, cudaStream_t st) {
    if (n <= 0) return;
    k_composite_prepare<<<(n + 255) / 256, 256, 0, st>>>(splats10, n, cam, tile_w, tile_h, rec, cnt, tdesc, dkey, ids);
}

}  // namespace rgs

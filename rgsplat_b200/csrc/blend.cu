// blend.cu -- per-tile alpha blending (forward) and its analytic reverse pass.
//
// Forward follows src/cpu/backward.rs:296-385 (`forward_pass`): per pixel, walk
// the tile's depth-ordered list; power = -1/2 d^T conic d; skip power > 0;
// alpha = min(opacity * e^power, 0.99); skip alpha < 1/255; composite
// front-to-back; stop after the update that drops T below 1e-4; output
// C + T * bg, the final T and the index of the last contributor.
// Backward follows backward.rs:391-512 (`backward_pass`): from the last
// contributor down to 0, rebuild T by T /= (1 - alpha) -- no per-Gaussian
// blend state is stored -- and accumulate d color, d opacity, d conic and
// d mean per splat.
//
// B200 mapping: one CTA per CTA tile (TW x TH pixels, one pixel per thread),
// persistent CTAs pulling tiles of every view of the batch from one atomic
// counter. Splat records are staged BATCH at a time in shared memory and read
// by all threads as broadcasts. The kernels are issue-bound, so work that the
// reference's own tests would discard is removed without changing any result:
//   * per splat, alpha < 1/255 is guaranteed once power < thr with
//     thr = ln(1 / (255 opacity)) - 0.01, so such pixels skip exp;
//   * per (tile, splat), if the conic's quadratic form is bounded below over
//     the box of the tile's pixel centres so that power < thr everywhere, the
//     splat is dropped from the staged batch (the batch is compacted, keeping
//     each splat's index in the full tile list for last_contrib);
//   * backward: per (warp, staged splat), the same test on the box of the
//     warp's own strip of pixel rows; a warp whose strip the splat cannot
//     reach skips it (warp-uniform). (The same skip in the forward measured
//     slower, as a per-splat branch and as a per-warp list of the needed
//     splats alike: a pair that does not contribute costs the packed forward
//     about five instructions per pixel, less than the strip tests add to
//     every staging round.)
//   * backward warps skip splats past the warp's largest last_contrib.
// Backward pre-reduces each splat's 9 partial gradients across the warp with
// shuffles (only when a lane contributed), across warps with shared-memory
// atomics, and issues one 3 x 16-byte vector reduction (red.global.add.v4.f32)
// per splat per CTA.
//
// CTA tiles other than 16x16 keep the reference's per-pixel semantics: each
// record carries its reference-tile rectangle in pixels and a pixel only
// evaluates splats whose rectangle contains it (RECT = true).
#include <algorithm>
#include <mutex>

#include "rgs_internal.cuh"
#include "rgs_math.cuh"
#include "tiles.cuh"

namespace rgs {

__device__ __forceinline__ int find_view(const DevCam* cams, int nviews, int tile) {
    int v = 0;
    while (v + 1 < nviews && cams[v + 1].tile_base <= tile) ++v;
    return v;
}

__device__ __forceinline__ bool in_rect(float rx, float ry, int px, int py) {
    uint32_t x = __float_as_uint(rx), y = __float_as_uint(ry);
    return px >= (int)(x & 0xffffu) && px < (int)(x >> 16) && py >= (int)(y & 0xffffu) && py < (int)(y >> 16);
}

// Stages the tile-list entries [first, end) (at most BATCH) into shared memory,
// dropping splats the tile test rejects; returns the kept count (block-uniform).
// li0 is the tile-list index of `first`. Must be called by the whole block.
// When s_rall is given, every staged entry's pixel rectangle (kept or not) is
// recorded at its batch position.
template <int NT, int BATCH, int RW, bool WMASK>
__device__ __forceinline__ int stage_batch(const BlendArgs& a, size_t S, uint32_t first, uint32_t end, int li0, float x0c,
                                           float x1c, float y0c, float y1c, int ytile, int height, float4* s_a, float4* s_c,
                                           float4* s_k, int* s_li, uint8_t* s_wm, uint32_t* s_slot, int* s_wsum, uint2* s_rall) {
    constexpr int NW = NT / 32;
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    int kept = 0;
#pragma unroll
    for (int c0 = 0; c0 < BATCH; c0 += NT) {
        const int j = c0 + tid;
        const uint32_t idx = first + (uint32_t)j;
        bool keep = false;
        float4 A, Q, K;
        uint32_t slot = 0, wm = 0;
        if (j < BATCH && idx < end) {
            slot = a.pair_vals[idx];
            A = a.rec[slot];
            Q = a.rec[S + slot];
            K = a.rec[2 * S + slot];
            A.w = power_floor(A.z);
            const TileTest t = tile_test_setup(A.x, A.y, Q.x, Q.y, Q.z, A.w);
            keep = !tile_rejects(t, x0c, x1c, y0c, y1c);
            if (WMASK && keep) {
                // warp ww owns pixel rows [ww*RW, ww*RW + RW) of the tile: keep the
                // warps the tile test cannot reject on their own strip of pixel
                // centres (strips past the image hold no pixel)
#pragma unroll
                for (int ww = 0; ww < NW; ++ww) {
                    const int r0 = ytile + ww * RW;
                    if (r0 >= height) continue;
                    const float sy0 = (float)r0 + 0.5f, sy1 = (float)(min(r0 + RW, height) - 1) + 0.5f;
                    if (!tile_rejects(t, x0c, x1c, sy0, sy1)) wm |= 1u << ww;
                }
            }
            if (s_rall) s_rall[j] = make_uint2(__float_as_uint(Q.w), __float_as_uint(K.w));
        }
        const unsigned m = __ballot_sync(0xffffffffu, keep);
        if (lane == 0) s_wsum[w] = __popc(m);
        __syncthreads();
        int off = kept, total = 0;
#pragma unroll
        for (int k = 0; k < NW; ++k) {
            const int t = s_wsum[k];
            off += k < w ? t : 0;
            total += t;
        }
        if (keep) {
            const int p = off + __popc(m & ((1u << lane) - 1u));
            s_a[p] = A;
            s_c[p] = Q;
            s_k[p] = K;
            s_li[p] = li0 + j;
            if (WMASK) s_wm[p] = (uint8_t)wm;
            if (s_slot) s_slot[p] = slot;
        }
        kept += total;
        __syncthreads();
    }
    return kept;
}

// Forward. PPT vertically adjacent pixels per thread share dx and the
// dx-only products of power, which are evaluated once per (splat, thread) in
// the reference's rounding order.
// The TW threads that share a pixel row would each form dy and Q.z*dy*dy for
// every splat; where the shared memory allows (ROWTERMS), the CTA forms them
// once per (staged splat, tile row) after staging, with the same operations.
template <int BATCH, int TH, int PPT>
struct RowTerms {
    static constexpr bool on = BATCH * TH <= 2048 && PPT % 2 == 0;
};

template <int TW, int TH, int BATCH, bool RECT, int PPT, bool STORE = false>
__global__ void __launch_bounds__(TW * TH / PPT) k_blend_fwd(BlendArgs a) {
    constexpr int NT = TW * TH / PPT;
    constexpr bool ROWTERMS = RowTerms<BATCH, TH, PPT>::on;
    // two pixels per thread in packed f32x2 lanes (the store-all study keeps
    // the scalar loop)
    constexpr bool PACK = PPT == 2 && !STORE;
    const float2 one2 = make_float2(a.one, a.one);
    __shared__ float4 s_a[BATCH];
    __shared__ float4 s_c[BATCH];
    __shared__ float4 s_k[BATCH];
    __shared__ int s_li[BATCH];
    __shared__ int s_wsum[NT / 32];
    __shared__ uint2 s_rall[RECT ? BATCH : 1];
    __shared__ __align__(16) float2 s_row[ROWTERMS ? BATCH : 1][ROWTERMS ? TH : 1];  // (dy, Q.z*dy*dy)
    __shared__ int s_tile;
    constexpr int RW = (32 / TW) * PPT;  // pixel rows per warp
    const int tid = threadIdx.x;
    const int total_tiles = a.total_tiles ? (int)*a.total_tiles : a.total_tiles_host;
    const size_t S = (size_t)a.n_per_view * a.nviews;
    for (;;) {
        if (tid == 0) s_tile = (int)atomicAdd(a.work, 1u);
        __syncthreads();
        const int tile = s_tile;
        if (tile >= total_tiles) break;
        const int v = find_view(a.cams, a.nviews, tile);
        const DevCam& c = a.cams[v];
        const int lt = tile - c.tile_base;
        const int tx = lt % c.tiles_x, ty = lt / c.tiles_x;
        const int px = tx * TW + (tid % TW), py0 = ty * TH + (tid / TW) * PPT;
        const float pxf = (float)px + 0.5f;
        // box of the tile's pixel centres
        const float x0c = (float)(tx * TW) + 0.5f, x1c = (float)(min(tx * TW + TW, c.width) - 1) + 0.5f;
        const float y0c = (float)(ty * TH) + 0.5f, y1c = (float)(min(ty * TH + TH, c.height) - 1) + 0.5f;
        const uint2 rg = a.ranges[tile];
        float T[PPT], C0[PPT], C1[PPT], C2[PPT], pyc[PPT];
        int last[PPT];
        bool done[PPT], seen[PPT];
        bool all_done = true;
#pragma unroll
        for (int p = 0; p < PPT; ++p) {
            pyc[p] = (float)(py0 + p) + 0.5f;
            T[p] = 1.0f;
            C0[p] = a.bg_start ? a.bg[0] : 0.0f;
            C1[p] = a.bg_start ? a.bg[1] : 0.0f;
            C2[p] = a.bg_start ? a.bg[2] : 0.0f;
            last[p] = -1;
            done[p] = !(px < c.width && py0 + p < c.height);
            all_done &= done[p];
            // whether the pixel's reference tile list is non-empty
            seen[p] = !RECT && rg.y > rg.x;
        }
        for (uint32_t b0 = rg.x; b0 < rg.y; b0 += BATCH) {
            if (__syncthreads_count(!all_done) == 0) break;
            const bool need_seen = RECT && a.empty_tile_black;
            const int nb = stage_batch<NT, BATCH, RW, false>(a, S, b0, rg.y, (int)(b0 - rg.x), x0c, x1c, y0c, y1c, ty * TH,
                                                             c.height, s_a, s_c, s_k, s_li, nullptr, nullptr, s_wsum,
                                                             need_seen ? s_rall : nullptr);
            if (need_seen) {
                // a pixel's reference tile list is non-empty iff some entry (kept
                // or rejected) covers the pixel
                const int staged = (int)min((uint32_t)BATCH, rg.y - b0);
#pragma unroll
                for (int p = 0; p < PPT; ++p)
                    for (int j = 0; j < staged && !seen[p]; ++j)
                        if (in_rect(__uint_as_float(s_rall[j].x), __uint_as_float(s_rall[j].y), px, py0 + p)) seen[p] = true;
            }
            if (ROWTERMS) {
                for (int idx = tid; idx < nb * TH; idx += NT) {
                    const int k = idx / TH, r = idx - k * TH;
                    const float dy = ((float)(ty * TH + r) + 0.5f) - s_a[k].y;
                    s_row[k][r] = make_float2(dy, s_c[k].z * dy * dy);
                }
                __syncthreads();
            }
            const int rbase = (tid / TW) * PPT;  // this thread's first row in the tile
            for (int k = 0; k < nb && !all_done; ++k) {
                const float4 A = s_a[k];
                const float4 Q = s_c[k];
                const float dx = pxf - A.x;
                const float tdx = Q.x * dx * dx;
                const float t2b = 2.0f * Q.y * dx;
                float4 rw[(PPT + 1) / 2];  // two rows' (dy, Q.z*dy*dy) per 16-byte load
#pragma unroll
                for (int h = 0; h < (PPT + 1) / 2; ++h)
                    rw[h] = ROWTERMS ? *reinterpret_cast<const float4*>(&s_row[k][rbase + 2 * h]) : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                if (PACK && !a.bg_start) {
                    // both pixels in packed f32x2 lanes, each lane rounded exactly as
                    // the scalar loop below rounds that pixel; a pixel that does not
                    // take this splat gets alpha = 0, which leaves its colour
                    // (+0 added to a non-negative sum) and T (times 1) unchanged
                    float2 dy2, qdd2;
                    if (ROWTERMS) {
                        dy2 = make_float2(rw[0].x, rw[0].z);
                        qdd2 = make_float2(rw[0].y, rw[0].w);
                    } else {
                        dy2 = __fadd2_rn(make_float2(pyc[0], pyc[PPT > 1 ? 1 : 0]), bc2(-A.y));
                        qdd2 = __fmul2_rn(__fmul2_rn(bc2(Q.z), dy2), dy2);
                    }
                    // power = -0.5 * ((tdx + t2b * dy) + qdd)
                    const float2 s1 = __ffma2_rn(__fmul2_rn(bc2(t2b), dy2), one2, bc2(tdx));
                    const float2 s2 = ROWTERMS ? __fadd2_rn(s1, qdd2) : __ffma2_rn(qdd2, one2, s1);
                    const float2 pw = __fmul2_rn(s2, bc2(-0.5f));
                    bool act0 = !done[0] && !(pw.x > 0.0f) && !(pw.x < A.w);
                    bool act1 = !done[PPT > 1 ? 1 : 0] && !(pw.y > 0.0f) && !(pw.y < A.w);
                    if (RECT) {
                        act0 = act0 && in_rect(Q.w, s_k[k].w, px, py0);
                        act1 = act1 && in_rect(Q.w, s_k[k].w, px, py0 + 1);
                    }
                    if (act0 || act1) {
                        const float2 ar = __fmul2_rn(bc2(A.z), expf_fast_nonpos2(pw, one2));
                        float al0 = fminf(ar.x, 0.99f), al1 = fminf(ar.y, 0.99f);
                        act0 = act0 && !(al0 < 1.0f / 255.0f);
                        act1 = act1 && !(al1 < 1.0f / 255.0f);
                        if (act0 || act1) {
                            const float4 K = s_k[k];
                            const float2 al = make_float2(act0 ? al0 : 0.0f, act1 ? al1 : 0.0f);
                            float2 T2 = make_float2(T[0], T[PPT > 1 ? 1 : 0]);
                            const float2 w = __fmul2_rn(al, T2);
                            const float2 c0 = __ffma2_rn(__fmul2_rn(bc2(K.x), w), one2, make_float2(C0[0], C0[PPT > 1 ? 1 : 0]));
                            const float2 c1 = __ffma2_rn(__fmul2_rn(bc2(K.y), w), one2, make_float2(C1[0], C1[PPT > 1 ? 1 : 0]));
                            const float2 c2 = __ffma2_rn(__fmul2_rn(bc2(K.z), w), one2, make_float2(C2[0], C2[PPT > 1 ? 1 : 0]));
                            T2 = __fmul2_rn(T2, __ffma2_rn(al, make_float2(-one2.x, -one2.y), one2));
                            C0[0] = c0.x; C1[0] = c1.x; C2[0] = c2.x; T[0] = T2.x;
                            C0[PPT - 1] = c0.y; C1[PPT - 1] = c1.y; C2[PPT - 1] = c2.y; T[PPT - 1] = T2.y;
                            const int li = s_li[k];
                            if (act0) {
                                last[0] = li;
                                if (T2.x < 1e-4f) done[0] = true;
                            }
                            if (act1) {
                                last[PPT - 1] = li;
                                if (T2.y < 1e-4f) done[PPT - 1] = true;
                            }
                        }
                    }
                } else {
#pragma unroll
                for (int p = 0; p < PPT; ++p) {
                    if (done[p]) continue;
                    if (RECT && !in_rect(Q.w, s_k[k].w, px, py0 + p)) continue;
                    float dy, qdd;
                    if (ROWTERMS) {
                        dy = (p & 1) ? rw[p >> 1].z : rw[p >> 1].x;
                        qdd = (p & 1) ? rw[p >> 1].w : rw[p >> 1].y;
                    } else {
                        dy = pyc[p] - A.y;
                        qdd = Q.z * dy * dy;
                    }
                    const float power = -0.5f * (tdx + t2b * dy + qdd);
                    if (power > 0.0f || power < A.w) continue;
                    const float alpha = fminf(A.z * expf_fast_nonpos(power), 0.99f);
                    if (alpha < 1.0f / 255.0f) continue;
                    const float4 K = s_k[k];
                    if (STORE) a.tstore[(size_t)(rg.x + (uint32_t)s_li[k]) * (TW * TH) + (tid / TW) * PPT * TW + p * TW + tid % TW] = T[p];
                    const float weight = alpha * T[p];
                    C0[p] += K.x * weight;
                    C1[p] += K.y * weight;
                    C2[p] += K.z * weight;
                    T[p] *= 1.0f - alpha;
                    last[p] = s_li[k];
                    if (T[p] < 1e-4f) done[p] = true;
                }
                }
                all_done = true;
#pragma unroll
                for (int p = 0; p < PPT; ++p) all_done &= done[p];
            }
            __syncthreads();
        }
#pragma unroll
        for (int p = 0; p < PPT; ++p) {
            const int py = py0 + p;
            if (px < c.width && py < c.height) {
                size_t pix = (size_t)c.pix_base + (size_t)py * c.width + px;
                // forward_pass skips tiles whose list is empty, leaving their pixels
                // at 0 rather than bg (src/cpu/backward.rs:313-315, 124)
                const bool black = a.empty_tile_black && !seen[p];
                a.rgb[pix * 3 + 0] = black ? 0.0f : a.bg_start ? C0[p] : C0[p] + T[p] * a.bg[0];
                a.rgb[pix * 3 + 1] = black ? 0.0f : a.bg_start ? C1[p] : C1[p] + T[p] * a.bg[1];
                a.rgb[pix * 3 + 2] = black ? 0.0f : a.bg_start ? C2[p] : C2[p] + T[p] * a.bg[2];
                a.final_t[pix] = T[p];
                a.last[pix] = last[p];
            }
        }
        __syncthreads();
    }
}


// Warp sum of nine per-lane values, added into dst[0..8] in shared memory.
// Values 0..7 are reduced with a transpose (reduce-scatter) pattern: at each
// xor step a lane keeps half of its values and trades the other half, so after
// three steps lane l holds value l >> 2 summed over the lanes that differ in
// bits 4..2, and two more steps finish it: 14 shuffles in place of 45, and
// eight lanes then add distinct addresses in one instruction.
__device__ __forceinline__ void warp_reduce_scatter9(const float (&g)[9], int lane, float* dst) {
    const bool b4 = lane & 16, b3 = lane & 8, b2 = lane & 4;
    float w[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const float send = b4 ? g[i] : g[i + 4];
        const float keep = b4 ? g[i + 4] : g[i];
        w[i] = keep + __shfl_xor_sync(0xffffffffu, send, 16);
    }
    float x[2];
#pragma unroll
    for (int i = 0; i < 2; ++i) {
        const float send = b3 ? w[i] : w[i + 2];
        const float keep = b3 ? w[i + 2] : w[i];
        x[i] = keep + __shfl_xor_sync(0xffffffffu, send, 8);
    }
    float y = (b2 ? x[1] : x[0]) + __shfl_xor_sync(0xffffffffu, b2 ? x[0] : x[1], 4);
    y += __shfl_xor_sync(0xffffffffu, y, 2);
    y += __shfl_xor_sync(0xffffffffu, y, 1);
    float z = g[8];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) z += __shfl_xor_sync(0xffffffffu, z, o);
    if ((lane & 3) == 0) atomicAdd(dst + (lane >> 2), y);
    if (lane == 0) atomicAdd(dst + 8, z);
}

__device__ __forceinline__ void red_add_v4(float4* addr, float x, float y, float z, float w) {
    asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(addr), "f"(x), "f"(y), "f"(z), "f"(w) : "memory");
}


// Backward. A thread owns PPT vertical pixels; their gradient contributions to
// a splat are summed in registers before the warp reduction. T is rebuilt as
// T * 1/(1 - alpha) with the hardware reciprocal (within 2 ulp; one reciprocal
// serves both uses, where the reference divides, backward.rs:452): over the
// at most few hundred splats a pixel rebuilds through, T stays within ~1e-5
// relative of the reference's, far inside the gradients' 1e-3 tolerance.
// Alpha is formed with the SFU exponential (within 1e-6 of the forward's
// value); wherever that value lies within 4e-6 relative of the 1/255 cut or
// the 0.99 clamp, the forward's exact exp decides instead, so the set of
// contributing splats and the clamped ones are exactly the forward's.
// The register budget is capped for occupancy: eight 128-thread CTAs per SM
// with two pixels per thread, twelve 64-thread CTAs with four (a few spilled
// words cost less than the lost warps: measured 2 % and 10 % faster backward
// passes on the 1M-Gaussian step; fourteen or sixteen 64-thread CTAs, at 72
// or 64 registers with more spilling, took 3.39 and 4.31 ms against 3.22).
template <int TW, int TH, int BATCH, bool RECT, int PPT, bool STORE = false>
__global__ void __launch_bounds__(TW * TH / PPT, PPT == 2 ? 8 : PPT == 4 ? 12 : 1) k_blend_bwd(BlendArgs a) {
    constexpr int NT = TW * TH / PPT;
    constexpr int NACC = 9;
    // pairs of pixels in packed f32x2 lanes (the store-all study keeps the
    // scalar loop)
    constexpr bool PACKB = PPT % 2 == 0 && !STORE;
    const float2 one2 = make_float2(a.one, a.one);
    __shared__ float4 s_a[BATCH];
    __shared__ float4 s_c[BATCH];
    __shared__ float4 s_k[BATCH];
    __shared__ int s_li[BATCH];
    __shared__ uint8_t s_wm[BATCH];
    __shared__ uint32_t s_slot[BATCH];
    __shared__ float s_acc[BATCH][NACC];
    __shared__ int s_wsum[NT / 32];
    __shared__ int s_tile;
    __shared__ int s_maxlc;
    constexpr int RW = (32 / TW) * PPT;  // pixel rows per warp
    const int tid = threadIdx.x, lane = tid & 31;
    const uint32_t wbit = 1u << (tid >> 5);
    const int total_tiles = a.total_tiles ? (int)*a.total_tiles : a.total_tiles_host;
    const size_t S = (size_t)a.n_per_view * a.nviews;
    for (;;) {
        if (tid == 0) {
            s_tile = (int)atomicAdd(a.work, 1u);
            s_maxlc = -1;
        }
        __syncthreads();
        const int tile = s_tile;
        if (tile >= total_tiles) break;
        const int v = find_view(a.cams, a.nviews, tile);
        const DevCam& c = a.cams[v];
        const int lt = tile - c.tile_base;
        const int tx = lt % c.tiles_x, ty = lt / c.tiles_x;
        const int px = tx * TW + (tid % TW), py0 = ty * TH + (tid / TW) * PPT;
        const float pxf = (float)px + 0.5f;
        const float x0c = (float)(tx * TW) + 0.5f, x1c = (float)(min(tx * TW + TW, c.width) - 1) + 0.5f;
        const float y0c = (float)(ty * TH) + 0.5f, y1c = (float)(min(ty * TH + TH, c.height) - 1) + 0.5f;
        const uint2 rg = a.ranges[tile];
        int lc[PPT];
        float T[PPT], dl0[PPT], dl1[PPT], dl2[PPT], sbe[PPT], pyc[PPT];
        int my_maxlc = -1;
#pragma unroll
        for (int p = 0; p < PPT; ++p) {
            const int py = py0 + p;
            pyc[p] = (float)py + 0.5f;
            lc[p] = -1;
            T[p] = 0.0f;
            dl0[p] = dl1[p] = dl2[p] = 0.0f;
            if (px < c.width && py < c.height) {
                size_t pix = (size_t)c.pix_base + (size_t)py * c.width + px;
                lc[p] = a.last[pix];
                T[p] = a.final_t[pix];
                dl0[p] = a.dl[pix * 3 + 0];
                dl1[p] = a.dl[pix * 3 + 1];
                dl2[p] = a.dl[pix * 3 + 2];
            }
            // dL/dpixel . (colour behind the current splat), behind = T_final * bg
            sbe[p] = __fmaf_rn(dl2[p], T[p] * a.bg[2], __fmaf_rn(dl1[p], T[p] * a.bg[1], dl0[p] * (T[p] * a.bg[0])));
            my_maxlc = max(my_maxlc, lc[p]);
        }
        const int warp_maxlc = __reduce_max_sync(0xffffffffu, my_maxlc);
        if (lane == 0 && warp_maxlc >= 0) atomicMax(&s_maxlc, warp_maxlc);
        __syncthreads();
        const int maxlc = s_maxlc;
        for (int hi = maxlc; hi >= 0; hi -= BATCH) {
            const int lo = max(hi - BATCH + 1, 0);
            const int nb = stage_batch<NT, BATCH, RW, true>(a, S, rg.x + (uint32_t)lo, rg.x + (uint32_t)hi + 1u, lo, x0c, x1c, y0c,
                                                      y1c, ty * TH, c.height, s_a, s_c, s_k, s_li, s_wm, s_slot, s_wsum, nullptr);
            for (int k = tid; k < nb; k += NT) {
#pragma unroll
                for (int q = 0; q < NACC; ++q) s_acc[k][q] = 0.0f;
            }
            __syncthreads();
            for (int k = nb - 1; k >= 0; --k) {
                const int li = s_li[k];
                if (li > warp_maxlc || !(s_wm[k] & wbit)) continue;  // warp-uniform
                float g[NACC];
#pragma unroll
                for (int q = 0; q < NACC; ++q) g[q] = 0.0f;
                bool contrib = false;
                if (li <= my_maxlc) {
                    const float4 A = s_a[k];
                    const float4 Q = s_c[k];
                    const float4 K = s_k[k];
                    const float dx = pxf - A.x;
                    const float tdx = Q.x * dx * dx;
                    const float t2b = 2.0f * Q.y * dx;
                    // per-entry factors of the conic / mean gradients
                    const float hdxx = -0.5f * dx * dx, qxdx = Q.x * dx, qydx = Q.y * dx;
                    float su = 0.0f, sud = 0.0f, sudd = 0.0f;  // sums over pixels of u, u dy, u dy^2
                    if (PACKB) {
                        // pixel pairs (p, p + 1) in packed f32x2 lanes; the power, and
                        // with it every decision, is rounded per lane exactly as the
                        // forward rounds it. A lane that does not take this splat
                        // keeps its T and behind-colour sum and adds zeros.
                        float2 G0 = bc2(0.0f), G1 = bc2(0.0f), G2 = bc2(0.0f), G3 = bc2(0.0f);
                        float2 SU = bc2(0.0f), SUD = bc2(0.0f), SUDD = bc2(0.0f);
#pragma unroll
                        for (int h = 0; h < PPT / 2; ++h) {
                            const int p0 = 2 * h, p1 = 2 * h + 1;
                            bool a0 = li <= lc[p0], a1 = li <= lc[p1];
                            if (RECT) {
                                a0 = a0 && in_rect(Q.w, K.w, px, py0 + p0);
                                a1 = a1 && in_rect(Q.w, K.w, px, py0 + p1);
                            }
                            if (!(a0 || a1)) continue;
                            const float2 dy2 = __fadd2_rn(make_float2(pyc[p0], pyc[p1]), bc2(-A.y));
                            const float2 qdd2 = __fmul2_rn(__fmul2_rn(bc2(Q.z), dy2), dy2);
                            const float2 s1 = __ffma2_rn(__fmul2_rn(bc2(t2b), dy2), one2, bc2(tdx));
                            const float2 pw = __fmul2_rn(__ffma2_rn(qdd2, one2, s1), bc2(-0.5f));
                            a0 = a0 && !(pw.x > 0.0f) && !(pw.x < A.w);
                            a1 = a1 && !(pw.y > 0.0f) && !(pw.y < A.w);
                            if (!(a0 || a1)) continue;
                            float2 ge = make_float2(exp_sfu_nonpos(pw.x), exp_sfu_nonpos(pw.y));
                            float2 ar = __fmul2_rn(bc2(A.z), ge);
                            if (fabsf(ar.x - 1.0f / 255.0f) < SFU_BAND * (1.0f / 255.0f) || fabsf(ar.x - 0.99f) < SFU_BAND * 0.99f) {
                                ge.x = expf_fast_nonpos(pw.x);
                                ar.x = A.z * ge.x;
                            }
                            if (fabsf(ar.y - 1.0f / 255.0f) < SFU_BAND * (1.0f / 255.0f) || fabsf(ar.y - 0.99f) < SFU_BAND * 0.99f) {
                                ge.y = expf_fast_nonpos(pw.y);
                                ar.y = A.z * ge.y;
                            }
                            const float al0 = fminf(ar.x, 0.99f), al1 = fminf(ar.y, 0.99f);
                            a0 = a0 && !(al0 < 1.0f / 255.0f);
                            a1 = a1 && !(al1 < 1.0f / 255.0f);
                            if (!(a0 || a1)) continue;
                            const float2 al = make_float2(a0 ? al0 : 0.0f, a1 ? al1 : 0.0f);
                            const float2 om = __ffma2_rn(al, bc2(-1.0f), bc2(1.0f));
                            const float2 inv = make_float2(__fdividef(1.0f, om.x), __fdividef(1.0f, om.y));
                            // a lane with alpha = 0 has 1 - alpha = 1 and rcp(1) = 1, so its
                            // T is multiplied by exactly 1
                            const float2 Tp = __fmul2_rn(make_float2(T[p0], T[p1]), inv);
                            T[p0] = Tp.x;
                            T[p1] = Tp.y;
                            const float2 w = __fmul2_rn(al, Tp);
                            const float2 d0 = make_float2(dl0[p0], dl0[p1]);
                            const float2 d1 = make_float2(dl1[p0], dl1[p1]);
                            const float2 d2 = make_float2(dl2[p0], dl2[p1]);
                            G0 = __ffma2_rn(d0, w, G0);
                            G1 = __ffma2_rn(d1, w, G1);
                            G2 = __ffma2_rn(d2, w, G2);
                            const float2 dk = __ffma2_rn(d2, bc2(K.z), __ffma2_rn(d1, bc2(K.y), __fmul2_rn(d0, bc2(K.x))));
                            const float2 sb = make_float2(sbe[p0], sbe[p1]);
                            const float2 dda = __ffma2_rn(Tp, dk, __fmul2_rn(make_float2(-sb.x, -sb.y), inv));
                            const float2 sbn = __ffma2_rn(w, dk, sb);
                            sbe[p0] = sbn.x;
                            sbe[p1] = sbn.y;
                            // zero for a lane that does not take the splat or whose raw
                            // alpha was clamped (backward.rs:459-461)
                            const float2 draw = make_float2(a0 && !(ar.x > 0.99f) ? dda.x : 0.0f, a1 && !(ar.y > 0.99f) ? dda.y : 0.0f);
                            // every lane's exp and raw alpha are finite (power <= 0 up to
                            // rounding), so a zero draw zeroes its terms
                            G3 = __ffma2_rn(draw, ge, G3);
                            const float2 u = __fmul2_rn(draw, ar);
                            SU = __fadd2_rn(SU, u);
                            SUD = __ffma2_rn(u, dy2, SUD);
                            SUDD = __ffma2_rn(__fmul2_rn(u, dy2), dy2, SUDD);
                            contrib = true;
                        }
                        if (contrib) {
                            g[0] = G0.x + G0.y;
                            g[1] = G1.x + G1.y;
                            g[2] = G2.x + G2.y;
                            g[3] = G3.x + G3.y;
                            su = SU.x + SU.y;
                            sud = SUD.x + SUD.y;
                            sudd = SUDD.x + SUDD.y;
                        }
                    } else {
#pragma unroll
                    for (int p = 0; p < PPT; ++p) {
                        if (li > lc[p]) continue;
                        if (RECT && !in_rect(Q.w, K.w, px, py0 + p)) continue;
                        // alpha exactly as the forward computed it
                        const float dy = pyc[p] - A.y;
                        const float power = -0.5f * (tdx + t2b * dy + Q.z * dy * dy);
                        if (power > 0.0f || power < A.w) continue;
                        // alpha to ~1e-6 from the SFU exponential; where that cannot
                        // settle the forward's decisions (alpha >= 1/255, alpha_raw >
                        // 0.99), the forward's own exp settles them, so the
                        // contributing set is exactly the forward's
                        float g_exp = exp_sfu_nonpos(power);
                        float alpha_raw = A.z * g_exp;
                        if (fabsf(alpha_raw - 1.0f / 255.0f) < SFU_BAND * (1.0f / 255.0f) ||
                            fabsf(alpha_raw - 0.99f) < SFU_BAND * 0.99f) {
                            g_exp = expf_fast_nonpos(power);
                            alpha_raw = A.z * g_exp;
                        }
                        const float alpha = fminf(alpha_raw, 0.99f);
                        if (alpha < 1.0f / 255.0f) continue;
                        float inv_1ma;
                        if (STORE) {
                            // store-all variant: T before this splat as the forward saw it
                            T[p] = a.tstore[(size_t)(rg.x + (uint32_t)li) * (TW * TH) + (tid / TW) * PPT * TW + p * TW + tid % TW];
                            inv_1ma = 1.0f / (1.0f - alpha);
                        } else {
                            inv_1ma = __fdividef(1.0f, 1.0f - alpha);
                            T[p] = T[p] * inv_1ma;
                        }
                        // gradient terms of backward.rs:453-484, as fused multiply-adds.
                        // The colour behind enters only as dL/dpixel . behind, so one
                        // scalar per pixel (sbe) replaces the three channels; the conic
                        // and mean terms are linear in u = dL/dpower per pixel, so the
                        // thread sums u, u dy and u dy^2 over its pixels and forms the
                        // five terms once per splat (dx is the thread's column).
                        const float weight = alpha * T[p];
                        g[0] = __fmaf_rn(dl0[p], weight, g[0]);
                        g[1] = __fmaf_rn(dl1[p], weight, g[1]);
                        g[2] = __fmaf_rn(dl2[p], weight, g[2]);
                        const float dk = __fmaf_rn(dl2[p], K.z, __fmaf_rn(dl1[p], K.y, dl0[p] * K.x));
                        const float dl_dalpha = __fmaf_rn(T[p], dk, -sbe[p] * inv_1ma);
                        sbe[p] = __fmaf_rn(weight, dk, sbe[p]);
                        const float dl_draw = alpha_raw > 0.99f ? 0.0f : dl_dalpha;
                        g[3] = __fmaf_rn(dl_draw, g_exp, g[3]);
                        const float u = dl_draw * alpha_raw;
                        su += u;
                        sud = __fmaf_rn(u, dy, sud);
                        sudd = __fmaf_rn(u * dy, dy, sudd);
                        contrib = true;
                    }
                    }
                    if (contrib) {
                        g[4] = hdxx * su;
                        g[5] = -dx * sud;
                        g[6] = -0.5f * sudd;
                        g[7] = __fmaf_rn(Q.y, sud, qxdx * su);
                        g[8] = __fmaf_rn(Q.z, sud, qydx * su);
                    }
                }
                const unsigned cm = __ballot_sync(0xffffffffu, contrib);
                if (cm != 0u) {
                    if ((cm & (cm - 1u)) == 0u) {
                        // a single contributing thread: add its values directly
                        if (contrib) {
#pragma unroll
                            for (int q = 0; q < NACC; ++q) atomicAdd(&s_acc[k][q], g[q]);
                        }
                    } else {
                        warp_reduce_scatter9(g, lane, &s_acc[k][0]);
                    }
                }
            }
            __syncthreads();
            for (int k = tid; k < nb; k += NT) {
                const float* q = s_acc[k];
                bool any = false;
#pragma unroll
                for (int i = 0; i < NACC; ++i) any |= (q[i] != 0.0f);
                if (any) {
                    const uint32_t slot = s_slot[k];
                    red_add_v4(a.acc + slot, q[0], q[1], q[2], q[3]);
                    red_add_v4(a.acc + S + slot, q[4], q[5], q[6], q[7]);
                    red_add_v4(a.acc + 2 * S + slot, q[8], 0.0f, 0.0f, 0.0f);
                }
            }
            __syncthreads();
        }
        __syncthreads();  // every thread has read s_tile / s_maxlc before thread 0 rewrites them
    }
}

// ---- launch plumbing -----------------------------------------------------
typedef void (*BlendKernel)(BlendArgs);

// The forward runs `pixels_per_thread` (1 or 2) pixels per thread, the
// backward twice that: its per-splat warp reduction is then shared by twice
// the pixels (measured 3 % faster at 4 than at 2 on the 1M-Gaussian step,
// while the forward is slower at 4).
template <int TW, int TH, int BATCH, bool RECT>
static BlendKernel pick(bool fwd, int ppt) {
    if (fwd) return ppt == 1 ? (BlendKernel)k_blend_fwd<TW, TH, BATCH, RECT, 1> : (BlendKernel)k_blend_fwd<TW, TH, BATCH, RECT, 2>;
    return ppt == 2 ? (BlendKernel)k_blend_bwd<TW, TH, BATCH, RECT, 2> : (BlendKernel)k_blend_bwd<TW, TH, BATCH, RECT, 4>;
}

template <int TW, int TH, bool RECT>
static BlendKernel pick_batch(int batch, bool fwd, int ppt) {
    switch (batch) {
        case 128: return pick<TW, TH, 128, RECT>(fwd, ppt);
        case 512: return pick<TW, TH, 512, RECT>(fwd, ppt);
        default: return pick<TW, TH, 256, RECT>(fwd, ppt);
    }
}

static BlendKernel select_kernel(int tw, int th, int batch, bool rect, bool fwd, int ppt) {
    if (tw == 8 && th == 32) return pick_batch<8, 32, true>(batch, fwd, ppt);
    if (tw == 32 && th == 8) return pick_batch<32, 8, true>(batch, fwd, ppt);
    return rect ? pick_batch<16, 16, true>(batch, fwd, ppt) : pick_batch<16, 16, false>(batch, fwd, ppt);
}

// Persistent grid of a blend kernel on the current device: SMs x resident CTAs,
// cached per (kernel, device ordinal).
static int grid_for(BlendKernel k, int threads) {
    struct Entry { BlendKernel k; int dev; int grid; };
    static std::mutex mu;
    static Entry cache[256];
    static int ncache = 0;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) cudaGetLastError();
    const int sms = device_sm_count();
    std::lock_guard<std::mutex> g(mu);
    for (int i = 0; i < ncache; ++i)
        if (cache[i].k == k && cache[i].dev == dev) return cache[i].grid;
    int per = 1;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, (const void*)k, threads, 0) != cudaSuccess) {
        cudaGetLastError();
        per = 1;
    }
    int grid = sms * std::max(per, 1);
    if (ncache < 256) cache[ncache++] = {k, dev, grid};
    return grid;
}

static void launch(const BlendArgs& a, int tw, int th, int batch, bool fwd, cudaStream_t st) {
    bool rect = a.rect_filter != 0 || !(tw == REF_TILE && th == REF_TILE);
    int ppt = (a.pixels_per_thread == 1 ? 1 : 2) * (fwd ? 1 : 2);
    BlendKernel k = select_kernel(tw, th, batch, rect, fwd, ppt);
    int threads = tw * th / ppt;
    cudaMemsetAsync(a.work, 0, sizeof(uint32_t), st);
    int grid = grid_for(k, threads);
    if (!a.total_tiles) grid = std::min(grid, std::max(a.total_tiles_host, 1));
    k<<<grid, threads, 0, st>>>(a);
}

// (pixel, splat) pairs the blend evaluates, per pixel of view blockIdx.y: the
// forward walks the pixel's tile list until T < 1e-4 ends it at its last
// contributor (final T below 1e-4) or the list runs out; the backward walks
// from the last contributor down to the front. out[0] += forward pairs,
// out[1] += backward pairs.
__global__ void __launch_bounds__(256) k_evaluated_pairs(const DevCam* __restrict__ cams, const uint2* __restrict__ ranges,
                                                         const float* __restrict__ final_t, const int* __restrict__ last,
                                                         int tile_w, int tile_h, unsigned long long* out) {
    const DevCam& c = cams[blockIdx.y];
    const uint32_t px = (uint32_t)c.width * (uint32_t)c.height;
    unsigned long long f = 0, b = 0;
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < px; p += gridDim.x * blockDim.x) {
        const uint32_t x = p % (uint32_t)c.width, y = p / (uint32_t)c.width;
        const uint2 r = ranges[c.tile_base + (y / tile_h) * c.tiles_x + x / tile_w];
        const int l = last[(size_t)c.pix_base + p];
        const float t = final_t[(size_t)c.pix_base + p];
        f += t < 1e-4f ? (unsigned long long)(l + 1) : (unsigned long long)(r.y - r.x);
        b += l >= 0 ? (unsigned long long)(l + 1) : 0ull;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        f += __shfl_down_sync(0xffffffffu, f, o);
        b += __shfl_down_sync(0xffffffffu, b, o);
    }
    if ((threadIdx.x & 31) == 0 && (f | b)) {
        atomicAdd(out, f);
        atomicAdd(out + 1, b);
    }
}

// Largest |exp_sfu_nonpos(x) / expf_fast_nonpos(x) - 1| over n points spaced
// evenly on [lo, hi] (hi <= 0), as float bits in *out (non-negative floats
// order like their bits).
__global__ void k_exp_sfu_error(float lo, float hi, uint32_t n, unsigned int* out) {
    float m = 0.0f;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float x = lo + (hi - lo) * ((float)i / (float)(n > 1 ? n - 1 : 1));
        const float e = expf_fast_nonpos(x);
        m = fmaxf(m, fabsf(exp_sfu_nonpos(x) / e - 1.0f));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, __float_as_uint(m));
}

void launch_exp_sfu_error(float lo, float hi, uint32_t n, unsigned int* out, cudaStream_t st) {
    k_exp_sfu_error<<<device_sm_count() * 4, 256, 0, st>>>(lo, hi, n, out);
}

void launch_evaluated_pairs(const DevCam* cams, int nviews, const uint2* ranges, const float* final_t, const int* last,
                            int tile_w, int tile_h, unsigned long long* out, cudaStream_t st) {
    if (nviews <= 0) return;
    k_evaluated_pairs<<<dim3((unsigned)device_sm_count() * 2, (unsigned)nviews), 256, 0, st>>>(cams, ranges, final_t, last,
                                                                                            tile_w, tile_h, out);
}

void launch_blend_forward(const BlendArgs& a, int tw, int th, int batch, cudaStream_t st) { launch(a, tw, th, batch, true, st); }
void launch_blend_backward(const BlendArgs& a, int tw, int th, int batch, cudaStream_t st) { launch(a, tw, th, batch, false, st); }

// Store-all variant (16x16 tiles, 256-splat batches, 2 pixels per thread): the
// forward writes T before every contributing splat of every pixel to
// a.tstore[(list position) * 256 + pixel in tile], the backward reads it back
// instead of rebuilding T from the final T.
void launch_blend_store_all(const BlendArgs& a, bool fwd, cudaStream_t st) {
    BlendKernel k = fwd ? (BlendKernel)k_blend_fwd<16, 16, 256, false, 2, true> : (BlendKernel)k_blend_bwd<16, 16, 256, false, 2, true>;
    cudaMemsetAsync(a.work, 0, sizeof(uint32_t), st);
    int grid = grid_for(k, 128);
    if (!a.total_tiles) grid = std::min(grid, std::max(a.total_tiles_host, 1));
    k<<<grid, 128, 0, st>>>(a);
}

}  // namespace rgs

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
// counter; BATCH splat records per round are staged in shared memory and read
// by all threads as broadcasts. Backward pre-reduces each splat's 9 partial
// gradients across the warp with shuffles (only when a lane contributed),
// then across warps with shared-memory atomics, and issues one 3 x 16-byte
// vector reduction (red.global.add.v4.f32) per splat per CTA.
//
// CTA tiles other than 16x16 keep the reference's per-pixel semantics: each
// record carries its reference-tile rectangle in pixels and a pixel only
// evaluates splats whose rectangle contains it (RECT = true).
#include <algorithm>
#include <mutex>

#include "rgs_internal.cuh"
#include "rgs_math.cuh"

namespace rgs {

// Below this power, opacity <= 1 gives opacity * e^power < 1/255 for every
// finite opacity, so the reference's own alpha test would skip the splat.
#define RGS_POWER_CUT (-5.55f)

__device__ __forceinline__ int find_view(const DevCam* cams, int nviews, int tile) {
    int v = 0;
    while (v + 1 < nviews && cams[v + 1].tile_base <= tile) ++v;
    return v;
}

__device__ __forceinline__ bool in_rect(float rx, float ry, int px, int py) {
    uint32_t x = __float_as_uint(rx), y = __float_as_uint(ry);
    return px >= (int)(x & 0xffffu) && px < (int)(x >> 16) && py >= (int)(y & 0xffffu) && py < (int)(y >> 16);
}

template <int TW, int TH, int BATCH, bool RECT>
__global__ void __launch_bounds__(TW * TH) k_blend_fwd(BlendArgs a) {
    constexpr int NT = TW * TH;
    __shared__ float4 s_a[BATCH];
    __shared__ float4 s_c[BATCH];
    __shared__ float4 s_k[BATCH];
    __shared__ int s_tile;
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
        const int px = tx * TW + (tid % TW), py = ty * TH + (tid / TW);
        const bool inside = px < c.width && py < c.height;
        const float pxf = (float)px + 0.5f, pyf = (float)py + 0.5f;
        const uint2 rg = a.ranges[tile];
        float T = 1.0f, C0 = 0.0f, C1 = 0.0f, C2 = 0.0f;
        int last = -1;
        bool done = !inside;
        // whether the pixel's reference tile list is non-empty
        bool seen = !RECT && rg.y > rg.x;
        for (uint32_t b0 = rg.x; b0 < rg.y; b0 += BATCH) {
            if (__syncthreads_count(!done) == 0) break;
            for (int j = tid; j < BATCH; j += NT) {
                uint32_t idx = b0 + j;
                if (idx < rg.y) {
                    uint32_t slot = a.pair_vals[idx];
                    s_a[j] = a.rec[slot];
                    s_c[j] = a.rec[S + slot];
                    s_k[j] = a.rec[2 * S + slot];
                }
            }
            __syncthreads();
            const int nb = (int)min((uint32_t)BATCH, rg.y - b0);
            for (int j = 0; j < nb && !done; ++j) {
                const float4 A = s_a[j];
                const float4 Q = s_c[j];
                if (RECT) {
                    if (!in_rect(Q.w, s_k[j].w, px, py)) continue;
                    seen = true;
                }
                const float dx = pxf - A.x, dy = pyf - A.y;
                const float power = -0.5f * (Q.x * dx * dx + 2.0f * Q.y * dx * dy + Q.z * dy * dy);
                if (power > 0.0f || power < RGS_POWER_CUT) continue;
                const float alpha = fminf(A.z * expf_fast(power), 0.99f);
                if (alpha < 1.0f / 255.0f) continue;
                const float4 K = s_k[j];
                const float weight = alpha * T;
                C0 += K.x * weight;
                C1 += K.y * weight;
                C2 += K.z * weight;
                T *= 1.0f - alpha;
                last = (int)(b0 - rg.x) + j;
                if (T < 1e-4f) done = true;
            }
            __syncthreads();
        }
        if (inside) {
            size_t pix = (size_t)c.pix_base + (size_t)py * c.width + px;
            // forward_pass skips tiles whose list is empty, leaving their pixels
            // at 0 rather than bg (src/cpu/backward.rs:313-315, 124)
            const bool black = a.empty_tile_black && !seen;
            a.rgb[pix * 3 + 0] = black ? 0.0f : C0 + T * a.bg[0];
            a.rgb[pix * 3 + 1] = black ? 0.0f : C1 + T * a.bg[1];
            a.rgb[pix * 3 + 2] = black ? 0.0f : C2 + T * a.bg[2];
            a.final_t[pix] = T;
            a.last[pix] = last;
        }
        __syncthreads();
    }
}

__device__ __forceinline__ void red_add_v4(float4* addr, float x, float y, float z, float w) {
    asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(addr), "f"(x), "f"(y), "f"(z), "f"(w) : "memory");
}

template <int TW, int TH, int BATCH, bool RECT>
__global__ void __launch_bounds__(TW * TH) k_blend_bwd(BlendArgs a) {
    constexpr int NT = TW * TH;
    constexpr int NACC = 9;
    __shared__ float4 s_a[BATCH];
    __shared__ float4 s_c[BATCH];
    __shared__ float4 s_k[BATCH];
    __shared__ uint32_t s_slot[BATCH];
    __shared__ float s_acc[BATCH][NACC];
    __shared__ int s_tile;
    __shared__ int s_maxlc;
    const int tid = threadIdx.x, lane = tid & 31;
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
        const int px = tx * TW + (tid % TW), py = ty * TH + (tid / TW);
        const bool inside = px < c.width && py < c.height;
        const float pxf = (float)px + 0.5f, pyf = (float)py + 0.5f;
        const uint2 rg = a.ranges[tile];
        int lc = -1;
        float T = 0.0f, dl0 = 0.0f, dl1 = 0.0f, dl2 = 0.0f;
        if (inside) {
            size_t pix = (size_t)c.pix_base + (size_t)py * c.width + px;
            lc = a.last[pix];
            T = a.final_t[pix];
            dl0 = a.dl[pix * 3 + 0];
            dl1 = a.dl[pix * 3 + 1];
            dl2 = a.dl[pix * 3 + 2];
        }
        float be0 = T * a.bg[0], be1 = T * a.bg[1], be2 = T * a.bg[2];
        if (lc >= 0) atomicMax(&s_maxlc, lc);
        __syncthreads();
        const int maxlc = s_maxlc;
        for (int hi = maxlc; hi >= 0; hi -= BATCH) {
            const int lo = max(hi - BATCH + 1, 0);
            const int nb = hi - lo + 1;
            for (int j = tid; j < nb; j += NT) {
                uint32_t slot = a.pair_vals[rg.x + lo + j];
                s_slot[j] = slot;
                s_a[j] = a.rec[slot];
                s_c[j] = a.rec[S + slot];
                s_k[j] = a.rec[2 * S + slot];
#pragma unroll
                for (int k = 0; k < NACC; ++k) s_acc[j][k] = 0.0f;
            }
            __syncthreads();
            for (int j = nb - 1; j >= 0; --j) {
                const int li = lo + j;
                float g[NACC];
#pragma unroll
                for (int k = 0; k < NACC; ++k) g[k] = 0.0f;
                bool contrib = false;
                if (li <= lc) {
                    const float4 A = s_a[j];
                    const float4 Q = s_c[j];
                    const float4 K = s_k[j];
                    bool ok = !RECT || in_rect(Q.w, K.w, px, py);
                    const float dx = pxf - A.x, dy = pyf - A.y;
                    const float power = -0.5f * (Q.x * dx * dx + 2.0f * Q.y * dx * dy + Q.z * dy * dy);
                    if (ok && power <= 0.0f && power >= RGS_POWER_CUT) {
                        const float g_exp = expf_fast(power);
                        const float alpha_raw = A.z * g_exp;
                        const float alpha = fminf(alpha_raw, 0.99f);
                        if (alpha >= 1.0f / 255.0f) {
                            T = T / (1.0f - alpha);
                            const float weight = alpha * T;
                            g[0] = dl0 * weight;
                            g[1] = dl1 * weight;
                            g[2] = dl2 * weight;
                            const float inv_1ma = 1.0f / (1.0f - alpha);
                            float dl_dalpha = 0.0f;
                            dl_dalpha += dl0 * (T * K.x - be0 * inv_1ma);
                            dl_dalpha += dl1 * (T * K.y - be1 * inv_1ma);
                            dl_dalpha += dl2 * (T * K.z - be2 * inv_1ma);
                            const float dl_draw = dl_dalpha * (alpha_raw > 0.99f ? 0.0f : 1.0f);
                            g[3] = dl_draw * g_exp;
                            const float dl_dpower = dl_draw * A.z * g_exp;
                            g[4] = dl_dpower * (-0.5f * dx * dx);
                            g[5] = dl_dpower * (-dx * dy);
                            g[6] = dl_dpower * (-0.5f * dy * dy);
                            g[7] = dl_dpower * (Q.x * dx + Q.y * dy);
                            g[8] = dl_dpower * (Q.y * dx + Q.z * dy);
                            be0 += weight * K.x;
                            be1 += weight * K.y;
                            be2 += weight * K.z;
                            contrib = true;
                        }
                    }
                }
                if (__any_sync(0xffffffffu, contrib)) {
#pragma unroll
                    for (int k = 0; k < NACC; ++k) {
                        float x = g[k];
#pragma unroll
                        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
                        g[k] = x;
                    }
                    if (lane == 0) {
#pragma unroll
                        for (int k = 0; k < NACC; ++k) atomicAdd(&s_acc[j][k], g[k]);
                    }
                }
            }
            __syncthreads();
            for (int j = tid; j < nb; j += NT) {
                const float* q = s_acc[j];
                bool any = false;
#pragma unroll
                for (int k = 0; k < NACC; ++k) any |= (q[k] != 0.0f);
                if (any) {
                    uint32_t slot = s_slot[j];
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

template <int TW, int TH, int BATCH, bool RECT>
static BlendKernel pick(bool fwd) {
    return fwd ? (BlendKernel)k_blend_fwd<TW, TH, BATCH, RECT> : (BlendKernel)k_blend_bwd<TW, TH, BATCH, RECT>;
}

template <int TW, int TH, bool RECT>
static BlendKernel pick_batch(int batch, bool fwd) {
    switch (batch) {
        case 128: return pick<TW, TH, 128, RECT>(fwd);
        case 512: return pick<TW, TH, 512, RECT>(fwd);
        default: return pick<TW, TH, 256, RECT>(fwd);
    }
}

static BlendKernel select_kernel(int tw, int th, int batch, bool rect, bool fwd) {
    if (tw == 8 && th == 32) return pick_batch<8, 32, true>(batch, fwd);
    if (tw == 32 && th == 8) return pick_batch<32, 8, true>(batch, fwd);
    return rect ? pick_batch<16, 16, true>(batch, fwd) : pick_batch<16, 16, false>(batch, fwd);
}

static int grid_for(BlendKernel k, int threads) {
    static std::mutex mu;
    static std::pair<BlendKernel, int> cache[64];
    static int ncache = 0;
    std::lock_guard<std::mutex> g(mu);
    for (int i = 0; i < ncache; ++i)
        if (cache[i].first == k) return cache[i].second;
    int dev = 0, sms = 148, per = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, (const void*)k, threads, 0);
    int grid = sms * std::max(per, 1);
    if (ncache < 64) cache[ncache++] = {k, grid};
    return grid;
}

static void launch(const BlendArgs& a, int tw, int th, int batch, bool fwd, cudaStream_t st) {
    bool rect = a.rect_filter != 0 || !(tw == REF_TILE && th == REF_TILE);
    BlendKernel k = select_kernel(tw, th, batch, rect, fwd);
    int threads = tw * th;
    cudaMemsetAsync(a.work, 0, sizeof(uint32_t), st);
    int grid = grid_for(k, threads);
    if (!a.total_tiles) grid = std::min(grid, std::max(a.total_tiles_host, 1));
    k<<<grid, threads, 0, st>>>(a);
}

void launch_blend_forward(const BlendArgs& a, int tw, int th, int batch, cudaStream_t st) { launch(a, tw, th, batch, true, st); }
void launch_blend_backward(const BlendArgs& a, int tw, int th, int batch, cudaStream_t st) { launch(a, tw, th, batch, false, st); }

}  // namespace rgs

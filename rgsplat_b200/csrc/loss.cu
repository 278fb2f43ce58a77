// loss.cu -- L = (1 - lambda) * L1 + lambda * (1 - SSIM) and dL/dpixel.
//
// Follows src/cpu/backward.rs:646-807: per channel, SSIM with an 11-tap
// Gaussian window (sigma 1.5, normalised, backward.rs:759-772) applied as a
// separable blur with zero padding (backward.rs:776-807), C1 = 0.01^2,
// C2 = 0.03^2, and the gradient through five further blurs of the maps P, Q,
// R, Q*mu_y, R*mu_x (backward.rs:718-755). dL1 uses Rust's signum (+1 for
// +0.0), written as copysignf.
//
// B200 mapping: one CTA per 32x32 output tile of any view of the batch. The
// CTA stages the rendered and target channels over a 52x52 region (two
// 5-pixel halos) in shared memory and runs all ten blurs there, so HBM sees
// each input pixel about once and dL/dpixel is written once. The blurs are
// register-blocked (a thread produces a run of outputs from one sliding
// window, so each shared-memory value and each product x^2, y^2, xy is
// formed once per run). Two kernels: k_loss keeps the reference's separate
// multiply and add per tap and its divisions (dL/dpixel bit-identical,
// rgs_options.exact_loss); k_loss_fused, the default, accumulates with fused
// multiply-adds on packed f32x2 pairs and forms the three SSIM quotients from
// one reciprocal. The scalar loss is reduced per CTA and then per view in a
// fixed order (deterministic). (Staging each channel by 4-byte asynchronous
// copies issued during the previous channel's passes 2-4, with the tile's
// centre kept apart for pass 4, measured slower: 0.84 against 0.80 ms.)
#include <mutex>

#include "rgs_internal.cuh"
#include "rgs_math.cuh"

namespace rgs {

constexpr int LT = 32;            // output tile edge
constexpr int LR = 5;             // window radius
constexpr int RG = LT + 4 * LR;   // 52: staged input region
constexpr int MG = LT + 2 * LR;   // 42: statistics / map region
constexpr int MGP = MG + 1;       // padded row stride of the maps (odd: no bank conflicts)
constexpr int LTP = LT + 1;       // padded row stride of the blurred maps
constexpr int LOSS_THREADS = 256;
// register blocking of the four separable passes: each thread produces a
// run of outputs along the blur direction from one sliding window of inputs
constexpr int H1 = 7;             // pass 1 (rows of x, y, x^2, y^2, xy): 6 runs per row
constexpr int V1 = 7;             // pass 2 (columns -> statistics): 6 runs per column
constexpr int H2 = 8;             // pass 3 (rows of the five maps): 4 runs per row
constexpr int V2 = 4;             // pass 4 (columns -> gradient): 8 runs per column
static_assert(MG % H1 == 0 && MG % V1 == 0 && LT % H2 == 0 && LT % V2 == 0, "run lengths must tile the regions");
constexpr size_t LOSS_SMEM =
    sizeof(float) * (2 * RG * RG + 5 * RG * MG + 5 * MG * MGP + 16 + 2 * LOSS_THREADS / 32);
static_assert(5 * MG * LTP <= 5 * RG * MG, "pass-3 output must fit in the pass-1 buffer");

__device__ __forceinline__ float block_sum_fixed(float v, float* s_red) {
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    __syncthreads();
    if (lane == 0) s_red[w] = v;
    __syncthreads();
    float t = 0.0f;
    for (int k = 0; k < LOSS_THREADS / 32; ++k) t += s_red[k];
    return t;
}

// From the blurred statistics of one pixel (means mx, my; second moments
// exx, eyy, exy): its SSIM value (returned) and the maps the gradient blurs
// (backward.rs:718-755): P, Q, R, Q*mu_y, R*mu_x. FAST: one reciprocal for the
// three quotients; otherwise the reference's divisions.
template <bool FAST>
__device__ __forceinline__ float ssim_maps(float mx, float my, float exx, float eyy, float exy, float& P, float& Q, float& R,
                                           float& QM, float& RM) {
    const float C1 = 0.01f * 0.01f;
    const float C2 = 0.03f * 0.03f;
    float sx2 = exx - mx * mx;
    float sy2 = eyy - my * my;
    float sxy = exy - mx * my;
    float a1 = 2.0f * mx * my + C1;
    float a2 = 2.0f * sxy + C2;
    float b1 = mx * mx + my * my + C1;
    float b2 = sx2 + sy2 + C2;
    float num = a1 * a2;
    float den = b1 * b2;
    float inv_den = 1.0f / den;
    const float s_map = FAST ? num * inv_den : num / den;
    const float s_den2 = FAST ? s_map * inv_den : num / (den * den);
    P = inv_den * (2.0f * my * a2) - s_den2 * (2.0f * mx * b2);
    Q = inv_den * (2.0f * a1);
    R = -s_den2 * b1;
    QM = Q * my;
    RM = R * mx;
    return s_map;
}

__global__ void __launch_bounds__(LOSS_THREADS) k_loss(const DevCam* __restrict__ cams, int nviews, const uint32_t* total_dev,
                                                       int total_host, const float* __restrict__ rgb, float lambda,
                                                       float* __restrict__ dl, float* __restrict__ partials) {
    extern __shared__ float smem[];
    float* in_x = smem;
    float* in_y = in_x + RG * RG;
    float* tmp = in_y + RG * RG;         // pass 1 out: [5][RG rows][MG cols]; pass 3 out: [5][MG][LTP]
    float* st = tmp + 5 * RG * MG;        // pass 2 out (maps): [5][MG][MGP]
    float* kw = st + 5 * MG * MGP;        // 11 taps
    float* s_red = kw + 16;
    const int tid = threadIdx.x;
    if (tid == 0) {
        // gaussian_kernel_1d(5, 1.5), backward.rs:759-772
        float sum = 0.0f;
        float v[11];
        for (int i = 0; i < 11; ++i) {
            float d = (float)i - 5.0f;
            v[i] = exp_cr(-0.5f * d * d / (1.5f * 1.5f));
            sum += v[i];
        }
        for (int i = 0; i < 11; ++i) kw[i] = v[i] / sum;
    }
    __syncthreads();
    float w11[11];
#pragma unroll
    for (int k = 0; k < 11; ++k) w11[k] = kw[k];
    const int total = total_dev ? (int)*total_dev : total_host;
    for (int blk = blockIdx.x; blk < total; blk += gridDim.x) {
        int v = 0;
        while (v + 1 < nviews && cams[v + 1].loss_base <= blk) ++v;
        const DevCam& c = cams[v];
        const int w = c.width, h = c.height;
        const int lb = blk - c.loss_base;
        const int ox = (lb % c.loss_bx) * LT, oy = (lb / c.loss_bx) * LT;
        const float m_total = (float)((size_t)w * h * 3);
        const float* tgt = c.target;
        const size_t pb = (size_t)c.pix_base;
        float l1_local = 0.0f, ssim_local = 0.0f;
        for (int ch = 0; ch < 3; ++ch) {
            for (int i = tid; i < RG * RG; i += LOSS_THREADS) {
                int r = i / RG, cc = i - r * RG;
                int gx = ox - 2 * LR + cc, gy = oy - 2 * LR + r;
                float xv = 0.0f, yv = 0.0f;
                if (gx >= 0 && gx < w && gy >= 0 && gy < h) {
                    size_t p = (size_t)gy * w + gx;
                    xv = rgb[(pb + p) * 3 + ch];
                    yv = tgt[p * 4 + ch];
                }
                in_x[i] = xv;
                in_y[i] = yv;
            }
            __syncthreads();
            // pass 1: horizontal blur of x, y, x^2, y^2, xy over rows [0, RG),
            // map columns [0, MG); a run of H1 outputs per thread
            for (int it = tid; it < RG * (MG / H1); it += LOSS_THREADS) {
                const int r = it / (MG / H1), c0 = (it - r * (MG / H1)) * H1;
                const float* rx = in_x + r * RG + c0;
                const float* ry = in_y + r * RG + c0;
                float a[H1][5];
#pragma unroll
                for (int o = 0; o < H1; ++o)
#pragma unroll
                    for (int q = 0; q < 5; ++q) a[o][q] = 0.0f;
#pragma unroll
                for (int j = 0; j < H1 + 10; ++j) {
                    const float xk = rx[j], yk = ry[j];
                    const float xx = xk * xk, yy = yk * yk, xy = xk * yk;
#pragma unroll
                    for (int o = 0; o < H1; ++o) {
                        const int k = j - o;
                        if (k < 0 || k > 10) continue;
                        a[o][0] += w11[k] * xk;
                        a[o][1] += w11[k] * yk;
                        a[o][2] += w11[k] * xx;
                        a[o][3] += w11[k] * yy;
                        a[o][4] += w11[k] * xy;
                    }
                }
#pragma unroll
                for (int o = 0; o < H1; ++o)
#pragma unroll
                    for (int q = 0; q < 5; ++q) tmp[q * RG * MG + r * MG + c0 + o] = a[o][q];
            }
            __syncthreads();
            // pass 2: vertical blur -> statistics, then the per-pixel SSIM
            // maps P, Q, R, Q*mu_y, R*mu_x (zero outside the image)
            for (int it = tid; it < MG * (MG / V1); it += LOSS_THREADS) {
                const int cm = it % MG, r0 = (it / MG) * V1;
                float mu[V1][5];
#pragma unroll
                for (int o = 0; o < V1; ++o)
#pragma unroll
                    for (int q = 0; q < 5; ++q) mu[o][q] = 0.0f;
#pragma unroll
                for (int j = 0; j < V1 + 10; ++j) {
                    float t[5];
#pragma unroll
                    for (int q = 0; q < 5; ++q) t[q] = tmp[q * RG * MG + (r0 + j) * MG + cm];
#pragma unroll
                    for (int o = 0; o < V1; ++o) {
                        const int k = j - o;
                        if (k < 0 || k > 10) continue;
#pragma unroll
                        for (int q = 0; q < 5; ++q) mu[o][q] += w11[k] * t[q];
                    }
                }
                const int gx = ox - LR + cm;
#pragma unroll
                for (int o = 0; o < V1; ++o) {
                    const int rm = r0 + o, gy = oy - LR + rm;
                    float P = 0.0f, Q = 0.0f, R = 0.0f, QM = 0.0f, RM = 0.0f;
                    if (gx >= 0 && gx < w && gy >= 0 && gy < h) {
                        const float s = ssim_maps<false>(mu[o][0], mu[o][1], mu[o][2], mu[o][3], mu[o][4], P, Q, R, QM, RM);
                        if (rm >= LR && rm < LR + LT && cm >= LR && cm < LR + LT) ssim_local += s;
                    }
                    float* sp = st + rm * MGP + cm;
                    sp[0 * MG * MGP] = P;
                    sp[1 * MG * MGP] = Q;
                    sp[2 * MG * MGP] = R;
                    sp[3 * MG * MGP] = QM;
                    sp[4 * MG * MGP] = RM;
                }
            }
            __syncthreads();
            // pass 3: horizontal blur of the maps: rows [0, MG), output cols [0, LT)
            for (int it = tid; it < MG * (LT / H2); it += LOSS_THREADS) {
                const int rm = it % MG, c0 = (it / MG) * H2;
#pragma unroll 1
                for (int q = 0; q < 5; ++q) {
                    const float* row = st + q * MG * MGP + rm * MGP + c0;
                    float a[H2];
#pragma unroll
                    for (int o = 0; o < H2; ++o) a[o] = 0.0f;
#pragma unroll
                    for (int j = 0; j < H2 + 10; ++j) {
                        const float t = row[j];
#pragma unroll
                        for (int o = 0; o < H2; ++o) {
                            const int k = j - o;
                            if (k < 0 || k > 10) continue;
                            a[o] += w11[k] * t;
                        }
                    }
#pragma unroll
                    for (int o = 0; o < H2; ++o) tmp[q * MG * LTP + rm * LTP + c0 + o] = a[o];
                }
            }
            __syncthreads();
            // pass 4: vertical blur -> gradient, combined with the L1 term
            for (int it = tid; it < LT * (LT / V2); it += LOSS_THREADS) {
                const int co = it % LT, r0 = (it / LT) * V2;
                float b[V2][5];
#pragma unroll
                for (int o = 0; o < V2; ++o)
#pragma unroll
                    for (int q = 0; q < 5; ++q) b[o][q] = 0.0f;
#pragma unroll
                for (int j = 0; j < V2 + 10; ++j) {
                    float t[5];
#pragma unroll
                    for (int q = 0; q < 5; ++q) t[q] = tmp[q * MG * LTP + (r0 + j) * LTP + co];
#pragma unroll
                    for (int o = 0; o < V2; ++o) {
                        const int k = j - o;
                        if (k < 0 || k > 10) continue;
#pragma unroll
                        for (int q = 0; q < 5; ++q) b[o][q] += w11[k] * t[q];
                    }
                }
                const int gx = ox + co;
#pragma unroll
                for (int o = 0; o < V2; ++o) {
                    const int ro = r0 + o, gy = oy + ro;
                    if (gx >= w || gy >= h) continue;
                    const int ri = (ro + 2 * LR) * RG + (co + 2 * LR);
                    const float x = in_x[ri], y = in_y[ri];
                    const float grad = b[o][0] + y * b[o][1] - b[o][3] + 2.0f * x * b[o][2] - 2.0f * b[o][4];
                    const float d = x - y;
                    l1_local += fabsf(d);
                    const float sg = (d != d) ? d : copysignf(1.0f, d);
                    float g = (1.0f - lambda) * sg / m_total;
                    g += -lambda * grad / m_total;
                    dl[(pb + (size_t)gy * w + gx) * 3 + ch] = g;
                }
            }
            __syncthreads();
        }
        float l1s = block_sum_fixed(l1_local, s_red);
        float sss = block_sum_fixed(ssim_local, s_red + LOSS_THREADS / 32);
        if (tid == 0) {
            partials[(size_t)blk * 2 + 0] = l1s;
            partials[(size_t)blk * 2 + 1] = sss;
        }
        __syncthreads();
    }
}

// The same loss with fused multiply-adds, two independent accumulators per
// packed f32x2 instruction (per lane the same rounding as one fmaf): the
// statistics as (x, y), (x^2, y^2), xy; the maps as (P, Q), (R, Q mu_y),
// R mu_x. Pass outputs live in shared memory as float2 planes of those pairs
// (plus one float plane), in the same regions as the exact kernel's.
__device__ __forceinline__ float2 f2(float a, float b) { return make_float2(a, b); }

__global__ void __launch_bounds__(LOSS_THREADS) k_loss_fused(const DevCam* __restrict__ cams, int nviews,
                                                             const uint32_t* total_dev, int total_host,
                                                             const float* __restrict__ rgb, float lambda,
                                                             float* __restrict__ dl, float* __restrict__ partials) {
    extern __shared__ float smem[];
    float* in_x = smem;
    float* in_y = in_x + RG * RG;
    float* tmp = in_y + RG * RG;   // pass 1 out: float2 [RG][MG] x2 + float [RG][MG]; pass 3 out: [MG][LTP] likewise
    float* st = tmp + 5 * RG * MG;  // pass 2 out (maps): float2 [MG][MGP] x2 + float [MG][MGP]
    float* kw = st + 5 * MG * MGP;
    float* s_red = kw + 16;
    float2* t01 = reinterpret_cast<float2*>(tmp);
    float2* t23 = t01 + RG * MG;
    float* t4 = reinterpret_cast<float*>(t23 + RG * MG);
    float2* m01 = reinterpret_cast<float2*>(st);
    float2* m23 = m01 + MG * MGP;
    float* m4 = reinterpret_cast<float*>(m23 + MG * MGP);
    float2* g01 = reinterpret_cast<float2*>(tmp);
    float2* g23 = g01 + MG * LTP;
    float* g4 = reinterpret_cast<float*>(g23 + MG * LTP);
    const int tid = threadIdx.x;
    if (tid == 0) {
        // gaussian_kernel_1d(5, 1.5), backward.rs:759-772
        float sum = 0.0f;
        float v[11];
        for (int i = 0; i < 11; ++i) {
            float d = (float)i - 5.0f;
            v[i] = exp_cr(-0.5f * d * d / (1.5f * 1.5f));
            sum += v[i];
        }
        for (int i = 0; i < 11; ++i) kw[i] = v[i] / sum;
    }
    __syncthreads();
    float2 ww[11];  // the taps, duplicated for the packed lanes
#pragma unroll
    for (int k = 0; k < 11; ++k) ww[k] = f2(kw[k], kw[k]);
    const int total = total_dev ? (int)*total_dev : total_host;
    for (int blk = blockIdx.x; blk < total; blk += gridDim.x) {
        int v = 0;
        while (v + 1 < nviews && cams[v + 1].loss_base <= blk) ++v;
        const DevCam& c = cams[v];
        const int w = c.width, h = c.height;
        const int lb = blk - c.loss_base;
        const int ox = (lb % c.loss_bx) * LT, oy = (lb / c.loss_bx) * LT;
        const float m_total = (float)((size_t)w * h * 3);
        const float* tgt = c.target;
        const size_t pb = (size_t)c.pix_base;
        float l1_local = 0.0f, ssim_local = 0.0f;
        for (int ch = 0; ch < 3; ++ch) {
            for (int i = tid; i < RG * RG; i += LOSS_THREADS) {
                int r = i / RG, cc = i - r * RG;
                int gx = ox - 2 * LR + cc, gy = oy - 2 * LR + r;
                float xv = 0.0f, yv = 0.0f;
                if (gx >= 0 && gx < w && gy >= 0 && gy < h) {
                    size_t p = (size_t)gy * w + gx;
                    xv = rgb[(pb + p) * 3 + ch];
                    yv = tgt[p * 4 + ch];
                }
                in_x[i] = xv;
                in_y[i] = yv;
            }
            __syncthreads();
            // pass 1: horizontal blur of (x, y), (x^2, y^2), xy over rows
            // [0, RG), map columns [0, MG); a run of H1 outputs per thread
            for (int it = tid; it < RG * (MG / H1); it += LOSS_THREADS) {
                const int r = it / (MG / H1), c0 = (it - r * (MG / H1)) * H1;
                const float* rx = in_x + r * RG + c0;
                const float* ry = in_y + r * RG + c0;
                float2 a01[H1], a23[H1];
                float a4[H1];
#pragma unroll
                for (int o = 0; o < H1; ++o) {
                    a01[o] = a23[o] = f2(0.0f, 0.0f);
                    a4[o] = 0.0f;
                }
#pragma unroll
                for (int j = 0; j < H1 + 10; ++j) {
                    const float2 xy = f2(rx[j], ry[j]);
                    const float2 sq = __fmul2_rn(xy, xy);
                    const float cr = xy.x * xy.y;
#pragma unroll
                    for (int o = 0; o < H1; ++o) {
                        const int k = j - o;
                        if (k < 0 || k > 10) continue;
                        a01[o] = __ffma2_rn(ww[k], xy, a01[o]);
                        a23[o] = __ffma2_rn(ww[k], sq, a23[o]);
                        a4[o] = __fmaf_rn(ww[k].x, cr, a4[o]);
                    }
                }
#pragma unroll
                for (int o = 0; o < H1; ++o) {
                    const int q = r * MG + c0 + o;
                    t01[q] = a01[o];
                    t23[q] = a23[o];
                    t4[q] = a4[o];
                }
            }
            __syncthreads();
            // pass 2: vertical blur -> statistics, then the per-pixel SSIM
            // maps (zero outside the image)
            for (int it = tid; it < MG * (MG / V1); it += LOSS_THREADS) {
                const int cm = it % MG, r0 = (it / MG) * V1;
                float2 mu01[V1], mu23[V1];
                float mu4[V1];
#pragma unroll
                for (int o = 0; o < V1; ++o) {
                    mu01[o] = mu23[o] = f2(0.0f, 0.0f);
                    mu4[o] = 0.0f;
                }
#pragma unroll
                for (int j = 0; j < V1 + 10; ++j) {
                    const int q = (r0 + j) * MG + cm;
                    const float2 u01 = t01[q], u23 = t23[q];
                    const float u4 = t4[q];
#pragma unroll
                    for (int o = 0; o < V1; ++o) {
                        const int k = j - o;
                        if (k < 0 || k > 10) continue;
                        mu01[o] = __ffma2_rn(ww[k], u01, mu01[o]);
                        mu23[o] = __ffma2_rn(ww[k], u23, mu23[o]);
                        mu4[o] = __fmaf_rn(ww[k].x, u4, mu4[o]);
                    }
                }
                const int gx = ox - LR + cm;
#pragma unroll
                for (int o = 0; o < V1; ++o) {
                    const int rm = r0 + o, gy = oy - LR + rm;
                    float P = 0.0f, Q = 0.0f, R = 0.0f, QM = 0.0f, RM = 0.0f;
                    if (gx >= 0 && gx < w && gy >= 0 && gy < h) {
                        const float s = ssim_maps<true>(mu01[o].x, mu01[o].y, mu23[o].x, mu23[o].y, mu4[o], P, Q, R, QM, RM);
                        if (rm >= LR && rm < LR + LT && cm >= LR && cm < LR + LT) ssim_local += s;
                    }
                    const int q = rm * MGP + cm;
                    m01[q] = f2(P, Q);
                    m23[q] = f2(R, QM);
                    m4[q] = RM;
                }
            }
            __syncthreads();
            // pass 3: horizontal blur of the maps: rows [0, MG), output cols [0, LT)
            for (int it = tid; it < MG * (LT / H2); it += LOSS_THREADS) {
                const int rm = it % MG, c0 = (it / MG) * H2;
#pragma unroll 1
                for (int pl = 0; pl < 2; ++pl) {
                    const float2* row = (pl ? m23 : m01) + rm * MGP + c0;
                    float2 a[H2];
#pragma unroll
                    for (int o = 0; o < H2; ++o) a[o] = f2(0.0f, 0.0f);
#pragma unroll
                    for (int j = 0; j < H2 + 10; ++j) {
                        const float2 t = row[j];
#pragma unroll
                        for (int o = 0; o < H2; ++o) {
                            const int k = j - o;
                            if (k < 0 || k > 10) continue;
                            a[o] = __ffma2_rn(ww[k], t, a[o]);
                        }
                    }
                    float2* out = (pl ? g23 : g01) + rm * LTP + c0;
#pragma unroll
                    for (int o = 0; o < H2; ++o) out[o] = a[o];
                }
                {
                    const float* row = m4 + rm * MGP + c0;
                    float a[H2];
#pragma unroll
                    for (int o = 0; o < H2; ++o) a[o] = 0.0f;
#pragma unroll
                    for (int j = 0; j < H2 + 10; ++j) {
                        const float t = row[j];
#pragma unroll
                        for (int o = 0; o < H2; ++o) {
                            const int k = j - o;
                            if (k < 0 || k > 10) continue;
                            a[o] = __fmaf_rn(ww[k].x, t, a[o]);
                        }
                    }
#pragma unroll
                    for (int o = 0; o < H2; ++o) g4[rm * LTP + c0 + o] = a[o];
                }
            }
            __syncthreads();
            // pass 4: vertical blur -> gradient, combined with the L1 term
            for (int it = tid; it < LT * (LT / V2); it += LOSS_THREADS) {
                const int co = it % LT, r0 = (it / LT) * V2;
                float2 b01[V2], b23[V2];
                float b4[V2];
#pragma unroll
                for (int o = 0; o < V2; ++o) {
                    b01[o] = b23[o] = f2(0.0f, 0.0f);
                    b4[o] = 0.0f;
                }
#pragma unroll
                for (int j = 0; j < V2 + 10; ++j) {
                    const int q = (r0 + j) * LTP + co;
                    const float2 u01 = g01[q], u23 = g23[q];
                    const float u4 = g4[q];
#pragma unroll
                    for (int o = 0; o < V2; ++o) {
                        const int k = j - o;
                        if (k < 0 || k > 10) continue;
                        b01[o] = __ffma2_rn(ww[k], u01, b01[o]);
                        b23[o] = __ffma2_rn(ww[k], u23, b23[o]);
                        b4[o] = __fmaf_rn(ww[k].x, u4, b4[o]);
                    }
                }
                const int gx = ox + co;
#pragma unroll
                for (int o = 0; o < V2; ++o) {
                    const int ro = r0 + o, gy = oy + ro;
                    if (gx >= w || gy >= h) continue;
                    const int ri = (ro + 2 * LR) * RG + (co + 2 * LR);
                    const float x = in_x[ri], y = in_y[ri];
                    const float grad = b01[o].x + y * b01[o].y - b23[o].y + 2.0f * x * b23[o].x - 2.0f * b4[o];
                    const float d = x - y;
                    l1_local += fabsf(d);
                    const float sg = (d != d) ? d : copysignf(1.0f, d);
                    float g = (1.0f - lambda) * sg / m_total;
                    g += -lambda * grad / m_total;
                    dl[(pb + (size_t)gy * w + gx) * 3 + ch] = g;
                }
            }
            __syncthreads();
        }
        float l1s = block_sum_fixed(l1_local, s_red);
        float sss = block_sum_fixed(ssim_local, s_red + LOSS_THREADS / 32);
        if (tid == 0) {
            partials[(size_t)blk * 2 + 0] = l1s;
            partials[(size_t)blk * 2 + 1] = sss;
        }
        __syncthreads();
    }
}

// One CTA per view: each thread sums a strided subset of the view's per-block
// partials in double, then a fixed-shape tree combines the threads, so the
// result does not depend on scheduling.
constexpr int FIN_THREADS = 256;
__global__ void __launch_bounds__(FIN_THREADS) k_loss_finalize(const DevCam* __restrict__ cams, int nviews,
                                                               const float* __restrict__ partials, float lambda,
                                                               float* __restrict__ losses) {
    __shared__ double s_l1[FIN_THREADS], s_ss[FIN_THREADS];
    const int v = blockIdx.x, tid = threadIdx.x;
    if (v >= nviews) return;
    const DevCam& c = cams[v];
    const int nb = c.loss_bx * ((c.height + LT - 1) / LT);
    double l1 = 0.0, ss = 0.0;
    for (int b = tid; b < nb; b += FIN_THREADS) {
        l1 += (double)partials[(size_t)(c.loss_base + b) * 2 + 0];
        ss += (double)partials[(size_t)(c.loss_base + b) * 2 + 1];
    }
    s_l1[tid] = l1;
    s_ss[tid] = ss;
    __syncthreads();
    for (int o = FIN_THREADS / 2; o > 0; o >>= 1) {
        if (tid < o) {
            s_l1[tid] += s_l1[tid + o];
            s_ss[tid] += s_ss[tid + o];
        }
        __syncthreads();
    }
    if (tid == 0) {
        float m = (float)((size_t)c.width * c.height * 3);
        float l1m = (float)(s_l1[0] / (double)m);
        float ssm = (float)(s_ss[0] / (double)m);
        losses[v] = (1.0f - lambda) * l1m + lambda * (1.0f - ssm);
    }
}

cudaError_t prepare_loss_kernel() {
    static std::mutex mu;
    static bool ready[64];
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(mu);
    if (ready[dev]) return cudaSuccess;
    e = cudaFuncSetAttribute(k_loss, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)LOSS_SMEM);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_loss_fused, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)LOSS_SMEM);
    if (e == cudaSuccess) ready[dev] = true;
    return e;
}

cudaError_t launch_loss(const DevCam* cams, int nviews, int total_blocks, const float* rgb, float lambda, float* dl,
                        float* partials, float* losses, const uint32_t* total_dev, bool exact, cudaStream_t st) {
    cudaError_t e = prepare_loss_kernel();
    if (e != cudaSuccess) return e;
    const int sms = device_sm_count();
    int grid = total_dev ? sms * 2 : (total_blocks < sms * 2 ? total_blocks : sms * 2);
    if (grid < 1) grid = 1;
    if (exact)
        k_loss<<<grid, LOSS_THREADS, LOSS_SMEM, st>>>(cams, nviews, total_dev, total_blocks, rgb, lambda, dl, partials);
    else
        k_loss_fused<<<grid, LOSS_THREADS, LOSS_SMEM, st>>>(cams, nviews, total_dev, total_blocks, rgb, lambda, dl,
                                                            partials);
    if (nviews > 0) k_loss_finalize<<<nviews, FIN_THREADS, 0, st>>>(cams, nviews, partials, lambda, losses);
    return cudaGetLastError();
}

}  // namespace rgs

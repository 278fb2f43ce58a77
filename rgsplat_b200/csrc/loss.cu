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
// formed once per run) and accumulate with FMA; the SSIM map arithmetic
// keeps the reference's expressions. The scalar loss is reduced per CTA and
// then per view in a fixed order (deterministic).
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
    const float C1 = 0.01f * 0.01f;
    const float C2 = 0.03f * 0.03f;
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
                        float mx = mu[o][0], my = mu[o][1];
                        float sx2 = mu[o][2] - mx * mx;
                        float sy2 = mu[o][3] - my * my;
                        float sxy = mu[o][4] - mx * my;
                        float a1 = 2.0f * mx * my + C1;
                        float a2 = 2.0f * sxy + C2;
                        float b1 = mx * mx + my * my + C1;
                        float b2 = sx2 + sy2 + C2;
                        float num = a1 * a2;
                        float den = b1 * b2;
                        if (rm >= LR && rm < LR + LT && cm >= LR && cm < LR + LT) ssim_local += num / den;
                        float inv_den = 1.0f / den;
                        P = inv_den * (2.0f * my * a2) - (num / (den * den)) * (2.0f * mx * b2);
                        Q = inv_den * (2.0f * a1);
                        R = -(num / (den * den)) * b1;
                        QM = Q * my;
                        RM = R * mx;
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
    if (e == cudaSuccess) ready[dev] = true;
    return e;
}

cudaError_t launch_loss(const DevCam* cams, int nviews, int total_blocks, const float* rgb, float lambda, float* dl,
                        float* partials, float* losses, const uint32_t* total_dev, cudaStream_t st) {
    cudaError_t e = prepare_loss_kernel();
    if (e != cudaSuccess) return e;
    const int sms = device_sm_count();
    int grid = total_dev ? sms * 2 : (total_blocks < sms * 2 ? total_blocks : sms * 2);
    if (grid < 1) grid = 1;
    k_loss<<<grid, LOSS_THREADS, LOSS_SMEM, st>>>(cams, nviews, total_dev, total_blocks, rgb, lambda, dl, partials);
    if (nviews > 0) k_loss_finalize<<<nviews, FIN_THREADS, 0, st>>>(cams, nviews, partials, lambda, losses);
    return cudaGetLastError();
}

}  // namespace rgs

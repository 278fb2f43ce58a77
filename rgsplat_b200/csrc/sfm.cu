// sfm.cu -- gaussians_from_sfm (src/pipeline/sfm.rs:365-404) and its
// estimate_initial_scales (:408-450) on the device.
//
// The reference sorts the points by x (a stable sort), finds each point's x
// in that order with Rust's binary search, and averages the 3 smallest
// distances to the other points of a 50-wide window there. Here:
//   k_sfm_keys    x -> an order-preserving u64 (-0.0 folded onto +0.0, so
//                 ties are ties exactly when partial_cmp says Equal), split
//                 into two u32 halves for two stable LSD radix sorts (low
//                 half first, then the high half gathered through the first
//                 permutation), which together are the stable sort by x;
//   k_sfm_sorted  the points gathered into x-sorted f64 planes;
//   k_sfm_scales  one thread per sorted position: Rust's binary search on the
//                 sorted x (the last of equal keys), the window, the 3
//                 smallest squared distances kept in registers (sqrt is
//                 monotone, so these are the 3 smallest distances), their
//                 square roots summed smallest first, / k, rounded to f32;
//   k_sfm_init    one thread per point: Gaussian3D::new, the DC colour from
//                 powf(u / 255, 2.2), log of the clamped scale, logit(0.1),
//                 written straight into the parameter planes.
// The distances use the reference's f64 operation order unfused (the
// translation unit is built with --fmad=false).
#include <cstdint>

#include "rgs_internal.cuh"
#include "rgs_math.cuh"

namespace rgs {

namespace {

__device__ __forceinline__ unsigned long long x_sort_key(double x) {
    if (x == 0.0) x = 0.0;  // -0.0 -> +0.0
    const unsigned long long b = (unsigned long long)__double_as_longlong(x);
    return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}

__global__ void __launch_bounds__(256) k_sfm_keys(const double* __restrict__ xyz, int n, uint32_t* __restrict__ klo,
                                                  uint32_t* __restrict__ khi, uint32_t* __restrict__ idx,
                                                  int* __restrict__ bad) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double x = xyz[3 * (size_t)i], y = xyz[3 * (size_t)i + 1], z = xyz[3 * (size_t)i + 2];
    if (!isfinite(x) || !isfinite(y) || !isfinite(z)) *bad = 1;
    const unsigned long long k = x_sort_key(x);
    klo[i] = (uint32_t)k;
    khi[i] = (uint32_t)(k >> 32);
    idx[i] = (uint32_t)i;
}

// Second sort's input: the high halves in the order of the first sort.
__global__ void __launch_bounds__(256) k_sfm_gather_hi(const uint32_t* __restrict__ perm1, const uint32_t* __restrict__ khi,
                                                       int n, uint32_t* __restrict__ khi2, uint32_t* __restrict__ idx2) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    const uint32_t i = perm1[p];
    khi2[p] = khi[i];
    idx2[p] = i;
}

__global__ void __launch_bounds__(256) k_sfm_sorted(const double* __restrict__ xyz, const uint32_t* __restrict__ perm, int n,
                                                    double* __restrict__ sx, double* __restrict__ sy, double* __restrict__ sz) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    const size_t i = perm[p];
    sx[p] = xyz[3 * i];
    sy[p] = xyz[3 * i + 1];
    sz[p] = xyz[3 * i + 2];
}

// Rust's slice::binary_search_by (the size-halving form without an early
// exit): among equal keys the last one is found. Returns -1 for Err, which
// the caller maps to unwrap_or(0); a point always finds its own x.
__device__ __forceinline__ long long rust_binary_search(const double* __restrict__ xs, int n, double t) {
    int base = 0, size = n;
    while (size > 1) {
        const int half = size >> 1;
        const int mid = base + half;
        if (!(__ldg(xs + mid) > t)) base = mid;
        size -= half;
    }
    return __ldg(xs + base) == t ? base : -1;
}

__global__ void __launch_bounds__(256) k_sfm_scales(const double* __restrict__ sx, const double* __restrict__ sy,
                                                    const double* __restrict__ sz, const uint32_t* __restrict__ perm, int n,
                                                    float* __restrict__ scales) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    const uint32_t i = perm[p];
    const double qx = sx[p], qy = sy[p], qz = sz[p];
    const int window = n < 50 ? n : 50;
    long long f = rust_binary_search(sx, n, qx);
    const int found = f < 0 ? 0 : (int)f;
    const int start = found - (found < window / 2 ? found : window / 2);
    const int end = start + window < n ? start + window : n;
    double d0 = __longlong_as_double(0x7ff0000000000000ll), d1 = d0, d2 = d0;  // +inf
    int cnt = 0;
    for (int j = start; j < end; ++j) {
        if (__ldg(perm + j) == i) continue;
        const double dx = __ldg(sx + j) - qx;
        const double dy = __ldg(sy + j) - qy;
        const double dz = __ldg(sz + j) - qz;
        const double d = dx * dx + dy * dy + dz * dz;
        ++cnt;
        if (d < d2) {
            if (d < d1) {
                d2 = d1;
                if (d < d0) { d1 = d0; d0 = d; } else { d1 = d; }
            } else {
                d2 = d;
            }
        }
    }
    float s;
    if (cnt == 0) {
        s = 0.01f;
    } else {
        const int k = cnt < 3 ? cnt : 3;
        double acc = -0.0;
        acc += sqrt(d0);
        if (k > 1) acc += sqrt(d1);
        if (k > 2) acc += sqrt(d2);
        s = __double2float_rn(acc / (double)k);
    }
    scales[i] = s;
}

// f32::powf(x, 2.2) for x = u / 255 in [0, 1]: exp(y ln x) in double, rounded once.
__device__ __forceinline__ float pow22(float x) {
    if (x == 0.0f) return 0.0f;
    return __double2float_rn(exp_core_d((double)2.2f * log_pos_d((double)x)));
}

__global__ void __launch_bounds__(256) k_sfm_init(const double* __restrict__ xyz, const uint8_t* __restrict__ rgb,
                                                  const float* __restrict__ scales, int n, float4* __restrict__ planes,
                                                  int cap) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float SH_C0_INV = 1.0f / 0.28209479177387814f;
    const float p = 0.1f;
    const float opacity_logit = log_cr(p / (1.0f - p));  // math::logit(0.1)
    const float s = log_cr(fmaxf(scales[i], 1e-4f));
    float dc[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) dc[c] = (pow22((float)rgb[3 * (size_t)i + c] / 255.0f) - 0.5f) * SH_C0_INV;
    float4* o = planes + i;
    const size_t C = (size_t)cap;
    o[0] = make_float4(__double2float_rn(xyz[3 * (size_t)i]), __double2float_rn(xyz[3 * (size_t)i + 1]),
                       __double2float_rn(xyz[3 * (size_t)i + 2]), opacity_logit);
    o[C] = make_float4(1.0f, 0.0f, 0.0f, 0.0f);
    o[2 * C] = make_float4(s, s, s, 0.0f);
    // sh[0], sh[16], sh[32] (the three DC terms) open planes 3, 7 and 11
#pragma unroll
    for (int q = 0; q < 12; ++q) o[(3 + q) * C] = make_float4(q % 4 == 0 ? dc[q / 4] : 0.0f, 0.0f, 0.0f, 0.0f);
}

inline unsigned blocks(int n) { return (unsigned)((n + 255) / 256); }

}  // namespace

int sfm_init_planes(const double* xyz, const uint8_t* rgb, int n, float4* planes, int cap, SfmScratch& w, int grid,
                    cudaStream_t st, int* bad_host, cudaError_t* err) {
    *err = cudaSuccess;
    *bad_host = 0;
    if (n <= 0) return 0;
    const size_t N = (size_t)n;
    if ((*err = w.f64.ensure(N * 8 * 3 + 64)) != cudaSuccess) return 0;
    if ((*err = w.scales.ensure(N * 4 + 16)) != cudaSuccess) return 0;
    if ((*err = w.flag.ensure(16)) != cudaSuccess) return 0;
    // sub-arrays on 16-byte boundaries (the sort stages full sub-tiles by bulk copy)
    const size_t NA = (N + 3) & ~(size_t)3;
    if ((*err = w.u32.ensure(NA * 4 * 4 + 64)) != cudaSuccess) return 0;
    uint32_t* klo = w.u32.as<uint32_t>();
    uint32_t* khi = klo + NA;
    uint32_t* idx = khi + NA;
    uint32_t* khi2 = idx + NA;
    int* bad = w.flag.as<int>();
    w.sort.fault = bad + 1;
    if ((*err = cudaMemsetAsync(bad, 0, 2 * sizeof(int), st)) != cudaSuccess) return 0;
    k_sfm_keys<<<blocks(n), 256, 0, st>>>(xyz, n, klo, khi, idx, bad);
    int cur = radix_sort_pairs(klo, idx, (uint32_t)n, nullptr, 32, w.sort, grid, st, err);
    if (*err != cudaSuccess) return 0;
    const uint32_t* perm1 = cur ? w.sort.vals2.as<uint32_t>() : idx;
    // the second sort's values take the place of the first sort's keys
    uint32_t* idx2 = klo;
    k_sfm_gather_hi<<<blocks(n), 256, 0, st>>>(perm1, khi, n, khi2, idx2);
    cur = radix_sort_pairs(khi2, idx2, (uint32_t)n, nullptr, 32, w.sort, grid, st, err);
    if (*err != cudaSuccess) return 0;
    const uint32_t* perm = cur ? w.sort.vals2.as<uint32_t>() : idx2;
    double* sx = w.f64.as<double>();
    double* sy = sx + N;
    double* sz = sy + N;
    k_sfm_sorted<<<blocks(n), 256, 0, st>>>(xyz, perm, n, sx, sy, sz);
    k_sfm_scales<<<blocks(n), 256, 0, st>>>(sx, sy, sz, perm, n, w.scales.as<float>());
    k_sfm_init<<<blocks(n), 256, 0, st>>>(xyz, rgb, w.scales.as<float>(), n, planes, cap);
    if ((*err = cudaGetLastError()) != cudaSuccess) return 0;
    int flags[2] = {0, 0};
    if ((*err = cudaMemcpyAsync(flags, bad, 2 * sizeof(int), cudaMemcpyDeviceToHost, st)) != cudaSuccess) return 0;
    if ((*err = cudaStreamSynchronize(st)) != cudaSuccess) return 0;
    *bad_host = flags[0];
    if (flags[1]) *err = cudaErrorLaunchTimeout;  // a sort pass's staged copies timed out
    return 0;
}

}  // namespace rgs

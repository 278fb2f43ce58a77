// layout.cu -- conversions between the reference's host records and the
// device planes, plus input validation.
//
// Host side (the reference's types): Gaussian3D is 59 packed f32
// (src/math/mod.rs:27-46); GaussianGrad is 60 f32 in field order
// (src/cpu/backward.rs:33-41); Adam moments are 59 f32 per Gaussian in the
// same flatten_grad order (src/pipeline/optimizer.rs:165-173). Device side:
// 15 float4 planes (rgs_internal.cuh).
#include "rgs_internal.cuh"

namespace rgs {

__global__ void k_aos_to_planes(const float* __restrict__ aos, float4* __restrict__ planes, int n, int cap) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float* r = aos + (size_t)i * NP;
    float4* o = planes + i;
    o[0] = make_float4(r[0], r[1], r[2], r[3]);
    o[(size_t)cap] = make_float4(r[4], r[5], r[6], r[7]);
    o[2 * (size_t)cap] = make_float4(r[8], r[9], r[10], 0.0f);
#pragma unroll
    for (int p = 0; p < 12; ++p) o[(size_t)(3 + p) * cap] = make_float4(r[11 + 4 * p], r[12 + 4 * p], r[13 + 4 * p], r[14 + 4 * p]);
}

__global__ void k_planes_to_aos(const float4* __restrict__ planes, float* __restrict__ aos, int n, int cap) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float* r = aos + (size_t)i * NP;
    const float4* s = planes + i;
    float4 a = s[0], b = s[(size_t)cap], c = s[2 * (size_t)cap];
    r[0] = a.x; r[1] = a.y; r[2] = a.z; r[3] = a.w;
    r[4] = b.x; r[5] = b.y; r[6] = b.z; r[7] = b.w;
    r[8] = c.x; r[9] = c.y; r[10] = c.z;
#pragma unroll
    for (int p = 0; p < 12; ++p) {
        float4 v = s[(size_t)(3 + p) * cap];
        r[11 + 4 * p] = v.x; r[12 + 4 * p] = v.y; r[13 + 4 * p] = v.z; r[14 + 4 * p] = v.w;
    }
}

// Planes -> flatten_grad rows of `stride` floats (60: GaussianGrad with
// screen_grad_norm from the pad lane; 59: an Adam-moment row).
__global__ void k_grads_to_aos(const float4* __restrict__ planes, float* __restrict__ aos, int n, int cap, int stride) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float* r = aos + (size_t)i * stride;
    const float4* s = planes + i;
    float4 a = s[0], b = s[(size_t)cap], c = s[2 * (size_t)cap];
    r[0] = a.x; r[1] = a.y; r[2] = a.z;
    r[3] = b.x; r[4] = b.y; r[5] = b.z; r[6] = b.w;
    r[7] = c.x; r[8] = c.y; r[9] = c.z;
    r[10] = a.w;
#pragma unroll
    for (int p = 0; p < 12; ++p) {
        float4 v = s[(size_t)(3 + p) * cap];
        r[11 + 4 * p] = v.x; r[12 + 4 * p] = v.y; r[13 + 4 * p] = v.z; r[14 + 4 * p] = v.w;
    }
    if (stride == NG) r[59] = c.w;
}

__global__ void k_aos_to_grad_planes(const float* __restrict__ aos, float4* __restrict__ planes, int n, int cap, int stride) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float* r = aos + (size_t)i * stride;
    float4* o = planes + i;
    o[0] = make_float4(r[0], r[1], r[2], r[10]);
    o[(size_t)cap] = make_float4(r[3], r[4], r[5], r[6]);
    o[2 * (size_t)cap] = make_float4(r[7], r[8], r[9], stride == NG ? r[59] : 0.0f);
#pragma unroll
    for (int p = 0; p < 12; ++p) o[(size_t)(3 + p) * cap] = make_float4(r[11 + 4 * p], r[12 + 4 * p], r[13 + 4 * p], r[14 + 4 * p]);
}

__global__ void k_check_finite(const float4* __restrict__ planes, int n, int cap, int* __restrict__ flag) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    bool bad = false;
#pragma unroll
    for (int p = 0; p < NPL; ++p) {
        float4 v = planes[(size_t)p * cap + i];
        bad |= !isfinite(v.x) || !isfinite(v.y) || !isfinite(v.z) || (p != 2 && !isfinite(v.w));
    }
    if (bad) atomicOr(flag, 1);
}

void launch_aos_to_planes(const float* aos, float4* planes, int n, int cap, cudaStream_t st) {
    if (n > 0) k_aos_to_planes<<<(n + 255) / 256, 256, 0, st>>>(aos, planes, n, cap);
}
void launch_planes_to_aos(const float4* planes, float* aos, int n, int cap, cudaStream_t st) {
    if (n > 0) k_planes_to_aos<<<(n + 255) / 256, 256, 0, st>>>(planes, aos, n, cap);
}
void launch_grads_to_aos(const float4* gplanes, float* aos, int n, int cap, int stride, cudaStream_t st) {
    if (n > 0) k_grads_to_aos<<<(n + 255) / 256, 256, 0, st>>>(gplanes, aos, n, cap, stride);
}
void launch_aos_to_grad_planes(const float* aos, float4* planes, int n, int cap, int stride, cudaStream_t st) {
    if (n > 0) k_aos_to_grad_planes<<<(n + 255) / 256, 256, 0, st>>>(aos, planes, n, cap, stride);
}
void launch_check_finite(const float4* planes, int n, int cap, int* flag, cudaStream_t st) {
    if (n > 0) k_check_finite<<<(n + 255) / 256, 256, 0, st>>>(planes, n, cap, flag);
}

}  // namespace rgs

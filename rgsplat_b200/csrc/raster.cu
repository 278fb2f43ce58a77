// raster.cu -- colour-space conversions at the two ends of the path:
//   * cpu::rasterize's output stage (src/cpu/rasterizer.rs:38-48, 171-186):
//     the preview framebuffer as RGBA float (colour, 1 - T) or as
//     Framebuffer::to_u8_srgb's gamma-encoded RGBA8, packed on the device
//     from the forward blend's colour and final transmittance so only the
//     final format crosses to the host;
//   * load_target's input stage (src/io/images.rs:67-72): an 8-bit sRGB
//     RGBA image becomes the loss's linear RGBA f32 target on the device, so
//     4 bytes per pixel cross PCIe instead of 16.
#include "rgs_internal.cuh"
#include "rgs_math.cuh"

namespace rgs {

__global__ void __launch_bounds__(256) k_pack_rgba(const float* __restrict__ rgb, const float* __restrict__ final_t, size_t npix,
                                                   float4* __restrict__ out) {
    for (size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x; p < npix; p += (size_t)gridDim.x * blockDim.x)
        out[p] = make_float4(rgb[p * 3], rgb[p * 3 + 1], rgb[p * 3 + 2], 1.0f - final_t[p]);
}

// RGB -> linear_to_srgb(clamp(v, 0, 1)) * 255 as u8; alpha -> clamp * 255 as u8
// (f32::clamp keeps a NaN, which the u8 cast turns into 0).
__device__ __forceinline__ unsigned char srgb8(float v) { return as_u8(linear_to_srgb(rclamp(v, 0.0f, 1.0f)) * 255.0f); }

__global__ void __launch_bounds__(256) k_pack_srgb8(const float* __restrict__ rgb, const float* __restrict__ final_t, size_t npix,
                                                    uchar4* __restrict__ out) {
    for (size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x; p < npix; p += (size_t)gridDim.x * blockDim.x)
        out[p] = make_uchar4(srgb8(rgb[p * 3]), srgb8(rgb[p * 3 + 1]), srgb8(rgb[p * 3 + 2]),
                             as_u8(rclamp(1.0f - final_t[p], 0.0f, 1.0f) * 255.0f));
}

// One thread per pixel: RGB through srgb_to_linear(u / 255), alpha u / 255.
// The conversion depends only on the byte, so each CTA first tabulates
// srgb_to_linear(u / 255) and u / 255 for the 256 byte values (one thread per
// entry, the same arithmetic as per pixel) and then looks pixels up: four
// shared-memory reads per pixel instead of three double-precision powers.
__global__ void __launch_bounds__(256) k_srgb8_to_linear(const uchar4* __restrict__ in, size_t npix, float4* __restrict__ out) {
    __shared__ float s_lin[256], s_alpha[256];
    {
        const float x = (float)threadIdx.x / 255.0f;
        s_lin[threadIdx.x] = srgb_to_linear(x);
        s_alpha[threadIdx.x] = x;
    }
    __syncthreads();
    for (size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x; p < npix; p += (size_t)gridDim.x * blockDim.x) {
        const uchar4 c = in[p];
        out[p] = make_float4(s_lin[c.x], s_lin[c.y], s_lin[c.z], s_alpha[c.w]);
    }
}

void launch_srgb8_to_linear(const void* rgba8, size_t npix, float* out, cudaStream_t st) {
    if (npix == 0) return;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const size_t want = (npix + 255) / 256;
    const unsigned grid = (unsigned)(want < (size_t)sms * 4 ? want : (size_t)sms * 4);
    k_srgb8_to_linear<<<grid, 256, 0, st>>>((const uchar4*)rgba8, npix, (float4*)out);
}

void launch_pack_framebuffer(const float* rgb, const float* final_t, size_t npix, int srgb8, void* out, cudaStream_t st) {
    if (npix == 0) return;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const size_t want = (npix + 255) / 256;
    const unsigned grid = (unsigned)(want < (size_t)sms * 8 ? want : (size_t)sms * 8);
    if (srgb8)
        k_pack_srgb8<<<grid, 256, 0, st>>>(rgb, final_t, npix, (uchar4*)out);
    else
        k_pack_rgba<<<grid, 256, 0, st>>>(rgb, final_t, npix, (float4*)out);
}

}  // namespace rgs

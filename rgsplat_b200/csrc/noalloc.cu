// noalloc.cu -- rgs_photometric_loss_grad_noalloc: the photometric loss and
// dL/dpixel on caller-owned device buffers, with no device allocation at all.
// It is for callers that must not allocate device memory themselves or through
// this library: applications whose own pool owns the whole GPU, and paths that
// cannot afford cudaMalloc's implicit synchronisation.
//
// Everything the loss kernels need besides the caller's buffers lives in one
// file-scope static __device__ array: a 256-byte header holding the view
// descriptor (DevCam) and then two floats (L1 sum, SSIM sum) per 32x32 loss
// block. Host code cannot use the array's name as a device address, so the
// address is looked up with cudaGetSymbolAddress, with the device current,
// on the first call on each device (that first call also sets the loss
// kernel's shared-memory limit; it should come before any stream capture).
// The kernels are the ones rgs_photometric_loss_grad runs (loss.cu) with the
// default options (fused blur taps); only where their scratch lives differs.
//
// The array keeps whatever the previous call left in it, and nothing in it has
// to start at zero: the header is written by a one-thread kernel on the
// caller's stream before the loss kernels, and every loss block writes its own
// partial-sum pair before the per-view finalize reads it. Calls that overlap
// on one device (two host threads, or two streams with work in flight at once)
// share the array and race; callers serialise them.
#include <mutex>

#include "rgs_internal.cuh"
#include "../../include/rgsplat.h"

namespace rgs {

constexpr int NA_HEADER = 256;
constexpr int NA_MAX_BLOCKS = RGS_NOALLOC_MAX_LOSS_BLOCKS;
constexpr int NA_TILE = 32;   // loss block edge (loss.cu)
static_assert(sizeof(DevCam) <= NA_HEADER, "view descriptor must fit the scratch header");

static __device__ __align__(256) unsigned char g_noalloc_scratch[NA_HEADER + NA_MAX_BLOCKS * 2 * sizeof(float)];

__global__ void k_noalloc_put_cam(DevCam c, DevCam* dst) { *dst = c; }

namespace {
constexpr int NA_MAX_DEVICES = 64;
std::mutex g_na_mutex;
void* g_na_ptr[NA_MAX_DEVICES];

void put_err(char* err, size_t err_len, const char* msg) {
    if (!err || err_len == 0) return;
    size_t i = 0;
    for (; msg[i] && i + 1 < err_len; ++i) err[i] = msg[i];
    err[i] = 0;
}

int cuda_err(char* err, size_t err_len, cudaError_t e) {
    put_err(err, err_len, cudaGetErrorString(e));
    return RGS_ERR_CUDA;
}
}  // namespace

}  // namespace rgs

using namespace rgs;

extern "C" int rgs_photometric_loss_grad_noalloc(int device, const float* rendered_rgb, const float* target_rgba,
                                                 uint32_t width, uint32_t height, float lambda, float* loss_out,
                                                 float* dl_out, void* cuda_stream, char* err, size_t err_len) {
    put_err(err, err_len, "");
    if (!rendered_rgb || !target_rgba || !loss_out || !dl_out) {
        put_err(err, err_len, "null argument");
        return RGS_ERR_INVALID_ARG;
    }
    if (width == 0 || height == 0 || width > 65535 || height > 65535) {
        put_err(err, err_len, "width and height must be in 1..65535");
        return RGS_ERR_INVALID_ARG;
    }
    const uint32_t bx = (width + NA_TILE - 1) / NA_TILE, by = (height + NA_TILE - 1) / NA_TILE;
    const uint64_t blocks = (uint64_t)bx * by;
    if (blocks > (uint64_t)NA_MAX_BLOCKS) {
        char msg[200];
        snprintf(msg, sizeof msg,
                 "image of %ux%u needs %llu loss blocks of 32x32; the static scratch holds %d "
                 "(4096x4096 pixels at most)",
                 width, height, (unsigned long long)blocks, NA_MAX_BLOCKS);
        put_err(err, err_len, msg);
        return RGS_ERR_CAPACITY;
    }
    if (device < 0 || device >= NA_MAX_DEVICES) {
        put_err(err, err_len, "device ordinal out of range");
        return RGS_ERR_INVALID_ARG;
    }
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || device >= ndev) {
        cudaGetLastError();
        put_err(err, err_len, "no such CUDA device");
        return RGS_ERR_NO_DEVICE;
    }
    int prev = 0;
    if ((e = cudaGetDevice(&prev)) != cudaSuccess) return cuda_err(err, err_len, e);
    if ((e = cudaSetDevice(device)) != cudaSuccess) return cuda_err(err, err_len, e);
    int rc = RGS_OK;
    unsigned char* scratch = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_na_mutex);
        if (!g_na_ptr[device]) {
            void* p = nullptr;
            e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
            // the loss kernel's shared-memory limit, set on this device now
            // rather than on a later call that may be inside a stream capture
            if (e == cudaSuccess) e = prepare_loss_kernel();
            if (e != cudaSuccess) rc = cuda_err(err, err_len, e);
            else g_na_ptr[device] = p;
        }
        scratch = (unsigned char*)g_na_ptr[device];
    }
    if (rc == RGS_OK) {
        DevCam c{};
        c.width = (int)width;
        c.height = (int)height;
        c.loss_bx = (int)bx;
        c.target = target_rgba;
        DevCam* cam_dev = (DevCam*)scratch;
        float* partials = (float*)(scratch + NA_HEADER);
        cudaStream_t st = (cudaStream_t)cuda_stream;
        k_noalloc_put_cam<<<1, 1, 0, st>>>(c, cam_dev);
        if ((e = cudaGetLastError()) == cudaSuccess)
            e = launch_loss(cam_dev, 1, (int)blocks, rendered_rgb, lambda, dl_out, partials, loss_out, nullptr, false, st);
        if (e != cudaSuccess) rc = cuda_err(err, err_len, e);
    }
    cudaSetDevice(prev);
    return rc;
}

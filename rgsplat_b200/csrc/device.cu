// device.cu -- per-device facts the launchers size their grids from, looked up
// once per device ordinal under a mutex, so a process that drives several GPUs
// (one context per device, or the no-allocation loss on more than one device)
// never reuses one device's answer for another; and the calling thread's
// device-memory counter (the context whose entry point is running).
#include <mutex>

#include "rgs_internal.cuh"

namespace rgs {

thread_local MemCounter* t_mem = nullptr;

namespace {
constexpr int MAX_DEVICES = 64;
std::mutex g_dev_mutex;
int g_sms[MAX_DEVICES];
}  // namespace

int device_sm_count() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= MAX_DEVICES) {
        cudaGetLastError();
        return 148;
    }
    std::lock_guard<std::mutex> lock(g_dev_mutex);
    if (!g_sms[dev]) {
        int s = 0;
        if (cudaDeviceGetAttribute(&s, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || s <= 0) {
            cudaGetLastError();
            return 148;
        }
        g_sms[dev] = s;
    }
    return g_sms[dev];
}

}  // namespace rgs

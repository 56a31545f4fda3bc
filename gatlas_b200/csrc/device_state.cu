// Per-device fault word and scratch cache.
#include <mutex>

#include "common.cuh"
#include "device_state.cuh"

namespace gatlas {

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_mu;
int *g_fault[kMaxDevices] = {nullptr};
void *g_scratch[kScratchSlots][kMaxDevices] = {{nullptr}};
size_t g_scratch_bytes[kScratchSlots][kMaxDevices] = {{0}};
cudaStream_t g_streams[kMaxDevices][kPoolStreams] = {{nullptr}};

int current_device() {
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return -1;
    return dev;
}
}  // namespace

int *device_fault_word() {
    const int dev = current_device();
    if (dev < 0) return nullptr;
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_fault[dev]) {
        int *p = nullptr;
        if (cudaMalloc(&p, sizeof(int)) != cudaSuccess) return nullptr;
        if (cudaMemset(p, 0, sizeof(int)) != cudaSuccess) {
            cudaFree(p);
            return nullptr;
        }
        g_fault[dev] = p;
    }
    return g_fault[dev];
}

void *device_scratch(size_t bytes, int slot) {
    const int dev = current_device();
    if (dev < 0 || slot < 0 || slot >= kScratchSlots) return nullptr;
    std::lock_guard<std::mutex> lk(g_mu);
    if (g_scratch_bytes[slot][dev] < bytes) {
        if (g_scratch[slot][dev]) {
            cudaDeviceSynchronize();
            cudaFree(g_scratch[slot][dev]);
            g_scratch[slot][dev] = nullptr;
            g_scratch_bytes[slot][dev] = 0;
        }
        // round up to 2 MiB so that slowly growing requests do not reallocate often
        const size_t want = (bytes + ((size_t)2 << 20) - 1) & ~(((size_t)2 << 20) - 1);
        void *p = nullptr;
        if (cudaMalloc(&p, want) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        g_scratch[slot][dev] = p;
        g_scratch_bytes[slot][dev] = want;
    }
    return g_scratch[slot][dev];
}

cudaStream_t pool_stream(int i) {
    const int dev = current_device();
    if (dev < 0 || i < 0 || i >= kPoolStreams) return nullptr;
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_streams[dev][i] && cudaStreamCreateWithFlags(&g_streams[dev][i], cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        g_streams[dev][i] = nullptr;
    }
    return g_streams[dev][i];
}

}  // namespace gatlas

extern "C" int gatlas_device_faults(int *flags, int clear) {
    int *w = gatlas::device_fault_word();
    if (!w) return gatlas::set_error(GATLAS_ERR_CUDA, "fault word unavailable");
    int v = 0;
    cudaError_t e = cudaMemcpy(&v, w, sizeof(int), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return gatlas::set_error(GATLAS_ERR_CUDA, "read fault word: %s", cudaGetErrorString(e));
    if (clear && v) cudaMemset(w, 0, sizeof(int));
    if (flags) *flags = v;
    return GATLAS_OK;
}

extern "C" int gatlas_device_count(int *count) {
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (count) *count = (e == cudaSuccess) ? n : 0;
    if (e != cudaSuccess) return gatlas::set_error(GATLAS_ERR_CUDA, "cudaGetDeviceCount: %s", cudaGetErrorString(e));
    return GATLAS_OK;
}

extern "C" int gatlas_set_device(int device) {
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return gatlas::set_error(GATLAS_ERR_CUDA, "cudaSetDevice(%d): %s", device, cudaGetErrorString(e));
    return GATLAS_OK;
}

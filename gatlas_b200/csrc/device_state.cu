// Per-device fault word and scratch cache.
#include <mutex>

#include "common.cuh"
#include "device_state.cuh"

namespace gatlas {

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_mu;
void *g_scratch[kScratchSlots][kMaxDevices] = {{nullptr}};
size_t g_scratch_bytes[kScratchSlots][kMaxDevices] = {{0}};
cudaStream_t g_streams[kMaxDevices][kPoolStreams] = {{nullptr}};

int current_device() {
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return -1;
    return dev;
}
}  // namespace

// The fault word lives in this file's device memory, so no call ever
// allocates it: one int per GPU that loads the library, zero when the module
// loads.  Host code may not use the name as a device address; the address is
// looked up once per device with cudaGetSymbolAddress, with that device
// current.
namespace {
__device__ int g_fault_word;
int *g_fault[kMaxDevices] = {nullptr};
}  // namespace

int *device_fault_word() {
    const int dev = current_device();
    if (dev < 0) return nullptr;
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_fault[dev]) {
        void *p = nullptr;
        if (cudaGetSymbolAddress(&p, g_fault_word) != cudaSuccess || !p) {
            cudaGetLastError();
            return nullptr;
        }
        g_fault[dev] = static_cast<int *>(p);
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

// ---------------------------------------------------------------------------
// bounded-wait self-test
// ---------------------------------------------------------------------------
namespace gatlas {
namespace {

// One thread waits on an mbarrier in the way every TMA/tcgen05 kernel here
// does: try_wait polls bounded by `limit_ns` of wall time.  With `arrive` the
// barrier's phase completes first and the wait succeeds; without it nothing
// ever completes the phase, the wait runs out, the fault word gets its bit and
// the kernel returns.
__global__ void selftest_wait_kernel(int *fault, uint64_t limit_ns, int arrive, int *result) {
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x != 0) return;
    mbar_init(&bar, 1);
    fence_mbarrier_init();
    if (arrive) mbar_arrive(&bar);
    uint64_t t0;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t0));
    bool ok = false;
    while (true) {
        if (mbar_try_wait(&bar, 0)) {
            ok = true;
            break;
        }
        uint64_t t;
        asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
        if (t - t0 > limit_ns) break;
    }
    if (!ok) report_fault(fault, kFaultSelftestWait);
    *result = ok ? 1 : 0;
}

}  // namespace
}  // namespace gatlas

extern "C" int gatlas_selftest_bounded_wait(int64_t limit_ns, int arrive, int *completed, void *stream) {
    using namespace gatlas;
    if (limit_ns <= 0 || limit_ns > 2000000000LL || !completed)
        return set_error(GATLAS_ERR_INVALID, "selftest: limit must be in (0, 2 s] and `completed` non-null");
    int *fault = device_fault_word();
    int *res = static_cast<int *>(device_scratch(sizeof(int), 1));
    if (!fault || !res) return set_error(GATLAS_ERR_NOMEM, "selftest: device words");
    selftest_wait_kernel<<<1, 32, 0, (cudaStream_t)stream>>>(fault, (uint64_t)limit_ns, arrive, res);
    int rc = check_launch("selftest_wait_kernel");
    if (rc) return rc;
    if (cudaMemcpyAsync(completed, res, sizeof(int), cudaMemcpyDeviceToHost, (cudaStream_t)stream) != cudaSuccess ||
        cudaStreamSynchronize((cudaStream_t)stream) != cudaSuccess)
        return check_launch("selftest result");
    return GATLAS_OK;
}

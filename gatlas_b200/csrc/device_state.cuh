// Per-device library state: the fault word that bounded device waits set when
// they give up, and cached scratch buffers for callers that pass no workspace.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>

namespace gatlas {

// Bits of the per-device fault word (read with gatlas_device_faults()).
enum FaultCode : int {
    kFaultSaxpyBulkWait = 1 << 0,
    kFaultGemvTmaWait = 1 << 1,
    kFaultGemmTmaWait = 1 << 2,
    kFaultTcProducerWait = 1 << 3,
    kFaultTcMmaWait = 1 << 4,
    kFaultTcEpilogueWait = 1 << 5,
    kFaultSelftestWait = 1 << 6,
};

// Device pointer to the current device's fault word: a file-scope __device__
// int (zero at module load, never allocated) whose address is looked up on
// the first use per device; nullptr if that lookup failed.
int *device_fault_word();

// Current device's cached scratch buffer `slot` of at least `bytes` (grown on
// demand, never shrunk).  Slot 0 serves the engines' workspaces, slot 1 the
// device copies of the host-buffer entry points.  nullptr on failure.  Not
// safe to grow during graph capture.
constexpr int kScratchSlots = 2;
void *device_scratch(size_t bytes, int slot = 0);

// Per-device non-blocking streams owned by the library (created on first use).
constexpr int kPoolStreams = 3;
cudaStream_t pool_stream(int i);

#ifdef __CUDACC__
__device__ __forceinline__ void report_fault(int *word, int code) {
    if (word) atomicOr(word, code);
}
#endif

}  // namespace gatlas

// Host-side TMA tensor-map encoding through the driver entry point (no
// link-time dependency on libcuda: the library loads on machines without a
// driver and resolves cuTensorMapEncodeTiled at first use).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace gatlas {

// Encodes a tiled tensor map.  dims/strides as in cuTensorMapEncodeTiled:
// dims[0] is the innermost (contiguous) extent, strides[i] is the byte stride
// of dimension i+1.  Returns GATLAS_OK or an error status (message recorded).
int make_tensor_map(CUtensorMap *map, CUtensorMapDataType dtype, int rank, void *base,
                    const uint64_t *dims, const uint64_t *strides_bytes, const uint32_t *box,
                    CUtensorMapSwizzle swizzle);

}  // namespace gatlas

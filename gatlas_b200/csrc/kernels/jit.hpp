// Run-time compilation of SIMT GEMM parameter points (see jit.cpp).
#pragma once

#include <cuda_runtime.h>

#include <string>

namespace gatlas {
namespace jit {

struct Point {
    int scalar;  // 0 float, 1 double
    int ta, tb, gh, gw, bh, bw, vl;
    int image = 0;  // 0: buffer template (gemm_simt.cuh), 1: image template (gemm_image.cuh)
};

bool available();                          // NVRTC loaded
bool point_ok(const Point &p);             // the template accepts the point
std::string simt_name(const Point &p);     // C++ name of the instantiation
std::string simt_source(const Point &p);   // full CUDA source compiled for the point
// Compiled kernel for the point on the current device (cached).
int simt_function(const Point &p, void **fn);
// Launch a compiled kernel with one by-value argument block.
int launch(void *fn, unsigned gx, unsigned gy, unsigned gz, unsigned block, void *args, cudaStream_t stream);
// Launch with several by-value arguments and dynamic shared memory.
int launch_args(void *fn, unsigned gx, unsigned gy, unsigned gz, unsigned block, unsigned smem, void **args,
                cudaStream_t stream);

}  // namespace jit
}  // namespace gatlas

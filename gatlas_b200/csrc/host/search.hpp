// Autotuning search spaces and the expectation-maximization search.
//
// Reference: getParams and the EM loops of benchMatmul.cpp (:217-304,
// :536-627), benchMatvec.cpp (:202-289) and benchSaxpy.cpp (:158-276).  The
// enumeration order and limits are the reference's, with the device's
// maximum work-group size taken as CUDA's 1024 threads per block.
#pragma once

#include <stddef.h>

#include <vector>

#include "kernel.hpp"

namespace gatlas {
namespace host {

constexpr size_t kMaxWorkGroupSize = 1024;

// Points for a matmul search; -1 means "free" for group size, block height
// and extra parameter.
std::vector<std::vector<size_t>> matmul_search(KernelMatmul &k, size_t vectorLength, size_t maxBlockHeight,
                                               size_t maxGroupSize, bool gemm, size_t M, size_t N, size_t K,
                                               bool tA, bool tB, long groupSize, long blockHeight, long extraParam);

std::vector<std::vector<size_t>> matvec_search(KernelMatvec &k, size_t vectorLength, size_t maxBlockHeight,
                                               size_t maxGroupSize, bool gemv, size_t M, size_t N, bool tA,
                                               long groupSize, long blockHeight, long extraParam);

std::vector<std::vector<size_t>> saxpy_search(KernelSaxpy &k, size_t vectorLength, size_t maxBlockHeight,
                                              size_t maxGroupSize, size_t M, size_t N, long groupHeight,
                                              long groupWidth, long blockHeight, long blockWidth, long extraParam);

}  // namespace host
}  // namespace gatlas

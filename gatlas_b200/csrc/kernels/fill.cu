// Seeded device-side data generators (same streams as the host oracle's
// counter-based generators: element i = f(splitmix64(splitmix64(seed) + offset + i))).
#include <type_traits>

#include "../common.cuh"

namespace gatlas {

template <typename T>
__device__ __forceinline__ T uniform_from(uint64_t x);

template <>
__device__ __forceinline__ float uniform_from<float>(uint64_t x) {
    const int64_t q = (int64_t)(x >> 40) - (int64_t)(1 << 23);  // 24 random bits, exact
    return (float)q * 0x1p-23f;
}

template <>
__device__ __forceinline__ double uniform_from<double>(uint64_t x) {
    const int64_t q = (int64_t)(x >> 11) - ((int64_t)1 << 52);
    return (double)q * 0x1p-52;
}

template <typename T>
__global__ void fill_kernel(T *out, size_t n, int dist, uint64_t key, uint64_t offset, T value) {
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        if (dist == GATLAS_DIST_CONST) {
            out[i] = value;
            continue;
        }
        const uint64_t x = splitmix64(key + offset + i);
        if (dist == GATLAS_DIST_UNIFORM) {
            out[i] = uniform_from<T>(x);
        } else {
            const int e = (int)((x >> 8) % 17) - 8;
            const T v = (T)ldexpf(1.0f, e);
            out[i] = (x & 1) ? -v : v;
        }
    }
}

template <typename T>
__device__ __forceinline__ T fill_value(int dist, uint64_t x) {
    if (dist == GATLAS_DIST_UNIFORM) return uniform_from<T>(x);
    const int e = (int)((x >> 8) % 17) - 8;
    const T v = (T)ldexpf(1.0f, e);
    return (x & 1) ? -v : v;
}

// 16-byte stores: each thread writes runs of 16 bytes (4 floats / 2 doubles)
// of the same counter-based stream; out is 16-byte aligned, n a multiple of
// the run length.  The values are those fill_kernel writes.
template <typename T>
__global__ void __launch_bounds__(256) fill_vec_kernel(T *out, size_t n, int dist, uint64_t key, uint64_t offset,
                                                       T value) {
    constexpr int R = 16 / sizeof(T);
    using V = typename std::conditional<sizeof(T) == 4, float4, double2>::type;
    const size_t runs = n / R, stride = (size_t)gridDim.x * blockDim.x;
    for (size_t r = (size_t)blockIdx.x * blockDim.x + threadIdx.x; r < runs; r += stride) {
        T v[R];
        const uint64_t base = key + offset + r * R;
#pragma unroll
        for (int j = 0; j < R; ++j) v[j] = dist == GATLAS_DIST_CONST ? value : fill_value<T>(dist, splitmix64(base + j));
        V w;
        memcpy(&w, v, sizeof(w));
        __stcs(reinterpret_cast<V *>(out) + r, w);
    }
}

template <typename T>
static int fill_launch(T *out, size_t n, int dist, uint64_t seed, uint64_t offset, T value,
                       cudaStream_t stream) {
    if (n == 0) return GATLAS_OK;
    if (!out) return set_error(GATLAS_ERR_INVALID, "fill: null pointer");
    if (dist < GATLAS_DIST_UNIFORM || dist > GATLAS_DIST_CONST)
        return set_error(GATLAS_ERR_INVALID, "fill: unknown distribution %d", dist);
    const size_t cap = (size_t)sm_count() * 16;
    constexpr size_t R = 16 / sizeof(T);
    const uint64_t key = splitmix64(seed);
    size_t done = 0;
    if (aligned16(out) && n >= R) {
        const size_t runs = n / R;
        size_t grid = (runs + 255) / 256;
        if (grid > cap) grid = cap;
        fill_vec_kernel<T><<<(unsigned)grid, 256, 0, stream>>>(out, runs * R, dist, key, offset, value);
        done = runs * R;
    }
    if (done < n) {  // unaligned base or the tail
        size_t grid = (n - done + 255) / 256;
        if (grid > cap) grid = cap;
        fill_kernel<T><<<(unsigned)grid, 256, 0, stream>>>(out + done, n - done, dist, key, offset + done, value);
    }
    return check_launch("fill_kernel");
}

}  // namespace gatlas

extern "C" int gatlas_fill_f32(float *out, size_t n, int dist, uint64_t seed, uint64_t offset,
                               float value, void *stream) {
    return gatlas::fill_launch<float>(out, n, dist, seed, offset, value, (cudaStream_t)stream);
}

extern "C" int gatlas_fill_f64(double *out, size_t n, int dist, uint64_t seed, uint64_t offset,
                               double value, void *stream) {
    return gatlas::fill_launch<double>(out, n, dist, seed, offset, value, (cudaStream_t)stream);
}

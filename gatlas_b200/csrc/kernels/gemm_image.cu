// Image engine for matmul: SIMT math fed by TMA tensor-map tiles.
//
// Host side of gemm_image.cuh: tensor maps (3-D: inner dimension, rows,
// packed instance; 128-byte swizzle for the tiles whose rows run along K),
// prebuilt instantiations of the common points, run-time compilation for the
// rest of the reference's image space (work group up to 16 x 16, inner
// blocking up to 16).
#include <cuda.h>

#include <cstring>

#include "../common.cuh"
#include "../device_state.cuh"
#include "../tma.hpp"
#include "gemm_engines.hpp"
#include "gemm_image.cuh"
#include "jit.hpp"

namespace gatlas {

namespace {

template <typename T>
struct ImgLaunch {
    img::TmapBlob a, b;
    img::ImgArgs<T> args;
};

using ImgFn = void (*)(dim3, unsigned, int, cudaStream_t, const void *);

template <typename T, bool TA, bool TB, int GH, int GW, int BH, int BW>
void img_launch_point(dim3 grid, unsigned smem, int, cudaStream_t s, const void *p) {
    const ImgLaunch<T> &l = *static_cast<const ImgLaunch<T> *>(p);
    auto k = img::gemm_image_kernel<T, TA, TB, GH, GW, BH, BW>;
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k<<<grid, GH * GW, smem, s>>>(l.a, l.b, l.args);
}

template <typename T, bool TA, bool TB, int GH, int GW, int BH, int BW>
constexpr int img_smem() {
    return img::ImgTile<T, TA, TB, GH, GW, BH, BW>::SMEM;
}

struct ImgEntry {
    int scalar, ta, tb, gh, gw, bh, bw;
    ImgFn fn;
};

#define IMG_E(T, SC, TA, TB, GH, GW, BH, BW) \
    {SC, TA, TB, GH, GW, BH, BW, &img_launch_point<T, (TA) != 0, (TB) != 0, GH, GW, BH, BW>}
#define IMG_LAYOUTS(T, SC, GH, GW, BH, BW) \
    IMG_E(T, SC, 0, 0, GH, GW, BH, BW), IMG_E(T, SC, 0, 1, GH, GW, BH, BW), IMG_E(T, SC, 1, 0, GH, GW, BH, BW), \
        IMG_E(T, SC, 1, 1, GH, GW, BH, BW)

const ImgEntry kImgTable[] = {
    IMG_LAYOUTS(float, 0, 16, 16, 8, 8), IMG_LAYOUTS(float, 0, 16, 16, 8, 4), IMG_LAYOUTS(float, 0, 8, 8, 8, 4),
    IMG_LAYOUTS(float, 0, 16, 16, 4, 4), IMG_LAYOUTS(float, 0, 8, 8, 4, 4),
    IMG_LAYOUTS(double, 1, 16, 16, 4, 4), IMG_LAYOUTS(double, 1, 8, 8, 4, 2), IMG_LAYOUTS(double, 1, 8, 8, 8, 2),
};

const ImgEntry *img_find(int scalar, int ta, int tb, int gh, int gw, int bh, int bw) {
    for (const ImgEntry &e : kImgTable)
        if (e.scalar == scalar && e.ta == ta && e.tb == tb && e.gh == gh && e.gw == gw && e.bh == bh && e.bw == bw)
            return &e;
    return nullptr;
}

// Dynamic shared memory of a point (ImgTile::SMEM computed on the host).
int img_smem_bytes(int scalar, bool ta, bool tb, int gh, int gw, int bh, int bw) {
    const int es = scalar ? 8 : 4;
    const int BK = scalar ? 16 : 32;
    const int BM = gh * bh, BN = gw * bw;
    const int align = 1024 / es;
    const int a_raw = (BM * BK + align - 1) / align * align, b_raw = (BN * BK + align - 1) / align * align;
    const int PA = ta ? BM : BM + 4, PB = tb ? BN + 4 : BN;
    return (2 * (a_raw + b_raw) + (ta ? 0 : BK * PA) + (tb ? BK * PB : 0)) * es + 1024;  // + alignment slack
}

template <typename T>
int matmul_image_impl(const gatlas_matmul_desc *d, const Geometry &g, const T *A, const T *B, T *C,
                      cudaStream_t stream) {
    const int scalar = sizeof(T) == 8 ? 1 : 0;
    int gh = (int)d->group_h, gw = (int)d->group_w, bh = (int)d->block_h, bw = (int)d->block_w;
    if (gh == 0 && gw == 0 && bh == 0 && bw == 0) {
        gh = gw = 16;
        bh = scalar ? 4 : 8;
        bw = scalar ? 4 : 8;
    }
    jit::Point pt{scalar, g.ta ? 1 : 0, g.tb ? 1 : 0, gh, gw, bh, bw, 0, 1};
    if (!jit::point_ok(pt))
        return set_error(GATLAS_ERR_UNSUPPORTED,
                         "matmul image engine: tile %dx%d x %dx%d does not fit the tensor-map alignment rules", gh, gw,
                         bh, bw);
    if (g.K == 0) {
        // empty contraction (C = beta*C or 0) has no tiles to map: SIMT path
        gatlas_matmul_desc s = *d;
        s.engine = GATLAS_ENGINE_BUFFER;
        s.group_h = s.group_w = s.block_h = s.block_w = s.vector_length = 0;
        if (scalar) return gatlas_matmul_f64(&s, (const double *)A, (const double *)B, (double *)C, nullptr, 0, stream);
        return gatlas_matmul_f32(&s, (const float *)A, (const float *)B, (float *)C, nullptr, 0, stream);
    }
    const int es = (int)sizeof(T), per16 = 16 / es;
    // operand rows and batch strides must be 16-byte aligned for TMA
    if (g.lda % per16 || g.ldb % per16 || !aligned16(A) || !aligned16(B) ||
        (g.batch > 1 && (g.stride_a % per16 || g.stride_b % per16)))
        return set_error(GATLAS_ERR_UNSUPPORTED,
                         "matmul image engine: operands need 16-byte aligned rows and bases (lda, ldb multiples of %d)",
                         per16);
    const int BK = scalar ? 16 : 32;
    const int BM = gh * bh, BN = gw * bw;
    const int64_t a_inner = g.ta ? g.M : g.K, a_rows = g.ta ? g.K : g.M;
    const int64_t b_inner = g.tb ? g.K : g.N, b_rows = g.tb ? g.N : g.K;
    CUtensorMap ma, mb;
    const CUtensorMapDataType dt = scalar ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
    {
        const uint64_t dims[3] = {(uint64_t)a_inner, (uint64_t)a_rows, (uint64_t)g.batch};
        const uint64_t str[2] = {(uint64_t)g.lda * es, (uint64_t)(g.batch > 1 ? g.stride_a : g.lda * a_rows) * es};
        const uint32_t box[3] = {(uint32_t)(g.ta ? BM : BK), (uint32_t)(g.ta ? BK : BM), 1};
        int rc = make_tensor_map(&ma, dt, 3, const_cast<T *>(A), dims, str, box,
                                 g.ta ? CU_TENSOR_MAP_SWIZZLE_NONE : CU_TENSOR_MAP_SWIZZLE_128B);
        if (rc) return rc;
    }
    {
        const uint64_t dims[3] = {(uint64_t)b_inner, (uint64_t)b_rows, (uint64_t)g.batch};
        const uint64_t str[2] = {(uint64_t)g.ldb * es, (uint64_t)(g.batch > 1 ? g.stride_b : g.ldb * b_rows) * es};
        const uint32_t box[3] = {(uint32_t)(g.tb ? BK : BN), (uint32_t)(g.tb ? BN : BK), 1};
        int rc = make_tensor_map(&mb, dt, 3, const_cast<T *>(B), dims, str, box,
                                 g.tb ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_NONE);
        if (rc) return rc;
    }
    ImgLaunch<T> l;
    static_assert(sizeof(img::TmapBlob) == sizeof(CUtensorMap), "tensor map size");
    std::memcpy(&l.a, &ma, sizeof(ma));
    std::memcpy(&l.b, &mb, sizeof(mb));
    l.args.C = C;
    l.args.M = g.M;
    l.args.N = g.N;
    l.args.K = g.K;
    l.args.ldc = g.ldc;
    l.args.stride_c = g.stride_c;
    l.args.alpha = (T)d->alpha;
    l.args.beta = (T)d->beta;
    l.args.gemm = d->gemm;
    l.args.fault = device_fault_word();
    const int64_t gx = (g.N + BN - 1) / BN, gy = (g.M + BM - 1) / BM;
    if (gx > 0x7fffffff || gy > 65535) return set_error(GATLAS_ERR_INVALID, "matmul: grid too large");
    const dim3 grid((unsigned)gx, (unsigned)gy, (unsigned)g.batch);
    const int smem = img_smem_bytes(scalar, g.ta, g.tb, gh, gw, bh, bw);
    if (smem > 227 * 1024) return set_error(GATLAS_ERR_UNSUPPORTED, "matmul image engine: tile needs %d bytes of smem", smem);
    if (const ImgEntry *e = img_find(scalar, g.ta, g.tb, gh, gw, bh, bw)) {
        e->fn(grid, (unsigned)smem, 0, stream, &l);
        return check_launch("gemm_image_kernel");
    }
    void *fn = nullptr;
    int rc = jit::simt_function(pt, &fn);
    if (rc) return rc;
    void *args[] = {&l.a, &l.b, &l.args};
    return jit::launch_args(fn, grid.x, grid.y, grid.z, (unsigned)(gh * gw), (unsigned)smem, args, stream);
}

}  // namespace

int matmul_image_f32(const gatlas_matmul_desc *d, const Geometry &g, const float *A, const float *B, float *C,
                     cudaStream_t stream) {
    return matmul_image_impl<float>(d, g, A, B, C, stream);
}

int matmul_image_f64(const gatlas_matmul_desc *d, const Geometry &g, const double *A, const double *B, double *C,
                     cudaStream_t stream) {
    return matmul_image_impl<double>(d, g, A, B, C, stream);
}

int image_supported(int scalar, const gatlas_matmul_desc *d) {
    int gh = (int)d->group_h, gw = (int)d->group_w, bh = (int)d->block_h, bw = (int)d->block_w;
    if (gh == 0 && gw == 0 && bh == 0 && bw == 0) return 1;
    if (img_find(scalar, d->trans_a != 0, d->trans_b != 0, gh, gw, bh, bw)) return 1;
    const jit::Point pt{scalar, d->trans_a != 0, d->trans_b != 0, gh, gw, bh, bw, 0, 1};
    return jit::available() && jit::point_ok(pt) ? 2 : 0;
}

}  // namespace gatlas

// Kernel families on B200: buffers, data, checks and launches.
#include "kernel.hpp"

#include <cmath>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <sstream>

#include "../../../include/gatlas.h"
#include "../kernels/gemm_engines.hpp"
#include "../kernels/jit.hpp"
#include "../kernels/reference.hpp"

namespace gatlas {
namespace host {

std::ostream &operator<<(std::ostream &os, const KernelInterface &k) { return k.print(os); }

// ---------------------------------------------------------------------------
// buffers
// ---------------------------------------------------------------------------
bool DeviceArray::ensure(size_t nbytes, bool host_mirror) {
    if (bytes == nbytes && d && (!host_mirror || h)) return true;
    release();
    if (nbytes == 0) return true;
    if (cudaMalloc(&d, nbytes) != cudaSuccess) {
        d = nullptr;
        std::cerr << "error: device allocation of " << nbytes << " bytes" << std::endl;
        return false;
    }
    if (host_mirror && cudaMallocHost(&h, nbytes) != cudaSuccess) {
        h = nullptr;
        release();
        std::cerr << "error: pinned host allocation of " << nbytes << " bytes" << std::endl;
        return false;
    }
    bytes = nbytes;
    return true;
}

void DeviceArray::release() {
    if (d) cudaFree(d);
    if (h) cudaFreeHost(h);
    d = h = nullptr;
    bytes = 0;
}

bool DeviceArray::upload(cudaStream_t s) const {
    return !bytes || cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, s) == cudaSuccess;
}

bool DeviceArray::download(cudaStream_t s) const {
    return !bytes || cudaMemcpyAsync(h, d, bytes, cudaMemcpyDeviceToHost, s) == cudaSuccess;
}

// ---------------------------------------------------------------------------
// host data helpers (OCLAppUtil.hpp:28-61, 212-264)
// ---------------------------------------------------------------------------
template <typename T>
static T posrand() {
    // OCLAppUtil.hpp:28-33: the double from drand48 is converted to the
    // scalar type, and drawn again while zero
    T a;
    while (0 == (a = (T)drand48())) ;
    return a;
}

template <typename T>
static void fillrand(void *p, size_t n) {
    T *q = static_cast<T *>(p);
    for (size_t i = 0; i < n; ++i) q[i] = posrand<T>();
}

template <typename T>
static void fillconst(void *p, size_t n, T v) {
    T *q = static_cast<T *>(p);
    for (size_t i = 0; i < n; ++i) q[i] = v;
}

template <typename T>
static bool check_array(const void *p, size_t n, T v) {
    const T *q = static_cast<const T *>(p);
    bool ok = true;
    for (size_t i = 0; i < n; ++i)
        if (q[i] != v) ok = false;
    return ok;
}

template <typename T>
static long double absdiff(const void *a, const void *b, size_t n) {
    const T *x = static_cast<const T *>(a);
    const T *y = static_cast<const T *>(b);
    long double acc = 0;
    for (size_t i = 0; i < n; ++i) acc += fabsl((long double)(x[i] - y[i]));
    return acc;
}

template <typename T>
static void print_array(const void *p, size_t width, size_t height) {
    const T *q = static_cast<const T *>(p);
    for (size_t i = 0; i < height; ++i) {
        std::cerr << "[" << i << "]";
        for (size_t j = 0; j < width; ++j) std::cerr << " " << q[i * width + j];
        std::cerr << std::endl;
    }
}

static int engine_of(Variant v) {
    switch (v) {
        case Variant::Buffer: return GATLAS_ENGINE_BUFFER;
        case Variant::Image: return GATLAS_ENGINE_IMAGE;
        case Variant::TcBf16: return GATLAS_ENGINE_TC_BF16;
        case Variant::TcSplit3: return GATLAS_ENGINE_TC_SPLIT3;
        case Variant::TcSplit6: return GATLAS_ENGINE_TC_SPLIT6;
        case Variant::TcFp8: return GATLAS_ENGINE_TC_FP8;
    }
    return -1;
}

static bool is_tc(Variant v) {
    return v == Variant::TcBf16 || v == Variant::TcSplit3 || v == Variant::TcSplit6 || v == Variant::TcFp8;
}

// Normwise error budgets of the tensor-core engines against FP64.
static double tc_budget(Variant v) {
    switch (v) {
        case Variant::TcBf16: return std::ldexp(1.0, -7);
        case Variant::TcSplit3: return 8e-6;
        case Variant::TcFp8: return std::ldexp(1.0, -4);  // E4M3 unit roundoff per operand
        default: return 2.5e-6;
    }
}

static bool sync(cudaStream_t s) {
    cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        std::cerr << "error: " << cudaGetErrorString(e) << std::endl;
        return false;
    }
    return true;
}

// ---------------------------------------------------------------------------
// matmul
// ---------------------------------------------------------------------------
KernelMatmul::KernelMatmul(Scalar s, Variant v, size_t vectorLength)
    : MatmulParams(v), scalar_(s), variant_(v), vl_(vectorLength) {}

std::string KernelMatmul::kernelName() const {
    // KernelMatmulBuffer.hpp:58-62, KernelMatmulImage.hpp:63-67
    std::stringstream ss;
    ss << "matmul" << variant_name(variant_) << scalar_name(scalar_) << vl_;
    return ss.str();
}

static gatlas_matmul_desc matmul_desc_of(const MatmulParams &p, Variant v, size_t vl, double alpha, double beta) {
    gatlas_matmul_desc d;
    std::memset(&d, 0, sizeof(d));
    d.engine = engine_of(v);
    d.gemm = p.generalizedMatmul();
    d.trans_a = p.transposeA();
    d.trans_b = p.transposeB();
    d.m = p.dimM();
    d.n = p.dimN();
    d.k = p.dimK();
    d.batch = p.packedCalc();
    d.alpha = alpha;
    d.beta = beta;
    if (!is_tc(v)) {
        d.group_h = (uint32_t)p.groupHeight();
        d.group_w = (uint32_t)p.groupWidth();
        d.block_h = (uint32_t)p.blockHeight();
        d.block_w = (uint32_t)p.blockWidth();
        d.vector_length = (uint32_t)vl;
        d.extra = (uint32_t)p.extraParam();
    }
    return d;
}

bool KernelMatmul::build() {
    if (!validParams()) {
        std::cerr << "error: invalid parameters" << std::endl;
        return false;
    }
    const gatlas_matmul_desc d = matmul_desc_of(*this, variant_, vl_, alpha_, beta_);
    const int support = gatlas_matmul_supported(scalar_ == Scalar::Double, &d);
    if (support == 0) {
        std::cerr << "error: no kernel for this point";
        return false;
    }
    if (support == 2) {
        // no prebuilt instantiation: compile it now, as the reference builds
        // its OpenCL program for every point (GatlasBenchmark.cpp:286-301)
        void *fn = nullptr;
        if (jit::simt_function(jit_point(), &fn) != GATLAS_OK) {
            char buf[512];
            gatlas_last_error(buf, sizeof(buf));
            std::cerr << "error: " << buf;
            return false;
        }
    }
    return true;
}

int KernelMatmul::supportLevel() const {
    const gatlas_matmul_desc d = matmul_desc_of(*this, variant_, vl_, alpha_, beta_);
    return gatlas_matmul_supported(scalar_ == Scalar::Double, &d);
}

jit::Point KernelMatmul::jit_point() const {
    return jit::Point{scalar_ == Scalar::Double ? 1 : 0, transposeA() ? 1 : 0, transposeB() ? 1 : 0,
                      (int)groupHeight(), (int)groupWidth(), (int)blockHeight(), (int)blockWidth(),
                      variant_ == Variant::Image ? 0 : (int)vl_, variant_ == Variant::Image ? 1 : 0};
}

bool KernelMatmul::setArgs(bool syncInput) {
    const size_t P = packedCalc(), M = dimM(), N = dimN(), K = dimK();
    const size_t e = elem();
    const bool realloc = !A_.d || M != allocM_ || N != allocN_ || K != allocK_ || P != allocP_ ||
                         generalizedMatmul() != allocGemm_;
    if (realloc) {
        if (!A_.ensure(P * M * K * e, true) || !B_.ensure(P * K * N * e, true) || !C_.ensure(P * M * N * e, true))
            return false;
        if (!Cin_.ensure(P * M * N * e, true)) return false;
        allocM_ = M, allocN_ = N, allocK_ = K, allocP_ = P, allocGemm_ = generalizedMatmul();
        // test pattern A = B = 1, C = 0 (KernelMatmulBuffer.hpp:88-92)
        if (e == 4) {
            fillconst<float>(A_.h, P * M * K, 1.0f);
            fillconst<float>(B_.h, P * K * N, 1.0f);
            fillconst<float>(Cin_.h, P * M * N, 0.0f);
        } else {
            fillconst<double>(A_.h, P * M * K, 1.0);
            fillconst<double>(B_.h, P * K * N, 1.0);
            fillconst<double>(Cin_.h, P * M * N, 0.0);
        }
        syncInput = true;
    }
    alpha_ = beta_ = 1;
    if (paranoid_) {
        // same draw order as the reference: alpha, beta, A, B, C
        // (KernelMatmulBuffer.hpp:104-116)
        if (generalizedMatmul()) {
            alpha_ = e == 4 ? (double)posrand<float>() : posrand<double>();
            beta_ = e == 4 ? (double)posrand<float>() : posrand<double>();
        }
        if (e == 4) {
            fillrand<float>(A_.h, P * M * K);
            fillrand<float>(B_.h, P * K * N);
            if (generalizedMatmul()) fillrand<float>(Cin_.h, P * M * N);
        } else {
            fillrand<double>(A_.h, P * M * K);
            fillrand<double>(B_.h, P * K * N);
            if (generalizedMatmul()) fillrand<double>(Cin_.h, P * M * N);
        }
        syncInput = true;
    }
    cudaStream_t s = 0;
    if (syncInput && (!A_.upload(s) || !B_.upload(s))) return false;
    // C starts from its initial contents (cleared, or random for GEMM)
    if (cudaMemcpyAsync(C_.d, Cin_.h, C_.bytes, cudaMemcpyHostToDevice, s) != cudaSuccess) return false;
    if (paranoid_ && !is_tc(variant_)) {
        if (!Cref_.ensure(C_.bytes, true)) return false;
        if (cudaMemcpyAsync(Cin_.d, Cin_.h, C_.bytes, cudaMemcpyHostToDevice, s) != cudaSuccess) return false;
        int rc = (e == 4) ? ref_matmul<float>((const float *)A_.d, (const float *)B_.d, (const float *)Cin_.d,
                                              (float *)Cref_.d, P, M, N, K, transposeA(), transposeB(),
                                              generalizedMatmul(), (float)alpha_, (float)beta_, s, paranoid_fused_)
                          : ref_matmul<double>((const double *)A_.d, (const double *)B_.d, (const double *)Cin_.d,
                                               (double *)Cref_.d, P, M, N, K, transposeA(), transposeB(),
                                               generalizedMatmul(), alpha_, beta_, s, paranoid_fused_);
        if (rc || !Cref_.download(s)) return false;
    }
    return sync(s);
}

bool KernelMatmul::enqueue(cudaStream_t stream) {
    const gatlas_matmul_desc d = matmul_desc_of(*this, variant_, vl_, alpha_, beta_);
    const int rc = scalar_ == Scalar::Float
                       ? gatlas_matmul_f32(&d, (const float *)A_.d, (const float *)B_.d, (float *)C_.d, nullptr, 0, stream)
                       : gatlas_matmul_f64(&d, (const double *)A_.d, (const double *)B_.d, (double *)C_.d, nullptr, 0,
                                           stream);
    if (rc != GATLAS_OK) {
        char buf[512];
        gatlas_last_error(buf, sizeof(buf));
        std::cerr << "error: " << buf << std::endl;
        return false;
    }
    return true;
}

bool KernelMatmul::syncOutput() { return C_.download(0) && sync(0); }

bool KernelMatmul::checkOutput(bool printOutput) {
    const size_t len = packedCalc() * dimM() * dimN();
    if (printOutput) {
        if (elem() == 4) print_array<float>(C_.h, dimN(), packedCalc() * dimM());
        else print_array<double>(C_.h, dimN(), packedCalc() * dimM());
    }
    if (!paranoid_) {
        // A = B = 1 (and alpha = beta = 1 on a cleared C): every element is K
        return elem() == 4 ? check_array<float>(C_.h, len, (float)dimK()) : check_array<double>(C_.h, len, (double)dimK());
    }
    if (!is_tc(variant_)) {
        const long double diff = elem() == 4 ? absdiff<float>(C_.h, Cref_.h, len) : absdiff<double>(C_.h, Cref_.h, len);
        absdiff_ = (double)diff;
        std::cerr << "absdiff: " << absdiff_ << "\t";
        return diff < static_cast<double>(1) / len;
    }
    // tensor-core engines: normwise error against the FP64 result on the device
    if (elem() != 4) return false;
    if (generalizedMatmul() && !Cin_.upload(0)) return false;
    double worst = 0;
    for (size_t p = 0; p < packedCalc(); ++p) {
        gatlas_matmul_desc d = matmul_desc_of(*this, variant_, vl_, alpha_, beta_);
        d.batch = 1;
        Geometry g;
        if (!resolve_geometry(&d, &g)) return false;
        double out[4];
        const size_t a_off = p * dimM() * dimK(), b_off = p * dimK() * dimN(), c_off = p * dimM() * dimN();
        if (matmul_residual(g, alpha_, beta_, generalizedMatmul(), (const float *)A_.d + a_off,
                            (const float *)B_.d + b_off, (const float *)Cin_.d + c_off, (const float *)C_.d + c_off,
                            out, 0) != GATLAS_OK)
            return false;
        const double err = out[1] > 0 ? out[0] / out[1] : out[0];
        if (err > worst) worst = err;
    }
    absdiff_ = worst;
    std::cerr << "normwise: " << worst << "\t";
    return worst <= tc_budget(variant_);
}

std::ostream &KernelMatmul::print(std::ostream &os) const {
    // The reference prints generated OpenCL C (KernelMatmulBuffer.hpp:174-342);
    // here the kernel is compiled CUDA and print() describes the instance.
    os << "// " << kernelName() << "  M=" << dimM() << " N=" << dimN() << " K=" << dimK()
       << " transposeA=" << transposeA() << " transposeB=" << transposeB()
       << " GEMM=" << generalizedMatmul() << " packed=" << packedCalc() << "\n";
    if (variant_ == Variant::TcFp8) {
        os << "// quant_fp8_kernel: E4M3 codes with one power-of-two FP32 scale per 128x128 block\n"
           << "// fp8_plan_kernel: per 128x256 tile, runs of up to " << (extraParam() ? extraParam() : 4)
           << " equally scaled 128-deep blocks\n"
           << "// tcgen05 kernel tc_gemm_persistent_kernel<tcfp8>: one CTA per SM over 128x256 output tiles, TMA "
           << "128B-swizzled E4M3 tiles (BK=128), tcgen05.mma kind::f8f6f4 M=128 N=256 K=32, each run promoted "
           << "scaled into FP32 registers, C stored through TMA\n";
    } else if (is_tc(variant_)) {
        const bool split6 = variant_ == Variant::TcSplit6, bf16 = variant_ == Variant::TcBf16;
        os << "// tcgen05 kernel tc_gemm_persistent_kernel<" << variant_name(variant_)
           << ">: one CTA per SM over 128x256 output tiles" << (bf16 ? "" : " (CTA pairs over 256x256 tiles when M > 128)")
           << ", TMA " << (split6 ? "64B-swizzled BF16 piece tiles (BK=32)" : "128B-swizzled BF16 piece tiles (BK=64)")
           << ", tcgen05.mma kind::f16 N=256 K=16, FP32 accumulation in TMEM ";
        if (bf16 && !extraParam())
            os << "over all of K (M > 128: tc_gemm_wide_kernel, 256x256 tiles as two M=128 accumulators)";
        else
            os << "promoted every " << (extraParam() ? extraParam() : 4) << " K-slices";
        os << ", C stored through TMA\n";
    } else {
        const size_t bm = groupHeight() * blockHeight(), bn = groupWidth() * blockWidth();
        const bool img = variant_ == Variant::Image;
        os << "// " << (img ? "gemm_image_kernel" : "gemm_simt_kernel") << "<"
           << scalar_name(scalar_) << ", TA=" << transposeA() << ", TB=" << transposeB() << ", GH=" << groupHeight()
           << ", GW=" << groupWidth() << ", BH=" << blockHeight() << ", BW=" << blockWidth();
        if (img)
            os << ", BK=" << (scalar_ == Scalar::Double ? 16 : 32)
               << ">: operand tiles by TMA tensor maps through a 2-stage mbarrier ring\n";
        else
            os << ", VL=" << vl_ << ", BK=8>\n";
        os
           << "// thread block " << groupHeight() << "x" << groupWidth() << ", CTA tile " << bm << "x" << bn
           << ", per-thread micro-tile " << blockHeight() << "x" << blockWidth()
           << ", grid (" << (dimN() + bn - 1) / bn << ", " << (dimM() + bm - 1) / bm << ", " << packedCalc() << ")\n"
           << "// extra parameter " << extraParam() << " = (";
        const std::vector<size_t> x = extraParamDetail();
        for (size_t i = 0; i < x.size(); ++i) os << (i ? " " : "") << x[i];
        os << ") [inlineMNK, loopOrder" << (variant_ == Variant::Image ? ", globalID" : "")
           << "]: recorded; every order accumulates k = 0..K-1 in sequence\n";
        os << "\n" << jit::simt_source(jit_point());
    }
    return os;
}

size_t KernelMatmul::numberBytes() const {
    return packedCalc() * elem() * (dimM() * dimK() + dimK() * dimN() + (generalizedMatmul() ? 2 : 1) * dimM() * dimN());
}

// ---------------------------------------------------------------------------
// matvec
// ---------------------------------------------------------------------------
KernelMatvec::KernelMatvec(Scalar s, Variant v, size_t vectorLength)
    : MatvecParams(v), scalar_(s), variant_(v), vl_(vectorLength) {}

std::string KernelMatvec::kernelName() const {
    std::stringstream ss;
    ss << "matvec" << variant_name(variant_) << scalar_name(scalar_) << vl_;
    return ss.str();
}

void KernelMatvec::setParams(const std::vector<size_t> &p) { MatvecParams::setParams(p); }

static gatlas_matvec_desc matvec_desc_of(const MatvecParams &p, Variant v, double alpha, double beta) {
    gatlas_matvec_desc d;
    std::memset(&d, 0, sizeof(d));
    d.engine = engine_of(v);
    d.gemv = p.generalizedMatvec();
    d.trans_a = p.transposeA();
    d.m = p.dimM();
    d.n = p.dimN();
    d.batch = p.packedCalc();
    d.alpha = alpha;
    d.beta = beta;
    return d;
}

bool KernelMatvec::build() {
    if (!validParams()) {
        std::cerr << "error: invalid parameters" << std::endl;
        return false;
    }
    if (variant_ != Variant::Buffer && variant_ != Variant::Image) return false;
    return true;
}

bool KernelMatvec::setArgs(bool syncInput) {
    const size_t P = packedCalc(), M = dimM(), N = dimN(), e = elem();
    if (!A_.d || M != allocM_ || N != allocN_ || P != allocP_) {
        if (!A_.ensure(P * M * N * e, true) || !b_.ensure(P * N * e, true) || !c_.ensure(P * M * e, true) ||
            !cin_.ensure(P * M * e, true))
            return false;
        allocM_ = M, allocN_ = N, allocP_ = P;
        if (e == 4) {
            fillconst<float>(A_.h, P * M * N, 1.0f);
            fillconst<float>(b_.h, P * N, 1.0f);
            fillconst<float>(cin_.h, P * M, 0.0f);
        } else {
            fillconst<double>(A_.h, P * M * N, 1.0);
            fillconst<double>(b_.h, P * N, 1.0);
            fillconst<double>(cin_.h, P * M, 0.0);
        }
        syncInput = true;
    }
    alpha_ = beta_ = 1;
    if (paranoid_) {
        // KernelMatvecBuffer.hpp:102-113: alpha, beta, A, b, c
        if (generalizedMatvec()) {
            alpha_ = e == 4 ? (double)posrand<float>() : posrand<double>();
            beta_ = e == 4 ? (double)posrand<float>() : posrand<double>();
        }
        if (e == 4) {
            fillrand<float>(A_.h, P * M * N);
            fillrand<float>(b_.h, P * N);
            if (generalizedMatvec()) fillrand<float>(cin_.h, P * M);
        } else {
            fillrand<double>(A_.h, P * M * N);
            fillrand<double>(b_.h, P * N);
            if (generalizedMatvec()) fillrand<double>(cin_.h, P * M);
        }
        syncInput = true;
    }
    if (syncInput && (!A_.upload(0) || !b_.upload(0))) return false;
    if (cudaMemcpyAsync(c_.d, cin_.h, c_.bytes, cudaMemcpyHostToDevice, 0) != cudaSuccess) return false;
    if (paranoid_) {
        if (!cref_.ensure(c_.bytes, true)) return false;
        if (!cin_.upload(0)) return false;
        int rc = (e == 4) ? ref_matvec<float>((const float *)A_.d, (const float *)b_.d, (const float *)cin_.d,
                                              (float *)cref_.d, P, M, N, transposeA(), generalizedMatvec(),
                                              (float)alpha_, (float)beta_, 0, paranoid_fused_)
                          : ref_matvec<double>((const double *)A_.d, (const double *)b_.d, (const double *)cin_.d,
                                               (double *)cref_.d, P, M, N, transposeA(), generalizedMatvec(), alpha_,
                                               beta_, 0, paranoid_fused_);
        if (rc || !cref_.download(0)) return false;
    }
    return sync(0);
}

bool KernelMatvec::enqueue(cudaStream_t stream) {
    const gatlas_matvec_desc d = matvec_desc_of(*this, variant_, alpha_, beta_);
    const int rc = scalar_ == Scalar::Float
                       ? gatlas_matvec_f32(&d, (const float *)A_.d, (const float *)b_.d, (float *)c_.d, nullptr, 0, stream)
                       : gatlas_matvec_f64(&d, (const double *)A_.d, (const double *)b_.d, (double *)c_.d, nullptr, 0,
                                           stream);
    if (rc != GATLAS_OK) {
        char buf[512];
        gatlas_last_error(buf, sizeof(buf));
        std::cerr << "error: " << buf << std::endl;
        return false;
    }
    return true;
}

bool KernelMatvec::syncOutput() { return c_.download(0) && sync(0); }

bool KernelMatvec::checkOutput(bool printOutput) {
    const size_t len = packedCalc() * dimM();
    if (printOutput) {
        if (elem() == 4) print_array<float>(c_.h, len, 1);
        else print_array<double>(c_.h, len, 1);
    }
    if (!paranoid_)
        return elem() == 4 ? check_array<float>(c_.h, len, (float)dimN()) : check_array<double>(c_.h, len, (double)dimN());
    // The reduction order differs from the sequential chain, so the check is
    // normwise against the sequential reference: within 4*N*u.
    long double num = 0, den = 0;
    for (size_t i = 0; i < len; ++i) {
        const long double a = elem() == 4 ? (long double)((const float *)c_.h)[i] : (long double)((const double *)c_.h)[i];
        const long double r = elem() == 4 ? (long double)((const float *)cref_.h)[i] : (long double)((const double *)cref_.h)[i];
        num += (a - r) * (a - r);
        den += r * r;
    }
    err_ = den > 0 ? (double)sqrtl(num / den) : (double)sqrtl(num);
    std::cerr << "normwise: " << err_ << "\t";
    const double u = elem() == 4 ? std::ldexp(1.0, -24) : std::ldexp(1.0, -53);
    return err_ <= 4.0 * (double)dimN() * u;
}

std::ostream &KernelMatvec::print(std::ostream &os) const {
    os << "// " << kernelName() << "  M=" << dimM() << " N=" << dimN() << " transposeA=" << transposeA()
       << " GEMV=" << generalizedMatvec() << " packed=" << packedCalc() << "\n"
       << "// " << (transposeA() ? "gemv_cols_kernel: CTA per 32x16-byte column block and row segment, "
                                   "cross-warp then cross-segment fixed-order reduction"
                                 : "gemv_rows_kernel: warp per 2 rows, 4 x 16-byte loads per row in flight, "
                                   "butterfly shuffle reduction")
       << "\n// work group " << groupSize() << ", block height " << blockHeight()
       << ": reference NDRange recorded; the CUDA grid is sized to the SM count\n";
    return os;
}

size_t KernelMatvec::numberBytes() const {
    return packedCalc() * elem() * (dimM() * dimN() + dimN() + (generalizedMatvec() ? 2 : 1) * dimM());
}

// ---------------------------------------------------------------------------
// saxpy
// ---------------------------------------------------------------------------
KernelSaxpy::KernelSaxpy(Scalar s, Variant v, size_t vectorLength)
    : SaxpyParams(v), scalar_(s), variant_(v), vl_(vectorLength) {}

std::string KernelSaxpy::kernelName() const {
    std::stringstream ss;
    ss << "saxpy" << variant_name(variant_) << scalar_name(scalar_) << vl_;
    return ss.str();
}

void KernelSaxpy::setParams(const std::vector<size_t> &p) { SaxpyParams::setParams(p); }

bool KernelSaxpy::build() {
    if (!validParams()) {
        std::cerr << "error: invalid parameters" << std::endl;
        return false;
    }
    return variant_ == Variant::Buffer || variant_ == Variant::Image;
}

bool KernelSaxpy::setArgs(bool syncInput) {
    const size_t n = length(), e = elem();
    if (!x_.d || n != allocLen_) {
        if (!x_.ensure(n * e, true) || !y_.ensure(n * e, true) || !z_.ensure(n * e, true)) return false;
        allocLen_ = n;
        if (e == 4) {
            fillconst<float>(x_.h, n, 1.0f);
            fillconst<float>(y_.h, n, 1.0f);
        } else {
            fillconst<double>(x_.h, n, 1.0);
            fillconst<double>(y_.h, n, 1.0);
        }
        syncInput = true;
    }
    alpha_ = 1;
    if (paranoid_) {
        // KernelSaxpyBuffer.hpp:103-115: alpha, X, Y
        alpha_ = e == 4 ? (double)posrand<float>() : posrand<double>();
        if (e == 4) {
            fillrand<float>(x_.h, n);
            fillrand<float>(y_.h, n);
        } else {
            fillrand<double>(x_.h, n);
            fillrand<double>(y_.h, n);
        }
        syncInput = true;
    }
    if (syncInput && (!x_.upload(0) || !y_.upload(0))) return false;
    if (cudaMemsetAsync(z_.d, 0, z_.bytes, 0) != cudaSuccess) return false;
    if (paranoid_) {
        if (!zref_.ensure(z_.bytes, true)) return false;
        int rc = (e == 4) ? ref_saxpy<float>((const float *)x_.d, (const float *)y_.d, (float *)zref_.d, n,
                                             (float)alpha_, 0, paranoid_fused_)
                          : ref_saxpy<double>((const double *)x_.d, (const double *)y_.d, (double *)zref_.d, n, alpha_, 0,
                                              paranoid_fused_);
        if (rc || !zref_.download(0)) return false;
    }
    return sync(0);
}

bool KernelSaxpy::enqueue(cudaStream_t stream) {
    const int eng = engine_of(variant_);
    const int rc = scalar_ == Scalar::Float
                       ? gatlas_saxpy_f32(eng, length(), (float)alpha_, (const float *)x_.d, (const float *)y_.d,
                                          (float *)z_.d, stream)
                       : gatlas_saxpy_f64(eng, length(), alpha_, (const double *)x_.d, (const double *)y_.d,
                                          (double *)z_.d, stream);
    if (rc != GATLAS_OK) {
        char buf[512];
        gatlas_last_error(buf, sizeof(buf));
        std::cerr << "error: " << buf << std::endl;
        return false;
    }
    return true;
}

bool KernelSaxpy::syncOutput() { return z_.download(0) && sync(0); }

bool KernelSaxpy::checkOutput(bool printOutput) {
    const size_t n = length();
    if (printOutput) {
        if (elem() == 4) print_array<float>(z_.h, n, 1);
        else print_array<double>(z_.h, n, 1);
    }
    if (!paranoid_)  // 1 * 1 + 1 (KernelSaxpyBuffer.hpp:80)
        return elem() == 4 ? check_array<float>(z_.h, n, 2.0f) : check_array<double>(z_.h, n, 2.0);
    const long double diff = elem() == 4 ? absdiff<float>(z_.h, zref_.h, n) : absdiff<double>(z_.h, zref_.h, n);
    absdiff_ = (double)diff;
    std::cerr << "absdiff: " << absdiff_ << "\t";
    return diff < static_cast<double>(1) / n;
}

std::ostream &KernelSaxpy::print(std::ostream &os) const {
    os << "// " << kernelName() << "  M=" << dimM() << " N=" << dimN() << " packed=" << packedCalc() << "\n"
       << "// " << (variant_ == Variant::Image ? "saxpy_bulk_kernel: persistent CTAs, 16 KiB cp.async.bulk chunks, "
                                                 "4-stage mbarrier ring, bulk stores"
                                               : "saxpy_vec_kernel: grid-stride 16-byte vectors, 4 per stream in flight")
       << ", z = fma(alpha, x, y)\n// work group " << groupHeight() << "x" << groupWidth() << ", blocking "
       << blockHeight() << "x" << blockWidth() << ": reference NDRange recorded\n";
    return os;
}

size_t KernelSaxpy::numberBytes() const { return 3 * length() * elem(); }

// ---------------------------------------------------------------------------
// factory
// ---------------------------------------------------------------------------
bool parse_type(const std::string &t, Scalar *s, Variant *v, size_t *vl) {
    struct Row {
        const char *name;
        Scalar s;
        Variant v;
        size_t vl;
    };
    static const Row rows[] = {
        {"float1", Scalar::Float, Variant::Buffer, 1},   {"float2", Scalar::Float, Variant::Buffer, 2},
        {"float4", Scalar::Float, Variant::Buffer, 4},   {"double1", Scalar::Double, Variant::Buffer, 1},
        {"double2", Scalar::Double, Variant::Buffer, 2}, {"double4", Scalar::Double, Variant::Buffer, 4},
        {"floatimg", Scalar::Float, Variant::Image, 4},  {"doubleimg", Scalar::Double, Variant::Image, 2},
        {"tcbf16", Scalar::Float, Variant::TcBf16, 4},   {"split3", Scalar::Float, Variant::TcSplit3, 4},
        {"split6", Scalar::Float, Variant::TcSplit6, 4},
        {"fp8", Scalar::Float, Variant::TcFp8, 4},
    };
    for (const Row &r : rows)
        if (t == r.name) {
            *s = r.s;
            *v = r.v;
            *vl = r.vl;
            return true;
        }
    return false;
}

KernelInterface *make_kernel(const std::string &op, const std::string &type) {
    Scalar s;
    Variant v;
    size_t vl;
    if (!parse_type(type, &s, &v, &vl)) return nullptr;
    if (op == "matmul") return new KernelMatmul(s, v, vl);
    if (is_tc(v)) return nullptr;
    if (op == "matvec") return new KernelMatvec(s, v, vl);
    if (op == "saxpy") return new KernelSaxpy(s, v, vl);
    return nullptr;
}

}  // namespace host
}  // namespace gatlas

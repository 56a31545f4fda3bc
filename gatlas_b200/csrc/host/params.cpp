// Parameter-space rules; see params.hpp for the reference citations.
#include "params.hpp"

namespace gatlas {
namespace host {

std::vector<size_t> ExtraParameter::detail() const {
    // KernelBaseMatmul.cpp:160-169: digit i = (value / prod(variations[0..i-1])) % variations[i]
    std::vector<size_t> d;
    size_t shift = 1;
    for (size_t i = 0; i < variations_.size(); ++i) {
        if (i > 0) shift *= variations_[i - 1];
        d.push_back((value_ / shift) % variations_[i]);
    }
    return d;
}

const char *scalar_name(Scalar s) { return s == Scalar::Float ? "float" : "double"; }

const char *variant_name(Variant v) {
    switch (v) {
        case Variant::Buffer: return "buffer";
        case Variant::Image: return "image";
        case Variant::TcBf16: return "tcbf16";
        case Variant::TcSplit3: return "tcsplit3";
        case Variant::TcSplit6: return "tcsplit6";
        case Variant::TcFp8: return "tcfp8";
    }
    return "?";
}

// Observers per family: buffer kernels inline the dimensions (2) and, for
// matmul, pick one of 6 inner-product loop orders; image kernels add the
// global/group ID choice (2).  KernelMatmulBuffer.hpp:27-29,
// KernelMatmulImage.hpp:27-30, KernelMatvec*.hpp:27-29, KernelSaxpy*.hpp:26-29.
// The tensor-core variants reuse the buffer layout of the extra parameter.
static std::vector<size_t> matmul_variations(Variant v) {
    if (v == Variant::Image) return {2, 6, 2};
    return {2, 6};
}
static std::vector<size_t> mv_variations(Variant v) {
    if (v == Variant::Image) return {2, 2};
    return {2};
}

// ---------------------------------------------------------------------------
// matmul
// ---------------------------------------------------------------------------
MatmulParams::MatmulParams(Variant v) : extra_(matmul_variations(v)) {}

bool MatmulParams::validParams() const {
    // KernelBaseMatmul.cpp:263-291 with VECTOR_LENGTH = blockWidth()
    const size_t VL = blockWidth();
    if (VL == 0 || gh_ == 0 || gw_ == 0 || bh_ == 0) return false;
    return packed_ > 0 &&
           M_ % VL == 0 && N_ % VL == 0 && K_ % VL == 0 &&
           M_ % (gh_ * bh_) == 0 && N_ % (gw_ * bw_) == 0 && K_ % (gh_ * VL) == 0 &&
           gh_ * bh_ <= M_ && gw_ * bw_ <= N_ && gh_ * VL <= K_ &&
           (tA_ ? (bh_ % VL == 0) : true) &&
           extraParam() < totalVariations();
}

bool MatmulParams::getParams(std::vector<size_t> &p) const {
    if (!validParams()) return false;
    // KernelBaseMatmul.cpp:293-325
    p = {packed_, (size_t)gemm_, M_, N_, K_, (size_t)tA_, (size_t)tB_, gh_, gw_, bh_, bw_, extraParam()};
    return true;
}

void MatmulParams::setParams(const std::vector<size_t> &p) {
    // KernelBaseMatmul.cpp:327-362
    if (p.size() < 12) return;
    setPackedCalc(p[0]);
    setGeneralizedMatmul(p[1] != 0);
    setMatrixDimensions(p[2], p[3], p[4]);
    setDataLayout(p[5] != 0, p[6] != 0);
    setWorkGroup(p[7], p[8]);
    setInnerBlocking(p[9], p[10]);
    setExtraParameter(p[11]);
}

std::vector<size_t> MatmulParams::globalWorkItems() const {
    return {bw_ ? N_ / bw_ : 0, bh_ ? M_ / bh_ : 0};  // KernelBaseMatmul.cpp:364-369
}

std::vector<size_t> MatmulParams::localWorkItems() const { return {gw_, gh_}; }

size_t MatmulParams::numberFlops() const {
    // KernelBaseMatmul.cpp:378-383
    if (gemm_) return packed_ * 2 * M_ * N_ * (K_ + 1);
    return packed_ * M_ * N_ * (2 * K_ - 1);
}

// ---------------------------------------------------------------------------
// matvec
// ---------------------------------------------------------------------------
MatvecParams::MatvecParams(Variant v) : extra_(mv_variations(v)) {}

bool MatvecParams::validParams() const {
    // KernelBaseMatvec.cpp:236-257
    if (vl_ == 0 || g_ == 0 || bh_ == 0) return false;
    return packed_ > 0 && M_ % vl_ == 0 && N_ % vl_ == 0 && M_ % (g_ * bh_) == 0 &&
           N_ % (g_ * vl_) == 0 && g_ * bh_ <= M_ && g_ * vl_ <= N_ && bh_ % vl_ == 0 &&
           extraParam() < totalVariations();
}

bool MatvecParams::getParams(std::vector<size_t> &p) const {
    if (!validParams()) return false;
    // KernelBaseMatvec.cpp:259-288
    p = {packed_, (size_t)gemv_, M_, N_, (size_t)tA_, g_, bh_, vl_, extraParam()};
    return true;
}

void MatvecParams::setParams(const std::vector<size_t> &p) {
    // KernelBaseMatvec.cpp:290-322
    if (p.size() < 9) return;
    setPackedCalc(p[0]);
    setGeneralizedMatvec(p[1] != 0);
    setMatrixDimensions(p[2], p[3]);
    setDataLayout(p[4] != 0);
    setWorkGroup(p[5]);
    setInnerBlocking(p[6], p[7]);
    setExtraParameter(p[8]);
}

std::vector<size_t> MatvecParams::globalWorkItems() const { return {bh_ ? M_ / bh_ : 0}; }
std::vector<size_t> MatvecParams::localWorkItems() const { return {g_}; }

size_t MatvecParams::numberFlops() const {
    // KernelBaseMatvec.cpp:336-341
    if (gemv_) return packed_ * 2 * M_ * (N_ + 1);
    return packed_ * M_ * (2 * N_ - 1);
}

// ---------------------------------------------------------------------------
// saxpy
// ---------------------------------------------------------------------------
SaxpyParams::SaxpyParams(Variant v) : extra_(mv_variations(v)) {}

bool SaxpyParams::validParams() const {
    // KernelBaseSaxpy.cpp:210-231
    if (vl_ == 0 || gh_ == 0 || bh_ == 0) return false;
    return packed_ > 0 && M_ % vl_ == 0 && N_ % vl_ == 0 && M_ % (gh_ * bh_) == 0 &&
           ((gw_ && bw_) ? N_ % (gw_ * bw_) == 0 : true) && gh_ * bh_ <= M_ && gw_ * bw_ <= N_ &&
           bw_ % vl_ == 0 && extraParam() < totalVariations();
}

bool SaxpyParams::getParams(std::vector<size_t> &p) const {
    if (!validParams()) return false;
    // KernelBaseSaxpy.cpp:233-258
    p = {packed_, M_, N_, gh_, gw_, bh_, bw_, vl_, extraParam()};
    return true;
}

void SaxpyParams::setParams(const std::vector<size_t> &p) {
    // KernelBaseSaxpy.cpp:260-287
    if (p.size() < 9) return;
    setPackedCalc(p[0]);
    setSaxpyDimensions(p[1], p[2]);
    setWorkGroup(p[3], p[4]);
    setInnerBlocking(p[5], p[6]);
    setVectorLength(p[7]);
    setExtraParameter(p[8]);
}

std::vector<size_t> SaxpyParams::globalWorkItems() const {
    // KernelBaseSaxpy.cpp:289-294
    std::vector<size_t> d = {bh_ ? M_ / bh_ : 0};
    if (bw_) d.push_back(N_ / bw_);
    return d;
}

std::vector<size_t> SaxpyParams::localWorkItems() const {
    std::vector<size_t> d = {gh_};
    if (gw_) d.push_back(gw_);
    return d;
}

size_t SaxpyParams::numberFlops() const { return packed_ * 2 * M_ * N_; }  // KernelBaseSaxpy.cpp:303-305

}  // namespace host
}  // namespace gatlas

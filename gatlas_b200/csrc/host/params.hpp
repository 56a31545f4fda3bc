// Parameter spaces of the three kernel families, with the reference's rules.
//
// Reference: KernelBaseMatmul (KernelBaseMatmul.hpp:34-429, KernelBaseMatmul.cpp:24-383),
// KernelBaseMatvec (KernelBaseMatvec.cpp:24-341), KernelBaseSaxpy
// (KernelBaseSaxpy.cpp:24-305).  Parameter vectors, their order, validity,
// NDRange, flop counts and the mixed-radix extra parameter are kept as the
// reference defines them, because journal keys and CLI output depend on them.
// One deliberate difference: a zero work group or block size, which divides by
// zero (a trap) in the reference's validParams, is invalid here.
#pragma once

#include <stddef.h>

#include <string>
#include <vector>

namespace gatlas {
namespace host {

// MatmulExtraParameter / observers (KernelBaseMatmul.cpp:135-175): the extra
// parameter is a mixed-radix number whose digits are the observers' values.
class ExtraParameter {
  public:
    explicit ExtraParameter(std::vector<size_t> variations) : variations_(std::move(variations)) {}
    void set(size_t value) { value_ = value; }
    size_t value() const { return value_; }
    size_t total() const {
        size_t t = 1;
        for (size_t v : variations_) t *= v;
        return t;
    }
    std::vector<size_t> detail() const;

  private:
    std::vector<size_t> variations_;
    size_t value_ = 0;
};

enum class Scalar { Float, Double };
enum class Variant { Buffer, Image, TcBf16, TcSplit3, TcSplit6, TcFp8 };

const char *scalar_name(Scalar s);
const char *variant_name(Variant v);

// KernelBaseMatmul
class MatmulParams {
  public:
    explicit MatmulParams(Variant v);
    // setters (KernelBaseMatmul.hpp:288-301)
    void setPackedCalc(size_t n) { packed_ = n; }
    void setGeneralizedMatmul(bool g) { gemm_ = g; }
    void setMatrixDimensions(size_t M, size_t N, size_t K) { M_ = M; N_ = N; K_ = K; }
    void setDataLayout(bool tA, bool tB) { tA_ = tA; tB_ = tB; }
    void setWorkGroup(size_t h, size_t w) { gh_ = h; gw_ = w; }
    void setWorkGroup(size_t s) { gh_ = gw_ = s; }
    void setInnerBlocking(size_t h, size_t w) { bh_ = h; bw_ = w; }
    void setExtraParameter(size_t x) { extra_.set(x); }
    // accessors
    size_t packedCalc() const { return packed_; }
    bool generalizedMatmul() const { return gemm_; }
    size_t dimM() const { return M_; }
    size_t dimN() const { return N_; }
    size_t dimK() const { return K_; }
    bool transposeA() const { return tA_; }
    bool transposeB() const { return tB_; }
    size_t groupHeight() const { return gh_; }
    size_t groupWidth() const { return gw_; }
    size_t groupSize() const { return gh_ == gw_ ? gw_ : 0; }
    size_t blockHeight() const { return bh_; }
    size_t blockWidth() const { return bw_; }
    size_t extraParam() const { return extra_.value(); }
    size_t totalVariations() const { return extra_.total(); }
    std::vector<size_t> extraParamDetail() const { return extra_.detail(); }

    bool validParams() const;
    bool getParams(std::vector<size_t> &params) const;
    void setParams(const std::vector<size_t> &params);
    std::vector<size_t> globalWorkItems() const;
    std::vector<size_t> localWorkItems() const;
    size_t numberFlops() const;

  private:
    size_t packed_ = 1, M_ = 0, N_ = 0, K_ = 0, gh_ = 0, gw_ = 0, bh_ = 0, bw_ = 0;
    bool gemm_ = false, tA_ = false, tB_ = false;
    ExtraParameter extra_;
};

// KernelBaseMatvec
class MatvecParams {
  public:
    explicit MatvecParams(Variant v);
    void setPackedCalc(size_t n) { packed_ = n; }
    void setGeneralizedMatvec(bool g) { gemv_ = g; }
    void setMatrixDimensions(size_t M, size_t N) { M_ = M; N_ = N; }
    void setDataLayout(bool tA) { tA_ = tA; }
    void setWorkGroup(size_t s) { g_ = s; }
    void setInnerBlocking(size_t h, size_t vl) { bh_ = h; vl_ = vl; }
    void setExtraParameter(size_t x) { extra_.set(x); }
    size_t packedCalc() const { return packed_; }
    bool generalizedMatvec() const { return gemv_; }
    size_t dimM() const { return M_; }
    size_t dimN() const { return N_; }
    bool transposeA() const { return tA_; }
    size_t groupSize() const { return g_; }
    size_t blockHeight() const { return bh_; }
    size_t vectorLength() const { return vl_; }
    size_t extraParam() const { return extra_.value(); }
    size_t totalVariations() const { return extra_.total(); }
    std::vector<size_t> extraParamDetail() const { return extra_.detail(); }

    bool validParams() const;
    bool getParams(std::vector<size_t> &params) const;
    void setParams(const std::vector<size_t> &params);
    std::vector<size_t> globalWorkItems() const;
    std::vector<size_t> localWorkItems() const;
    size_t numberFlops() const;

  private:
    size_t packed_ = 1, M_ = 0, N_ = 0, g_ = 0, bh_ = 0, vl_ = 0;
    bool gemv_ = false, tA_ = false;
    ExtraParameter extra_;
};

// KernelBaseSaxpy
class SaxpyParams {
  public:
    explicit SaxpyParams(Variant v);
    void setPackedCalc(size_t n) { packed_ = n; }
    void setSaxpyDimensions(size_t M, size_t N) { M_ = M; N_ = N; }
    void setWorkGroup(size_t h, size_t w = 0) { gh_ = h; gw_ = w; }
    void setInnerBlocking(size_t h, size_t w = 0) { bh_ = h; bw_ = w; }
    void setVectorLength(size_t vl) { vl_ = vl; }
    void setExtraParameter(size_t x) { extra_.set(x); }
    size_t packedCalc() const { return packed_; }
    size_t dimM() const { return M_; }
    size_t dimN() const { return N_; }
    size_t groupHeight() const { return gh_; }
    size_t groupWidth() const { return gw_; }
    size_t blockHeight() const { return bh_; }
    size_t blockWidth() const { return bw_; }
    size_t vectorLength() const { return vl_; }
    size_t extraParam() const { return extra_.value(); }
    size_t totalVariations() const { return extra_.total(); }
    std::vector<size_t> extraParamDetail() const { return extra_.detail(); }

    bool validParams() const;
    bool getParams(std::vector<size_t> &params) const;
    void setParams(const std::vector<size_t> &params);
    std::vector<size_t> globalWorkItems() const;
    std::vector<size_t> localWorkItems() const;
    size_t numberFlops() const;

  private:
    size_t packed_ = 1, M_ = 0, N_ = 0, gh_ = 0, gw_ = 0, bh_ = 0, bw_ = 0, vl_ = 0;
    ExtraParameter extra_;
};

}  // namespace host
}  // namespace gatlas

// The plugin interface and the three kernel families on B200.
//
// Reference: KernelInterface (GatlasBenchmark.hpp:28-58) and its
// implementations KernelMatmul{Buffer,Image}, KernelMatvec{Buffer,Image},
// KernelSaxpy{Buffer,Image}.  The reference's kernel objects own host arrays
// and OpenCL buffers and print OpenCL source; here they own device buffers
// (plus pinned host mirrors for the bus-transfer timings) and launch the
// library's compiled CUDA kernels through the C ABI.  The OpenCL-specific
// arguments (OCLApp&, kernel handle) are gone from the signatures; build()
// and enqueue() take the place of the OpenCL program build and
// clEnqueueNDRangeKernel.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>

#include <ostream>
#include <string>
#include <vector>

#include "../kernels/jit.hpp"
#include "params.hpp"

namespace gatlas {
namespace host {

class KernelInterface {
  public:
    virtual ~KernelInterface() {}
    virtual std::string kernelName() const = 0;
    virtual size_t numberFlops() const = 0;
    virtual void setParams(const std::vector<size_t> &params) = 0;
    virtual bool getParams(std::vector<size_t> &params) const = 0;
    virtual bool validParams() const = 0;
    virtual std::vector<size_t> extraParamDetail() const = 0;
    virtual size_t totalVariations() const = 0;
    // allocate device buffers if needed, fill them (test pattern, or random data
    // plus a device reference when paranoid) and upload when syncInput
    virtual bool setArgs(bool syncInput) = 0;
    virtual bool syncOutput() = 0;
    virtual bool checkOutput(bool printOutput = false) = 0;
    virtual void paranoidCheck() = 0;
    // arithmetic of the paranoid reference: the generated kernels' fused mad
    // chain (true, the default) or the reference's separately rounded host
    // loops (false)
    virtual void paranoidFused(bool fused) = 0;
    // absdiff (normwise error for the tensor-core engines and GEMV) of the
    // last paranoid check
    virtual double lastCheck() const = 0;
    virtual std::vector<size_t> globalWorkItems() const = 0;
    virtual std::vector<size_t> localWorkItems() const = 0;
    virtual std::ostream &print(std::ostream &os) const = 0;
    // select the compiled kernel for the current parameters (false: none)
    virtual bool build() = 0;
    // one launch of the selected kernel on the bound buffers
    virtual bool enqueue(cudaStream_t stream) = 0;
    // bytes the kernel moves (algorithmic), for GB/s reporting
    virtual size_t numberBytes() const = 0;
};

std::ostream &operator<<(std::ostream &os, const KernelInterface &k);

// Device array with a pinned host mirror.
struct DeviceArray {
    void *d = nullptr;
    void *h = nullptr;
    size_t bytes = 0;
    bool ensure(size_t nbytes, bool host_mirror);
    void release();
    bool upload(cudaStream_t s) const;
    bool download(cudaStream_t s) const;
    ~DeviceArray() { release(); }
};

class KernelMatmul : public KernelInterface, public MatmulParams {
  public:
    KernelMatmul(Scalar s, Variant v, size_t vectorLength);
    std::string kernelName() const override;
    size_t numberFlops() const override { return MatmulParams::numberFlops(); }
    void setParams(const std::vector<size_t> &p) override { MatmulParams::setParams(p); }
    bool getParams(std::vector<size_t> &p) const override { return MatmulParams::getParams(p); }
    bool validParams() const override { return MatmulParams::validParams(); }
    std::vector<size_t> extraParamDetail() const override { return MatmulParams::extraParamDetail(); }
    size_t totalVariations() const override { return MatmulParams::totalVariations(); }
    bool setArgs(bool syncInput) override;
    bool syncOutput() override;
    bool checkOutput(bool printOutput) override;
    void paranoidCheck() override { paranoid_ = true; }
    void paranoidFused(bool fused) override { paranoid_fused_ = fused; }
    double lastCheck() const override { return absdiff_; }
    std::vector<size_t> globalWorkItems() const override { return MatmulParams::globalWorkItems(); }
    std::vector<size_t> localWorkItems() const override { return MatmulParams::localWorkItems(); }
    std::ostream &print(std::ostream &os) const override;
    bool build() override;
    bool enqueue(cudaStream_t stream) override;
    size_t numberBytes() const override;

    Scalar scalar() const { return scalar_; }
    Variant variant() const { return variant_; }
    size_t vectorLength() const { return vl_; }
    double lastAbsdiff() const { return absdiff_; }
    // 1: prebuilt kernel, 2: compiled at run time on first use, 0: cannot run
    int supportLevel() const;

  private:
    size_t elem() const { return scalar_ == Scalar::Float ? 4 : 8; }
    jit::Point jit_point() const;
    Scalar scalar_;
    Variant variant_;
    size_t vl_;
    bool paranoid_ = false;
    bool paranoid_fused_ = true;
    double alpha_ = 1, beta_ = 1, absdiff_ = 0;
    size_t allocM_ = 0, allocN_ = 0, allocK_ = 0, allocP_ = 0;
    bool allocGemm_ = false;
    DeviceArray A_, B_, C_, Cin_, Cref_;
};

class KernelMatvec : public KernelInterface, public MatvecParams {
  public:
    KernelMatvec(Scalar s, Variant v, size_t vectorLength);
    std::string kernelName() const override;
    size_t numberFlops() const override { return MatvecParams::numberFlops(); }
    void setParams(const std::vector<size_t> &p) override;
    bool getParams(std::vector<size_t> &p) const override { return MatvecParams::getParams(p); }
    bool validParams() const override { return MatvecParams::validParams(); }
    std::vector<size_t> extraParamDetail() const override { return MatvecParams::extraParamDetail(); }
    size_t totalVariations() const override { return MatvecParams::totalVariations(); }
    bool setArgs(bool syncInput) override;
    bool syncOutput() override;
    bool checkOutput(bool printOutput) override;
    void paranoidCheck() override { paranoid_ = true; }
    void paranoidFused(bool fused) override { paranoid_fused_ = fused; }
    double lastCheck() const override { return err_; }
    std::vector<size_t> globalWorkItems() const override { return MatvecParams::globalWorkItems(); }
    std::vector<size_t> localWorkItems() const override { return MatvecParams::localWorkItems(); }
    std::ostream &print(std::ostream &os) const override;
    bool build() override;
    bool enqueue(cudaStream_t stream) override;
    size_t numberBytes() const override;
    double lastError() const { return err_; }

  private:
    size_t elem() const { return scalar_ == Scalar::Float ? 4 : 8; }
    Scalar scalar_;
    Variant variant_;
    size_t vl_;
    bool paranoid_ = false;
    bool paranoid_fused_ = true;
    double alpha_ = 1, beta_ = 1, err_ = 0;
    size_t allocM_ = 0, allocN_ = 0, allocP_ = 0;
    DeviceArray A_, b_, c_, cin_, cref_;
};

class KernelSaxpy : public KernelInterface, public SaxpyParams {
  public:
    KernelSaxpy(Scalar s, Variant v, size_t vectorLength);
    std::string kernelName() const override;
    size_t numberFlops() const override { return SaxpyParams::numberFlops(); }
    void setParams(const std::vector<size_t> &p) override;
    bool getParams(std::vector<size_t> &p) const override { return SaxpyParams::getParams(p); }
    bool validParams() const override { return SaxpyParams::validParams(); }
    std::vector<size_t> extraParamDetail() const override { return SaxpyParams::extraParamDetail(); }
    size_t totalVariations() const override { return SaxpyParams::totalVariations(); }
    bool setArgs(bool syncInput) override;
    bool syncOutput() override;
    bool checkOutput(bool printOutput) override;
    void paranoidCheck() override { paranoid_ = true; }
    void paranoidFused(bool fused) override { paranoid_fused_ = fused; }
    double lastCheck() const override { return absdiff_; }
    std::vector<size_t> globalWorkItems() const override { return SaxpyParams::globalWorkItems(); }
    std::vector<size_t> localWorkItems() const override { return SaxpyParams::localWorkItems(); }
    std::ostream &print(std::ostream &os) const override;
    bool build() override;
    bool enqueue(cudaStream_t stream) override;
    size_t numberBytes() const override;
    double lastAbsdiff() const { return absdiff_; }

  private:
    size_t elem() const { return scalar_ == Scalar::Float ? 4 : 8; }
    size_t length() const { return packedCalc() * dimM() * dimN(); }
    Scalar scalar_;
    Variant variant_;
    size_t vl_;
    bool paranoid_ = false;
    bool paranoid_fused_ = true;
    double alpha_ = 1, absdiff_ = 0;
    size_t allocLen_ = 0;
    DeviceArray x_, y_, z_, zref_;
};

// Factory from the reference's -T kernel type names (benchMatmul.cpp:141-160),
// extended with the tensor-core types tcbf16, split3, split6 and fp8 (matmul only).
// op: "matmul" | "matvec" | "saxpy".  Returns nullptr for unknown types.
KernelInterface *make_kernel(const std::string &op, const std::string &type);

// Scalar, variant and vector length of a -T type; false if unknown.
bool parse_type(const std::string &type, Scalar *s, Variant *v, size_t *vl);

}  // namespace host
}  // namespace gatlas

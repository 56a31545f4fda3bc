// Run-time compilation of SIMT GEMM parameter points (NVRTC).
//
// The reference builds an OpenCL program for every parameter point it times
// (Bench::rebuildProgram -> clBuildProgram, GatlasBenchmark.cpp:286-301), so
// its whole search space is runnable.  The library prebuilds the common
// points; any other valid point of the reference's space (odd work groups,
// inner blockings up to 12, every layout) is compiled here on first use from
// the same kernel template, for sm_100a, and cached per device for the
// process.  NVRTC is loaded lazily (dlopen), so the library still loads where
// it is absent; the driver entry points come from cudaGetDriverEntryPoint.
#include <cuda.h>
#include <cuda_runtime.h>
#include <dlfcn.h>

#include <map>
#include <mutex>
#include <sstream>
#include <string>
#include <tuple>

#include "../status.hpp"
#include "jit.hpp"

namespace gatlas {
namespace jit {

namespace {

const char kSimtSource[] =
#include "gemm_simt_source.inc"
    ;
const char kImageSource[] =
#include "gemm_image_source.inc"
    ;

// NVRTC entry points (nvrtc.h), resolved with dlsym.
typedef int nvrtcResult;
typedef struct _nvrtcProgram *nvrtcProgram;
struct Nvrtc {
    nvrtcResult (*create)(nvrtcProgram *, const char *, const char *, int, const char *const *, const char *const *);
    nvrtcResult (*add_name)(nvrtcProgram, const char *);
    nvrtcResult (*compile)(nvrtcProgram, int, const char *const *);
    nvrtcResult (*lowered)(nvrtcProgram, const char *, const char **);
    nvrtcResult (*cubin_size)(nvrtcProgram, size_t *);
    nvrtcResult (*cubin)(nvrtcProgram, char *);
    nvrtcResult (*log_size)(nvrtcProgram, size_t *);
    nvrtcResult (*log)(nvrtcProgram, char *);
    nvrtcResult (*destroy)(nvrtcProgram *);
    bool ok = false;
};

struct Driver {
    CUresult (*load)(CUmodule *, const void *) = nullptr;
    CUresult (*get_function)(CUfunction *, CUmodule, const char *) = nullptr;
    CUresult (*launch)(CUfunction, unsigned, unsigned, unsigned, unsigned, unsigned, unsigned, unsigned, CUstream,
                       void **, void **) = nullptr;
    CUresult (*set_attr)(CUfunction, CUfunction_attribute, int) = nullptr;
    bool ok = false;
};

std::once_flag g_once;
Nvrtc g_nvrtc;
Driver g_drv;
std::mutex g_mu;
std::map<std::tuple<int, int, int, int, int, int, int, int, int, int>, CUfunction> g_cache;

template <typename F>
bool sym(void *h, const char *name, F *out) {
    *out = reinterpret_cast<F>(dlsym(h, name));
    return *out != nullptr;
}

template <typename F>
bool drv(const char *name, F *out) {
    void *fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint(name, &fn, cudaEnableDefault, &q) != cudaSuccess || q != cudaDriverEntryPointSuccess)
        return false;
    *out = reinterpret_cast<F>(fn);
    return true;
}

void init() {
    const char *paths[] = {"libnvrtc.so.12", "/usr/local/cuda/lib64/libnvrtc.so.12", "/usr/local/cuda/lib64/libnvrtc.so",
                           "libnvrtc.so"};
    void *h = nullptr;
    for (const char *p : paths)
        if ((h = dlopen(p, RTLD_NOW | RTLD_LOCAL))) break;
    if (h) {
        Nvrtc &n = g_nvrtc;
        n.ok = sym(h, "nvrtcCreateProgram", &n.create) && sym(h, "nvrtcAddNameExpression", &n.add_name) &&
               sym(h, "nvrtcCompileProgram", &n.compile) && sym(h, "nvrtcGetLoweredName", &n.lowered) &&
               sym(h, "nvrtcGetCUBINSize", &n.cubin_size) && sym(h, "nvrtcGetCUBIN", &n.cubin) &&
               sym(h, "nvrtcGetProgramLogSize", &n.log_size) && sym(h, "nvrtcGetProgramLog", &n.log) &&
               sym(h, "nvrtcDestroyProgram", &n.destroy);
    }
}

bool init_driver() {
    if (g_drv.ok) return true;
    g_drv.ok = drv("cuModuleLoadData", &g_drv.load) && drv("cuModuleGetFunction", &g_drv.get_function) &&
               drv("cuLaunchKernel", &g_drv.launch) && drv("cuFuncSetAttribute", &g_drv.set_attr);
    return g_drv.ok;
}

}  // namespace

bool available() {
    std::call_once(g_once, init);
    return g_nvrtc.ok;
}

std::string simt_name(const Point &p) {
    std::stringstream ss;
    const char *T = p.scalar ? "double" : "float";
    if (p.image) {
        ss << "gatlas::img::gemm_image_kernel<" << T << ", " << (p.ta ? "true" : "false") << ", "
           << (p.tb ? "true" : "false") << ", " << p.gh << ", " << p.gw << ", " << p.bh << ", " << p.bw << ">";
    } else {
        ss << "gatlas::simt::gemm_simt_kernel<" << T << ", " << (p.ta ? "true" : "false") << ", "
           << (p.tb ? "true" : "false") << ", " << p.gh << ", " << p.gw << ", " << p.bh << ", " << p.bw << ", "
           << p.vl << ", 8>";
    }
    return ss.str();
}

std::string simt_source(const Point &p) {
    std::stringstream ss;
    const char *T = p.scalar ? "double" : "float";
    ss << (p.image ? kImageSource : kSimtSource) << "\n// instantiation compiled for this point:\ntemplate __global__ void "
       << simt_name(p);
    if (p.image)
        ss << "(const __grid_constant__ gatlas::img::TmapBlob, const __grid_constant__ gatlas::img::TmapBlob, "
              "gatlas::img::ImgArgs<"
           << T << ">);\n";
    else
        ss << "(gatlas::simt::GemmArgs<" << T << ">);\n";
    return ss.str();
}

// Whether the template accepts the point (mirrors the static_asserts and,
// for the image template, the tensor-map alignment rules).
bool point_ok(const Point &p) {
    if (p.gh < 1 || p.gw < 1 || p.bh < 1 || p.bw < 1 || p.gh * p.gw > 1024) return false;
    if (p.bh > 16 || p.bw > 16) return false;
    if (p.image) {
        const int per16 = p.scalar ? 2 : 4;  // elements per 16 bytes
        if (p.ta && (p.gh * p.bh) % per16) return false;
        if (!p.tb && (p.gw * p.bw) % per16) return false;
        if (p.gh * p.bh > 256 || p.gw * p.bw > 256) return false;
        return true;
    }
    if (p.vl != 1 && p.vl != 2 && p.vl != 4) return false;
    if (8 % p.vl != 0) return false;
    if (p.ta && (p.gh * p.bh) % p.vl != 0) return false;
    if (!p.tb && (p.gw * p.bw) % p.vl != 0) return false;
    return true;
}

int simt_function(const Point &p, void **fn) {
    if (!available()) return set_error(GATLAS_ERR_UNSUPPORTED, "jit: NVRTC is not available");
    if (!point_ok(p)) return set_error(GATLAS_ERR_UNSUPPORTED, "jit: the SIMT template does not take this point");
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return set_error(GATLAS_ERR_CUDA, "jit: no current device");
    const auto key = std::make_tuple(dev, p.image, p.scalar, p.ta, p.tb, p.gh, p.gw, p.bh, p.bw, p.image ? 0 : p.vl);
    std::lock_guard<std::mutex> lk(g_mu);
    auto it = g_cache.find(key);
    if (it != g_cache.end()) {
        *fn = it->second;
        return GATLAS_OK;
    }
    if (!init_driver()) return set_error(GATLAS_ERR_CUDA, "jit: driver entry points unavailable");
    cudaFree(nullptr);  // make the runtime's primary context current
    const Nvrtc &n = g_nvrtc;
    nvrtcProgram prog = nullptr;
    if (n.create(&prog, p.image ? kImageSource : kSimtSource, p.image ? "gemm_image.cu" : "gemm_simt.cu", 0, nullptr,
                 nullptr) != 0)
        return set_error(GATLAS_ERR_CUDA, "jit: nvrtcCreateProgram failed");
    const std::string name = simt_name(p);
    n.add_name(prog, name.c_str());
    const char *opts[] = {"--gpu-architecture=sm_100a", "-std=c++17", "-default-device", "-lineinfo"};
    const nvrtcResult rc = n.compile(prog, 4, opts);
    if (rc != 0) {
        size_t ls = 0;
        n.log_size(prog, &ls);
        std::string log(ls, '\0');
        if (ls) n.log(prog, &log[0]);
        n.destroy(&prog);
        return set_error(GATLAS_ERR_UNSUPPORTED, "jit: compile of %s failed: %.300s", name.c_str(), log.c_str());
    }
    const char *lowered = nullptr;
    size_t cubin_size = 0;
    n.lowered(prog, name.c_str(), &lowered);
    n.cubin_size(prog, &cubin_size);
    std::string cubin(cubin_size, '\0');
    n.cubin(prog, &cubin[0]);
    const std::string lowered_name = lowered ? lowered : "";
    n.destroy(&prog);
    CUmodule mod = nullptr;
    CUfunction f = nullptr;
    if (g_drv.load(&mod, cubin.data()) != CUDA_SUCCESS || g_drv.get_function(&f, mod, lowered_name.c_str()) != CUDA_SUCCESS)
        return set_error(GATLAS_ERR_CUDA, "jit: loading the compiled module failed");
    g_cache[key] = f;
    *fn = f;
    return GATLAS_OK;
}

int launch_args(void *fn, unsigned gx, unsigned gy, unsigned gz, unsigned block, unsigned smem, void **args,
                cudaStream_t stream) {
    if (smem > 48 * 1024 &&
        g_drv.set_attr(static_cast<CUfunction>(fn), CU_FUNC_ATTRIBUTE_MAX_DYNAMIC_SHARED_SIZE_BYTES, (int)smem) != CUDA_SUCCESS)
        return set_error(GATLAS_ERR_CUDA, "jit: shared memory attribute");
    CUresult r = g_drv.launch(static_cast<CUfunction>(fn), gx, gy, gz, block, 1, 1, smem, (CUstream)stream, args, nullptr);
    if (r != CUDA_SUCCESS) return set_error(GATLAS_ERR_CUDA, "jit: cuLaunchKernel failed (%d)", (int)r);
    return GATLAS_OK;
}

int launch(void *fn, unsigned gx, unsigned gy, unsigned gz, unsigned block, void *args, cudaStream_t stream) {
    void *params[] = {args};
    CUresult r = g_drv.launch(static_cast<CUfunction>(fn), gx, gy, gz, block, 1, 1, 0, (CUstream)stream, params, nullptr);
    if (r != CUDA_SUCCESS) return set_error(GATLAS_ERR_CUDA, "jit: cuLaunchKernel failed (%d)", (int)r);
    return GATLAS_OK;
}

}  // namespace jit
}  // namespace gatlas

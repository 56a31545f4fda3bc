// print_matmul: validate one matmul parameter point and describe its kernel.
//
// Reference: printMatmul.cpp (options :50-160, print :162-248).  The
// reference streams the generated OpenCL source; here the kernels are
// compiled CUDA and the tool prints the instance that would run (template
// parameters, tile, grid) and whether it is built into the library.
#include <unistd.h>

#include <cstdlib>
#include <iostream>
#include <string>

#include "../../include/gatlas.h"
#include "host/kernel.hpp"

using namespace gatlas::host;
using std::cerr;
using std::cout;
using std::endl;

int main(int argc, char **argv) {
    size_t packed = 1;
    std::string type = "<unspecified>";
    long M = -1, N = -1, K = -1, g = -1, bh = -1, xp = -1;
    bool gemm = false, tA = false, tB = false;
    int opt;
    while ((opt = getopt(argc, argv, "habvGC:T:m:n:k:g:y:x:")) != -1) {
        switch (opt) {
            case 'h':
                cerr << "usage: " << argv[0]
                     << " -T float1|float2|float4|double1|double2|double4|floatimg|doubleimg|tcbf16|split3|split6|fp8"
                        " -n N [-m M -k K] -g groupSize -y blockHeight -x extraParam [-C numKernels] [-G] [-a] [-b]"
                        " [-v] [-h]"
                     << endl;
                exit(1);
            case 'C': packed = (size_t)atoi(optarg); break;
            case 'T': type = optarg; break;
            case 'm': M = atoi(optarg); break;
            case 'n': N = atoi(optarg); break;
            case 'k': K = atoi(optarg); break;
            case 'g': g = atoi(optarg); break;
            case 'y': bh = atoi(optarg); break;
            case 'x': xp = atoi(optarg); break;
            case 'G': gemm = true; break;
            case 'a': tA = true; break;
            case 'b': tB = true; break;
            case 'v': break;
        }
    }
    Scalar s;
    Variant v;
    size_t vl = 1;
    bool rc = true;
    if (!parse_type(type, &s, &v, &vl)) {
        cerr << "error: invalid kernel type of " << type << endl;
        rc = false;
    }
    if (N == -1) {
        cerr << "error: matrix dimension N must be specified" << endl;
        rc = false;
    } else if (M == -1 && K == -1) {
        M = K = N;
    } else if ((M != -1) != (K != -1)) {
        cerr << "error: all matrix dimensions M, N and K must be specified" << endl;
        rc = false;
    }
    const long VL = (long)vl;
    if (rc && (N % VL || M % VL || K % VL)) {
        cerr << "error: matrix dimensions must be multiples of " << VL << endl;
        rc = false;
    }
    if (g == -1) { cerr << "error: must specify work item group size" << endl; rc = false; }
    if (bh == -1) { cerr << "error: must specify inner blocking height" << endl; rc = false; }
    if (xp == -1) { cerr << "error: must specify extra parameter" << endl; rc = false; }
    if (g != -1 && (g < 1 || g > 16)) {
        cerr << "error: work item group size must be a number from 1 to 16 inclusive" << endl;
        rc = false;
    }
    if (tA && bh != -1 && bh % VL) {
        cerr << "error: inner blocking height must be multiple of " << VL << " when matrix A is transposed" << endl;
        rc = false;
    }
    if (bh != -1 && bh < VL) { cerr << "error: invalid inner blocking height" << endl; rc = false; }
    if (!rc) exit(1);
    KernelMatmul k(s, v, vl);
    k.setPackedCalc(packed);
    k.setGeneralizedMatmul(gemm);
    k.setMatrixDimensions((size_t)M, (size_t)N, (size_t)K);
    k.setDataLayout(tA, tB);
    k.setWorkGroup((size_t)g);
    k.setInnerBlocking((size_t)bh, vl);
    k.setExtraParameter((size_t)xp);
    if (!k.validParams()) {
        cerr << "error: invalid parameters (coalescedKernels, M, N, K, groupSize, blockHeight, extraParam): ("
             << packed << ", " << M << ", " << N << ", " << K << ", " << g << ", " << bh << ", " << xp << ")" << endl;
        exit(1);
    }
    cout << k;
    const int level = k.supportLevel();
    cout << "// " << (level == 1 ? "prebuilt in the library" : level == 2 ? "compiled at run time (NVRTC) on first use"
                                                                          : "no kernel for this point")
         << endl;
    return 0;
}

// print_matvec: validate one matvec parameter point and describe its kernel.
// Reference: printMatvec.cpp (options :48-150, print :150-232).
#include <unistd.h>

#include <cstdlib>
#include <iostream>
#include <string>

#include "host/kernel.hpp"

using namespace gatlas::host;
using std::cerr;
using std::cout;
using std::endl;

int main(int argc, char **argv) {
    size_t packed = 1;
    std::string type = "<unspecified>";
    long M = -1, N = -1, g = -1, bh = -1, xp = -1;
    bool gemv = false, tA = false;
    int opt;
    while ((opt = getopt(argc, argv, "havGC:T:m:n:g:y:x:")) != -1) {
        switch (opt) {
            case 'h':
                cerr << "usage: " << argv[0]
                     << " -T float1|float2|float4|double1|double2|double4|floatimg|doubleimg -n N [-m M]"
                        " -g groupSize -y blockHeight -x extraParam [-C numKernels] [-G] [-a] [-v] [-h]"
                     << endl;
                exit(1);
            case 'C': packed = (size_t)atoi(optarg); break;
            case 'T': type = optarg; break;
            case 'm': M = atoi(optarg); break;
            case 'n': N = atoi(optarg); break;
            case 'g': g = atoi(optarg); break;
            case 'y': bh = atoi(optarg); break;
            case 'x': xp = atoi(optarg); break;
            case 'G': gemv = true; break;
            case 'a': tA = true; break;
            case 'v': break;
        }
    }
    Scalar s;
    Variant v;
    size_t vl = 1;
    bool rc = true;
    if (!parse_type(type, &s, &v, &vl) || (v != Variant::Buffer && v != Variant::Image)) {
        cerr << "error: invalid kernel type of " << type << endl;
        rc = false;
    }
    if (N == -1) { cerr << "error: matrix dimension N must be specified" << endl; rc = false; }
    else if (M == -1) M = N;
    if (g == -1 || bh == -1 || xp == -1) {
        cerr << "error: must specify work item group size, inner blocking height and extra parameter" << endl;
        rc = false;
    }
    if (!rc) exit(1);
    KernelMatvec k(s, v, vl);
    k.setPackedCalc(packed);
    k.setGeneralizedMatvec(gemv);
    k.setMatrixDimensions((size_t)M, (size_t)N);
    k.setDataLayout(tA);
    k.setWorkGroup((size_t)g);
    k.setInnerBlocking((size_t)bh, vl);
    k.setExtraParameter((size_t)xp);
    if (!k.validParams()) {
        cerr << "error: invalid parameters (coalescedKernels, M, N, groupSize, blockHeight, extraParam): (" << packed
             << ", " << M << ", " << N << ", " << g << ", " << bh << ", " << xp << ")" << endl;
        exit(1);
    }
    cout << k;
    return 0;
}

// print_saxpy: validate one saxpy parameter point and describe its kernel.
// Reference: printSaxpy.cpp (options :48-150, print :150-225): -G/-Y group
// width/height, -g/-y block width/height.
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
    long M = -1, N = -1, gw = -1, gh = -1, bw = -1, bh = -1, xp = -1;
    int opt;
    while ((opt = getopt(argc, argv, "hvC:T:m:n:G:Y:g:y:x:")) != -1) {
        switch (opt) {
            case 'h':
                cerr << "usage: " << argv[0]
                     << " -T float1|float2|float4|double1|double2|double4|floatimg|doubleimg -m M [-n N]"
                        " -Y groupHeight [-G groupWidth] -y blockHeight [-g blockWidth] -x extraParam"
                        " [-C numKernels] [-v] [-h]"
                     << endl;
                exit(1);
            case 'C': packed = (size_t)atoi(optarg); break;
            case 'T': type = optarg; break;
            case 'm': M = atoi(optarg); break;
            case 'n': N = atoi(optarg); break;
            case 'G': gw = atoi(optarg); break;
            case 'Y': gh = atoi(optarg); break;
            case 'g': bw = atoi(optarg); break;
            case 'y': bh = atoi(optarg); break;
            case 'x': xp = atoi(optarg); break;
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
    if (M == -1) { cerr << "error: matrix dimension M must be specified" << endl; rc = false; }
    if (N == -1) N = (long)vl;
    if (gh == -1 || bh == -1 || xp == -1) {
        cerr << "error: must specify group height, block height and extra parameter" << endl;
        rc = false;
    }
    if (!rc) exit(1);
    KernelSaxpy k(s, v, vl);
    k.setPackedCalc(packed);
    k.setSaxpyDimensions((size_t)M, (size_t)N);
    k.setVectorLength(vl);
    k.setWorkGroup((size_t)gh, gw == -1 ? 0 : (size_t)gw);
    k.setInnerBlocking((size_t)bh, bw == -1 ? 0 : (size_t)bw);
    k.setExtraParameter((size_t)xp);
    if (!k.validParams()) {
        cerr << "error: invalid parameters" << endl;
        exit(1);
    }
    cout << k;
    return 0;
}

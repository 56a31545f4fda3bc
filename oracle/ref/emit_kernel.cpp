// Prints the reference's generated OpenCL C kernel for one parameter point.
//
// TEST INFRASTRUCTURE: a thin driver over the reference's own kernel
// generators (cjang/GATLAS), compiled from its sources by oracle/ref/Makefile.
// It does what the reference's print_matmul / print_matvec / print_saxpy do
// (printMatmul.cpp:162-248, printMatvec.cpp, printSaxpy.cpp), but takes the
// parameter vector in journal order and sets it with the generator's own
// setParams (KernelBaseMatmul.cpp:293-325, KernelBaseMatvec.cpp:259-288,
// KernelBaseSaxpy.cpp:233-258), so any valid point of the parameter space can
// be emitted, not only those the print tools' option checks allow.
//
//   emit_kernel matmul|matvec|saxpy <-T type> p0 p1 ...
//
// The kernel source goes to stdout, followed by one line
//   //@ name=<kernelName> global=<g0,g1> local=<l0,l1>
// with the generator's globalWorkItems() and localWorkItems().  Exit status 1
// for an invalid point.
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <string>
#include <vector>

#include "KernelMatmulBuffer.hpp"
#include "KernelMatmulImage.hpp"
#include "KernelMatvecBuffer.hpp"
#include "KernelMatvecImage.hpp"
#include "KernelSaxpyBuffer.hpp"
#include "KernelSaxpyImage.hpp"

#include "using_namespace"

using namespace std;

template <typename K>
static int emit(K& kernel, const vector<size_t>& params) {
    kernel.setParams(params);
    if (!kernel.validParams()) {
        cerr << "error: invalid parameters" << endl;
        return 1;
    }
    cout << kernel;
    const vector<size_t> g = kernel.globalWorkItems(), l = kernel.localWorkItems();
    cout << "//@ name=" << kernel.kernelName() << " global=";
    for (size_t i = 0; i < g.size(); i++) cout << (i ? "," : "") << g[i];
    cout << " local=";
    for (size_t i = 0; i < l.size(); i++) cout << (i ? "," : "") << l[i];
    cout << endl;
    return 0;
}

#define PICK(FAMILY)                                                                    \
    if (type == "float1") { FAMILY##Buffer<float, 1> k; return emit(k, params); }        \
    if (type == "float2") { FAMILY##Buffer<float, 2> k; return emit(k, params); }        \
    if (type == "float4") { FAMILY##Buffer<float, 4> k; return emit(k, params); }        \
    if (type == "double1") { FAMILY##Buffer<double, 1> k; return emit(k, params); }      \
    if (type == "double2") { FAMILY##Buffer<double, 2> k; return emit(k, params); }      \
    if (type == "double4") { FAMILY##Buffer<double, 4> k; return emit(k, params); }      \
    if (type == "floatimg") { FAMILY##Image<float, 4> k; return emit(k, params); }       \
    if (type == "doubleimg") { FAMILY##Image<double, 2> k; return emit(k, params); }

int main(int argc, char* argv[]) {
    if (argc < 4) {
        cerr << "usage: " << argv[0] << " matmul|matvec|saxpy type p0 p1 ..." << endl;
        return 2;
    }
    const string op = argv[1], type = argv[2];
    vector<size_t> params;
    for (int i = 3; i < argc; i++) params.push_back(strtoul(argv[i], NULL, 10));
    if (op == "matmul") { PICK(KernelMatmul) }
    if (op == "matvec") { PICK(KernelMatvec) }
    if (op == "saxpy") { PICK(KernelSaxpy) }
    cerr << "error: unknown op or type" << endl;
    return 2;
}

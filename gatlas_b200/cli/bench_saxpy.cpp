// bench_saxpy: autotune and time the saxpy kernels on a B200.
//
// Reference: benchSaxpy.cpp (options :59-150, search :158-276, EM :490-600;
// maxBlockHeight 16 and maxGroupSize 256).  Its EM alternates the work group
// with the inner blocking and extra parameter.  -d gpuN selects a CUDA device.
#include <unistd.h>

#include <cstdlib>
#include <iostream>
#include <string>
#include <vector>

#include "../../include/gatlas.h"
#include "host/bench.hpp"
#include "host/kernel.hpp"
#include "host/search.hpp"

using namespace gatlas::host;
using std::cerr;
using std::cout;
using std::endl;
using std::string;
using std::vector;

namespace {

struct Opts {
    string device = "<unspecified>", journal, type = "<unspecified>";
    size_t packed = 1, trials = 1, vl = 1;
    long M = -1, N = -1, topN = -1;
    bool em = false, busTo = false, busFrom = false, paranoid = false, debug = false;
};

constexpr size_t kMaxBlockHeight = 16, kMaxGroupSize = 256;

bool parse(int argc, char **argv, Opts &o) {
    int opt;
    while ((opt = getopt(argc, argv, "hesrpvzd:j:C:T:m:n:t:w:")) != -1) {
        switch (opt) {
            case 'h':
                cerr << "usage: " << argv[0]
                     << " -d gpu|gpuX -j journalFile -T float1|float2|float4|double1|double2|double4|floatimg|doubleimg"
                        " -m M [-n N] [-C numKernels] [-t numberTrials] [-w topN] [-e] [-s] [-r] [-p] [-v] [-z] [-h]"
                     << endl
                     << "***DONE***" << endl;
                exit(1);
            case 'd': o.device = optarg; break;
            case 'j': o.journal = optarg; break;
            case 'C': o.packed = (size_t)atoi(optarg); break;
            case 'T': o.type = optarg; break;
            case 'm': o.M = atoi(optarg); break;
            case 'n': o.N = atoi(optarg); break;
            case 't': o.trials = (size_t)atoi(optarg); break;
            case 'w': o.topN = atoi(optarg); break;
            case 'e': o.em = true; break;
            case 's': o.busTo = true; break;
            case 'r': o.busFrom = true; break;
            case 'p': o.paranoid = true; break;
            case 'v': break;
            case 'z': o.debug = true; break;
        }
    }
    bool rc = true;
    if (o.device.compare(0, 3, "gpu") != 0) { cerr << "error: invalid device " << o.device << endl; rc = false; }
    if (o.journal.empty()) { cerr << "error: journal file must be specified" << endl; rc = false; }
    if (o.packed == 0) { cerr << "error: number of kernels to coalesce must be at least one" << endl; rc = false; }
    Scalar s;
    Variant v;
    if (!parse_type(o.type, &s, &v, &o.vl) || (v != Variant::Buffer && v != Variant::Image)) {
        cerr << "error: invalid kernel type of " << o.type << endl;
        rc = false;
        o.vl = 1;
    }
    const long VL = (long)o.vl;
    if (o.M == -1) {
        cerr << "error: matrix dimension M must be specified" << endl;
        rc = false;
    } else if (o.N == -1) {
        o.N = VL;  // 1-D work groups when N equals the vector length
    }
    if (o.M % VL) { cerr << "error: matrix dimension M must be multiple of " << VL << endl; rc = false; }
    if (o.N % VL) { cerr << "error: matrix dimension N must be multiple of " << VL << endl; rc = false; }
    return rc;
}

size_t mainLoop(KernelSaxpy &k, Bench &bench, Journal &journal, const vector<vector<size_t>> &pargs,
                vector<bool> &ok, vector<double> &avg, size_t trials, long topN, const Opts &o) {
    vector<size_t> time, flops;
    vector<double> var, avgDummy;
    vector<vector<size_t>> extra;
    vector<bool> okDummy;
    AppUtil::benchInit(pargs, okDummy, time, flops, avgDummy, var, extra);
    if (o.paranoid) k.paranoidCheck();
    size_t good = 0;
    for (size_t t = 0; t < trials; ++t) {
        good = AppUtil::benchLoop(t, k, bench, &journal, pargs, ok, time, flops, avg, var, extra, o.busTo, o.busFrom,
                                  t == 0, o.debug);
        if (topN != -1) AppUtil::markBench((size_t)topN, ok, time);
    }
    AppUtil::printBench(trials, pargs, ok, time, avg, var, extra);
    return good;
}

}  // namespace

int main(int argc, char **argv) {
    Opts o;
    if (!parse(argc, argv, o)) {
        cerr << "***DONE***" << endl;
        return 1;
    }
    Scalar s;
    Variant v;
    size_t vl;
    parse_type(o.type, &s, &v, &vl);
    KernelSaxpy kernel(s, v, vl);
    kernel.setPackedCalc(o.packed);
    Journal journal(o.journal);
    Bench bench(kernel, journal);
    const int dev = AppUtil::getDeviceIndex(o.device);
    if (dev >= 0) gatlas_set_device(dev);
    const size_t M = (size_t)o.M, N = (size_t)o.N;
    auto params = [&](long gh, long gw, long bh, long bw, long x) {
        return saxpy_search(kernel, vl, kMaxBlockHeight, kMaxGroupSize, M, N, gh, gw, bh, bw, x);
    };
    auto need_device = [&](const vector<vector<size_t>> &pargs) {
        if (dev >= 0) return;
        for (const auto &p : pargs)
            if (journal.memoRunState(kernel, p) == Journal::MISSING) {
                cerr << "error: no CUDA device " << o.device << endl << "***DONE***" << endl;
                exit(1);
            }
    };
    if (!o.em) {
        vector<vector<size_t>> pargs = params(-1, -1, -1, -1, -1);
        vector<bool> ok(pargs.size(), true);
        vector<double> avg(pargs.size(), 0.0);
        journal.loadMemo();
        need_device(pargs);
        mainLoop(kernel, bench, journal, pargs, ok, avg, o.trials, o.topN, o);
        cout << "***DONE***" << endl;
        return 0;
    }
    size_t bestGH = 0, bestGW = 0, bestBH = 1, bestBW = (vl == N) ? 0 : vl, bestXP = 0;
    int bestIndex = -1;
    bool foundMax = false;
    vector<vector<size_t>> pargs;
    while (!foundMax) {
        for (int emStep = 0; emStep <= 1; ++emStep) {
            while (bestIndex == -1) {
                if (emStep == 0)
                    pargs = params(-1, -1, (long)bestBH, (long)bestBW, (long)bestXP);
                else
                    pargs = params((long)bestGH, (long)bestGW, -1, -1, -1);
                vector<bool> ok(pargs.size(), true);
                vector<double> avg(pargs.size(), 0.0);
                journal.loadMemo();
                need_device(pargs);
                mainLoop(kernel, bench, journal, pargs, ok, avg, 1, o.topN, o);
                bestIndex = AppUtil::rankBench(0, ok, avg);
                if (bestIndex == -1) {
                    cerr << "error: no good kernels found for group height " << bestGH << ", group width " << bestGW
                         << ", block height " << bestBH << ", block width " << bestBW << " and extra parameter "
                         << bestXP << " so giving up" << endl
                         << "***DONE***" << endl;
                    return 1;
                }
                kernel.setParams(pargs[bestIndex]);
                if (bestGH == kernel.groupHeight() && bestGW == kernel.groupWidth() &&
                    bestBH == kernel.blockHeight() && bestBW == kernel.blockWidth() && bestXP == kernel.extraParam())
                    foundMax = true;
                bestGH = kernel.groupHeight();
                bestGW = kernel.groupWidth();
                bestBH = kernel.blockHeight();
                bestBW = kernel.blockWidth();
                bestXP = kernel.extraParam();
            }
            bestIndex = -1;
        }
    }
    if (o.trials > 1) {
        pargs = params((long)bestGH, (long)bestGW, (long)bestBH, (long)bestBW, (long)bestXP);
        vector<bool> ok(pargs.size(), true);
        vector<double> avg(pargs.size(), 0.0);
        need_device(pargs);
        mainLoop(kernel, bench, journal, pargs, ok, avg, o.trials, o.topN, o);
    }
    cout << "***DONE***" << endl;
    return 0;
}

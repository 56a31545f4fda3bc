// bench_matvec: autotune and time the matvec kernels on a B200.
//
// Reference: benchMatvec.cpp (options :68-200, search :202-289, EM loop as in
// benchMatmul.cpp :536-627).  Same options and output lines; -d gpuN selects
// a CUDA device.
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
    size_t packed = 1, trials = 1, maxBH = 64, maxWG = 256, vl = 1;
    long M = -1, N = -1, group = -1, bh = -1, xp = -1, topN = -1;
    bool gemv = false, em = false, tA = false, busTo = false, busFrom = false, paranoid = false, debug = false;
};

bool parse(int argc, char **argv, Opts &o) {
    int opt;
    while ((opt = getopt(argc, argv, "heasrpvzGd:j:C:T:m:n:g:y:x:t:w:")) != -1) {
        switch (opt) {
            case 'h':
                cerr << "usage: " << argv[0]
                     << " -d gpu|gpuX -j journalFile -T float1|float2|float4|double1|double2|double4|floatimg|doubleimg"
                        " -n N [-m M] [-C numKernels] [-g groupSize [-y blockHeight [-x extraParam]]]"
                        " [-t numberTrials] [-w topN] [-G] [-e] [-a] [-s] [-r] [-p] [-v] [-z] [-h]"
                     << endl
                     << "\t-G use general matrix vector multiply (default no)" << endl
                     << "\t-a transpose A (default no)" << endl
                     << "\t-e use faster expectation maximization optimization (default no)" << endl
                     << "\t-p paranoid output check (default no)" << endl
                     << "***DONE***" << endl;
                exit(1);
            case 'd': o.device = optarg; break;
            case 'j': o.journal = optarg; break;
            case 'C': o.packed = (size_t)atoi(optarg); break;
            case 'T': o.type = optarg; break;
            case 'm': o.M = atoi(optarg); break;
            case 'n': o.N = atoi(optarg); break;
            case 'g': o.group = atoi(optarg); break;
            case 'y': o.bh = atoi(optarg); break;
            case 'x': o.xp = atoi(optarg); break;
            case 't': o.trials = (size_t)atoi(optarg); break;
            case 'w': o.topN = atoi(optarg); break;
            case 'G': o.gemv = true; break;
            case 'e': o.em = true; break;
            case 'a': o.tA = true; break;
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
    if (!parse_type(o.type, &s, &v, &o.vl) || v == Variant::TcBf16 || v == Variant::TcSplit3 ||
        v == Variant::TcSplit6 || v == Variant::TcFp8) {
        cerr << "error: invalid kernel type of " << o.type << endl;
        rc = false;
        o.vl = 1;
    }
    const long VL = (long)o.vl;
    if (o.N == -1) { cerr << "error: matrix dimension N must be specified" << endl; rc = false; }
    else if (o.M == -1) o.M = o.N;
    if (o.N % VL) { cerr << "error: matrix dimension N must be multiple of " << VL << endl; rc = false; }
    if (o.M % VL) { cerr << "error: matrix dimension M must be multiple of " << VL << endl; rc = false; }
    if (o.group == -1 && o.bh != -1) { cerr << "error: group size must be specified with block height" << endl; rc = false; }
    if (o.group == -1 && o.bh == -1 && o.xp != -1) {
        cerr << "error: group size and block height must be specified with extra parameter" << endl;
        rc = false;
    }
    // benchMatvec.cpp:180 inherits the matmul limit of 16 for an explicit -g
    if (o.group != -1 && (o.group < 1 || o.group > 16)) {
        cerr << "error: work item group size must be a number from 1 to 16 inclusive" << endl;
        rc = false;
    }
    if (o.bh != -1 && (o.bh % VL)) { cerr << "error: inner blocking height must be multiple of " << VL << endl; rc = false; }
    if (o.bh != -1 && o.bh < VL) { cerr << "error: invalid inner blocking height" << endl; rc = false; }
    if (o.em && (o.group != -1 || o.bh != -1 || o.xp != -1)) {
        cerr << "error: expectation maximization optimization will find optimal blocking" << endl;
        rc = false;
    }
    return rc;
}

size_t mainLoop(KernelMatvec &k, Bench &bench, Journal &journal, const vector<vector<size_t>> &pargs,
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
    KernelMatvec kernel(s, v, vl);
    kernel.setPackedCalc(o.packed);
    Journal journal(o.journal);
    Bench bench(kernel, journal);
    const int dev = AppUtil::getDeviceIndex(o.device);
    if (dev >= 0) gatlas_set_device(dev);
    auto params = [&](long g, long b, long x) {
        return matvec_search(kernel, vl, o.maxBH, o.maxWG, o.gemv, (size_t)o.M, (size_t)o.N, o.tA, g, b, x);
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
        vector<vector<size_t>> pargs = params(o.group, o.bh, o.xp);
        vector<bool> ok(pargs.size(), true);
        vector<double> avg(pargs.size(), 0.0);
        journal.loadMemo();
        need_device(pargs);
        mainLoop(kernel, bench, journal, pargs, ok, avg, o.trials, o.topN, o);
        cout << "***DONE***" << endl;
        return 0;
    }
    size_t bestGroup = 0, bestBH = 0, bestXP = 0, loopCount = 0;
    int bestIndex = -1;
    bool foundMax = false;
    vector<vector<size_t>> pargs;
    while (!foundMax) {
        for (int emStep = 0; emStep <= 1; ++emStep) {
            while (bestIndex == -1) {
                pargs = params(emStep == 0 ? -1 : (long)bestGroup, emStep == 0 ? -1 : (long)bestBH,
                               emStep == 0 ? (long)bestXP : -1);
                vector<bool> ok(pargs.size(), true);
                vector<double> avg(pargs.size(), 0.0);
                journal.loadMemo();
                need_device(pargs);
                mainLoop(kernel, bench, journal, pargs, ok, avg, 1, o.topN, o);
                bestIndex = AppUtil::rankBench(0, ok, avg);
                if (bestIndex == -1) {
                    if (emStep == 0) {
                        bestXP = (bestXP + 1) % kernel.totalVariations();
                        if (kernel.totalVariations() == loopCount++) {
                            cerr << "error: no good kernels found so giving up" << endl << "***DONE***" << endl;
                            return 1;
                        }
                        continue;
                    }
                    cerr << "error: no good kernels found for group size " << bestGroup << " and block height "
                         << bestBH << " so giving up" << endl << "***DONE***" << endl;
                    return 1;
                }
                loopCount = 0;
                kernel.setParams(pargs[bestIndex]);
                if (bestGroup == kernel.groupSize() && bestBH == kernel.blockHeight() && bestXP == kernel.extraParam())
                    foundMax = true;
                bestGroup = kernel.groupSize();
                bestBH = kernel.blockHeight();
                bestXP = kernel.extraParam();
            }
            bestIndex = -1;
        }
    }
    if (o.trials > 1) {
        pargs = params((long)bestGroup, (long)bestBH, (long)bestXP);
        vector<bool> ok(pargs.size(), true);
        vector<double> avg(pargs.size(), 0.0);
        need_device(pargs);
        mainLoop(kernel, bench, journal, pargs, ok, avg, o.trials, o.topN, o);
    }
    cout << "***DONE***" << endl;
    return 0;
}

// Crash journal, one-point benchmark run, and the autotuning loop utilities.
//
// Reference: Journal and Bench (GatlasBenchmark.hpp:62-122,
// GatlasBenchmark.cpp:41-289) and AppUtil (GatlasAppUtil.hpp:29-99,
// GatlasAppUtil.cpp:28-416).  The journal file format, key format, run
// states, memo replay, purge rules, Welford statistics, top-N pruning,
// ranking and printed line formats are the reference's.  Timing uses CUDA
// events on the launch stream instead of gettimeofday, still reported in
// whole microseconds.
#pragma once

#include <cuda_runtime.h>

#include <map>
#include <string>
#include <vector>

#include "kernel.hpp"

namespace gatlas {
namespace host {

class Journal {
  public:
    enum RunState { MISSING = 0, BUILD_IN_PROGRESS = -1, BUILD_OK = -2, RUN_IN_PROGRESS = -3, RUN_OK = -4 };

    explicit Journal(const std::string &journalFile) : file_(journalFile) {}

    bool loadMemo();
    int purgeMemo(bool deleteTimes = false);
    size_t memoGood() const { return time_.size(); }
    int memoRunState(const KernelInterface &k, const std::vector<size_t> &params) const;
    int memoTime(const KernelInterface &k, const std::vector<size_t> &params, size_t trialNumber) const;
    bool takeMemo(const KernelInterface &k, const std::vector<size_t> &params, int value) const;

    static std::string key(const KernelInterface &k, const std::vector<size_t> &params);

    // The same records for a search whose subject is not a KernelInterface
    // (the grouped engine's tile tuner): `name` stands for kernelName().
    int memoRunState(const std::string &name, const std::vector<size_t> &params) const;
    int memoTime(const std::string &name, const std::vector<size_t> &params, size_t trialNumber) const;
    bool takeMemo(const std::string &name, const std::vector<size_t> &params, int value) const;
    static std::string key(const std::string &name, const std::vector<size_t> &params);

  private:
    std::string file_;
    std::map<std::string, int> state_;                  // all keys
    std::map<std::string, std::vector<size_t>> time_;   // keys with a time
};

class Bench {
  public:
    Bench(KernelInterface &kernel, bool printStatus = true) : kernel_(kernel), journal_(nullptr), print_(printStatus) {}
    Bench(KernelInterface &kernel, Journal &journal, bool printStatus = true)
        : kernel_(kernel), journal_(&journal), print_(printStatus) {}
    ~Bench();

    bool printStatus() const { return print_; }

    // Elapsed microseconds of numTrials launches, 0 on error or failed check.
    // busTransferToDevice / FromDevice include the host<->device copies of
    // the inputs / outputs in the timed region (GatlasBenchmark.cpp:198-265).
    size_t run(size_t numTrials, const std::vector<size_t> &args, bool busTransferToDevice,
               bool busTransferFromDevice, bool printDebug = false);

  private:
    KernelInterface &kernel_;
    Journal *journal_;
    bool print_;
    cudaStream_t stream_ = nullptr;  // legacy default stream
    cudaEvent_t ev0_ = nullptr, ev1_ = nullptr;
};

namespace AppUtil {

// "gpu", "gpu0", "gpuN" -> CUDA device index; "cpu"/"acc" have no device
// here and return -1 (GatlasAppUtil.cpp:30-60).
int getDeviceIndex(const std::string &device);

void benchInit(const std::vector<std::vector<size_t>> &pargs, std::vector<bool> &pargsOk,
               std::vector<size_t> &pargsTime, std::vector<size_t> &pargsFlops, std::vector<double> &pargsAverage,
               std::vector<double> &pargsVariance, std::vector<std::vector<size_t>> &pargsExtraDetail);

size_t benchLoop(size_t trialNumber, KernelInterface &kernel, Bench &bench, Journal *journal,
                 const std::vector<std::vector<size_t>> &pargs, std::vector<bool> &pargsOk,
                 std::vector<size_t> &pargsTime, std::vector<size_t> &pargsFlops, std::vector<double> &pargsAverage,
                 std::vector<double> &pargsVariance, std::vector<std::vector<size_t>> &pargsExtraDetail,
                 bool busTransferToDevice, bool busTransferFromDevice, bool dummyRun = false,
                 bool printDebug = false);

void markBench(size_t topN, std::vector<bool> &pargsOk, const std::vector<size_t> &pargsTime);
void markBench(size_t topN, std::vector<bool> &pargsOk, const std::vector<double> &pargsAverage);
int rankBench(size_t nthPlace, std::vector<bool> &pargsOk, const std::vector<double> &pargsAverage);
void printBench(size_t numberTrials, const std::vector<std::vector<size_t>> &pargs, const std::vector<bool> &pargsOk,
                const std::vector<size_t> &pargsTime, const std::vector<double> &pargsAverage,
                const std::vector<double> &pargsVariance, const std::vector<std::vector<size_t>> &pargsExtraDetail);

}  // namespace AppUtil

}  // namespace host
}  // namespace gatlas

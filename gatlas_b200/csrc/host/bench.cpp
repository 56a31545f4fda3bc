// Journal, Bench::run and AppUtil; see bench.hpp for the reference citations.
//
// The journal's file format and key format, the run states, the printed
// status lines and the statistics (Welford mean and variance, top-N pruning,
// ranking) restate GATLAS's GatlasBenchmark.cpp and GatlasAppUtil.cpp
// (Copyright 2010 Chris Jang), which are free software under the GNU Lesser
// General Public License, version 3 or later (the reference's
// COPYING.LESSER); the formats are kept byte for byte so that journals and
// tool output interoperate with the reference's.
#include "bench.hpp"

#include <cmath>
#include <fstream>
#include <iostream>
#include <set>
#include <sstream>

#include "../../../include/gatlas.h"

namespace gatlas {
namespace host {

// ---------------------------------------------------------------------------
// Journal (GatlasBenchmark.cpp:41-137)
// ---------------------------------------------------------------------------
std::string Journal::key(const std::string &name, const std::vector<size_t> &params) {
    std::stringstream ss;
    ss << name << "_";
    for (size_t p : params) ss << p << "_";
    return ss.str();
}

std::string Journal::key(const KernelInterface &k, const std::vector<size_t> &params) {
    return key(k.kernelName(), params);
}

bool Journal::loadMemo() {
    std::ifstream in(file_.c_str());
    if (!in.is_open()) return false;
    state_.clear();
    time_.clear();
    std::string k;
    int value;
    // a record is "key<whitespace>int"; reading stops at the first malformed record
    while (!in.eof() && (in >> k >> value)) {
        if (value < 0)
            state_[k] = value;
        else
            time_[k].push_back((size_t)value);
    }
    return true;
}

int Journal::purgeMemo(bool deleteTimes) {
    int count = -1;
    std::ofstream out(file_.c_str());
    if (out.is_open()) {
        count = 0;
        for (const auto &kv : state_) {
            auto t = time_.find(kv.first);
            if (t == time_.end()) {
                // no time recorded: a kernel that crashed while building or hung while running
                out << kv.first << "\t" << kv.second << std::endl;
                ++count;
            } else if (!deleteTimes) {
                out << kv.first << "\t" << kv.second << std::endl;
                for (size_t v : t->second) out << kv.first << "\t" << v << std::endl;
            }
        }
    }
    return count;
}

int Journal::memoRunState(const std::string &name, const std::vector<size_t> &params) const {
    auto it = state_.find(key(name, params));
    return it == state_.end() ? MISSING : it->second;
}

int Journal::memoTime(const std::string &name, const std::vector<size_t> &params, size_t trial) const {
    auto it = time_.find(key(name, params));
    if (it == time_.end() || trial >= it->second.size()) return -1;
    return (int)it->second[trial];
}

bool Journal::takeMemo(const std::string &name, const std::vector<size_t> &params, int value) const {
    // append and close on every record, so a crash loses nothing already written
    std::ofstream out(file_.c_str(), std::ios::app);
    if (!out.is_open()) return false;
    out << key(name, params) << "\t" << value << std::endl;
    return true;
}

int Journal::memoRunState(const KernelInterface &k, const std::vector<size_t> &params) const {
    return memoRunState(k.kernelName(), params);
}

int Journal::memoTime(const KernelInterface &k, const std::vector<size_t> &params, size_t trial) const {
    return memoTime(k.kernelName(), params, trial);
}

bool Journal::takeMemo(const KernelInterface &k, const std::vector<size_t> &params, int value) const {
    return takeMemo(k.kernelName(), params, value);
}

// ---------------------------------------------------------------------------
// Bench (GatlasBenchmark.cpp:139-289)
// ---------------------------------------------------------------------------
Bench::~Bench() {
    if (ev0_) cudaEventDestroy(ev0_);
    if (ev1_) cudaEventDestroy(ev1_);
}

size_t Bench::run(size_t numTrials, const std::vector<size_t> &args, bool busToDevice, bool busFromDevice,
                  bool printDebug) {
    kernel_.setParams(args);
    if (print_ && printDebug) std::cerr << kernel_ << std::endl;

    if (journal_) journal_->takeMemo(kernel_, args, Journal::BUILD_IN_PROGRESS);
    if (print_) std::cerr << "rebuilding kernel...";
    if (!kernel_.build()) return 0;  // state stays BUILD_IN_PROGRESS: "bad" on the next run
    if (print_) std::cerr << " done\t";
    if (journal_) journal_->takeMemo(kernel_, args, Journal::BUILD_OK);

    // Everything runs on the legacy default stream, where the kernel objects
    // also do their copies, so the events bracket copies and launches alike.
    if (!ev0_) {
        if (cudaEventCreate(&ev0_) != cudaSuccess || cudaEventCreate(&ev1_) != cudaSuccess) {
            if (print_) std::cerr << "error: event creation" << std::endl;
            return 0;
        }
    }
    if (!busToDevice && !kernel_.setArgs(false)) return 0;
    if (journal_) journal_->takeMemo(kernel_, args, Journal::RUN_IN_PROGRESS);

    int faults = 0;
    gatlas_device_faults(&faults, 1);
    cudaEventRecord(ev0_, stream_);
    if (busToDevice && !kernel_.setArgs(true)) return 0;
    for (size_t i = 0; i < numTrials; ++i) {
        if (!kernel_.enqueue(stream_)) {
            if (print_) std::cerr << "error: enqueue kernel " << i << std::endl;
            cudaStreamSynchronize(stream_);
            return 0;
        }
    }
    if (busFromDevice && !kernel_.syncOutput()) return 0;
    cudaEventRecord(ev1_, stream_);
    if (cudaEventSynchronize(ev1_) != cudaSuccess) {
        if (print_) std::cerr << "error: waiting for all kernels" << std::endl;
        return 0;  // state stays RUN_IN_PROGRESS
    }
    float ms = 0;
    cudaEventElapsedTime(&ms, ev0_, ev1_);
    if (gatlas_device_faults(&faults, 1) == GATLAS_OK && faults != 0) {
        // a bounded device wait gave up: treat like a hung kernel and leave the
        // journal in RUN_IN_PROGRESS so that a resumed search skips this point
        if (print_) std::cerr << "error: device wait timed out (fault flags " << faults << ")" << std::endl;
        return 0;
    }
    if (!busFromDevice && !kernel_.syncOutput()) {
        if (print_) std::cerr << "error: read output data from device" << std::endl;
        return 0;
    }
    size_t usec = (size_t)std::llround((double)ms * 1000.0);
    if (usec == 0) usec = 1;

    const bool ok = kernel_.checkOutput(printDebug);
    if (!ok && print_) std::cerr << "fail";
    if (journal_) {
        journal_->takeMemo(kernel_, args, Journal::RUN_OK);
        journal_->takeMemo(kernel_, args, ok ? (int)usec : 0);
    }
    return ok ? usec : 0;
}

// ---------------------------------------------------------------------------
// AppUtil (GatlasAppUtil.cpp:28-416)
// ---------------------------------------------------------------------------
namespace AppUtil {

int getDeviceIndex(const std::string &device) {
    if (device.compare(0, 3, "gpu") != 0) return -1;
    size_t index = 0;
    if (device.size() > 3) {
        std::stringstream ss(device.substr(3));
        ss >> index;
    }
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || (int)index >= count) return -1;
    return (int)index;
}

void benchInit(const std::vector<std::vector<size_t>> &pargs, std::vector<bool> &ok, std::vector<size_t> &time,
               std::vector<size_t> &flops, std::vector<double> &avg, std::vector<double> &var,
               std::vector<std::vector<size_t>> &extra) {
    const size_t n = pargs.size();
    ok.assign(n, true);
    time.assign(n, 0);
    flops.assign(n, 0);
    avg.assign(n, 0);
    var.assign(n, 0);
    extra.assign(n, std::vector<size_t>());
}

static void print_point(const std::vector<size_t> &args, const std::vector<size_t> &extra) {
    for (size_t i = 0; i < args.size(); ++i) std::cout << args[i] << (i + 1 < args.size() ? " " : "");
    std::cout << "\t(";
    for (size_t i = 0; i < extra.size(); ++i) std::cout << extra[i] << (i + 1 < extra.size() ? " " : "");
    std::cout << ")" << std::endl;
}

namespace {

// One candidate's time for this trial: a new point is run on the device; a
// point the journal recorded as good replays its recorded time for this
// trial (run only if the journal has no time for it); a point the journal
// recorded mid-build or mid-run (a crash or hang) scores 0 without running.
size_t trial_time(size_t trial, KernelInterface &kernel, Bench &bench, const Journal *journal, int memoState,
                  const std::vector<size_t> &args, bool toDevice, bool fromDevice, bool printDebug) {
    if (memoState == Journal::MISSING) return bench.run(1, args, toDevice, fromDevice, printDebug);
    kernel.setParams(args);
    if (memoState != Journal::RUN_OK) {
        if (bench.printStatus()) std::cout << "bad";
        return 0;
    }
    const int memo = journal->memoTime(kernel, args, trial);
    return memo == -1 ? bench.run(1, args, toDevice, fromDevice, printDebug) : (size_t)memo;
}

// Running GFLOPS mean and variance over the trials (Welford's update).
void accumulate(size_t trial, double rate, double &mean, double &var) {
    if (trial == 0) {
        mean = rate;
        return;
    }
    const double delta = rate - mean;
    mean += delta / (double)(trial + 1);
    var += (double)trial / (double)(trial + 1) * delta * delta;
}

}  // namespace

size_t benchLoop(size_t trialNumber, KernelInterface &kernel, Bench &bench, Journal *journal,
                 const std::vector<std::vector<size_t>> &pargs, std::vector<bool> &pargsOk,
                 std::vector<size_t> &pargsTime, std::vector<size_t> &pargsFlops, std::vector<double> &pargsAverage,
                 std::vector<double> &pargsVariance, std::vector<std::vector<size_t>> &pargsExtraDetail,
                 bool busToDevice, bool busFromDevice, bool dummyRun, bool printDebug) {
    const bool status = bench.printStatus();
    bool warmed = !dummyRun;  // one untimed launch before the first point that really runs
    size_t good = 0;
    for (size_t j = 0; j < pargs.size(); ++j) {
        if (!pargsOk[j]) continue;
        const std::vector<size_t> &args = pargs[j];
        const int memoState = journal ? journal->memoRunState(kernel, args) : (int)Journal::MISSING;
        if (!warmed && memoState == Journal::MISSING) {
            std::cout << "[dummy run] ";
            bench.run(1, args, busToDevice, busFromDevice, printDebug);
            std::cout << std::endl;
            warmed = true;
        }
        if (status) std::cout << "[trial " << trialNumber << "] ";
        const size_t usec =
            trial_time(trialNumber, kernel, bench, journal, memoState, args, busToDevice, busFromDevice, printDebug);
        pargsExtraDetail[j] = kernel.extraParamDetail();
        if (usec > 0) {
            const size_t nflops = kernel.numberFlops();
            pargsTime[j] += usec;
            pargsFlops[j] += nflops;
            accumulate(trialNumber, (double)nflops / (double)usec / 1000.0, pargsAverage[j], pargsVariance[j]);
            ++good;
        } else {
            pargsOk[j] = false;  // pruned from every later trial
        }
        if (status) {
            if (usec > 0) std::cout << usec;
            std::cout << "\t";
            print_point(args, pargsExtraDetail[j]);
        }
    }
    return good;
}

void markBench(size_t topN, std::vector<bool> &ok, const std::vector<size_t> &time) {
    // keep the topN fastest accumulated times; equal times are kept together
    std::set<size_t> times;
    for (size_t i = 0; i < ok.size(); ++i)
        if (ok[i]) times.insert(time[i]);
    std::set<size_t> top;
    size_t count = 0;
    for (size_t t : times) {
        if (count++ >= topN) break;
        top.insert(t);
    }
    for (size_t i = 0; i < ok.size(); ++i)
        if (ok[i] && !top.count(time[i])) ok[i] = false;
}

void markBench(size_t topN, std::vector<bool> &ok, const std::vector<double> &avg) {
    std::set<double> avgs;
    for (size_t i = 0; i < ok.size(); ++i)
        if (ok[i]) avgs.insert(avg[i]);
    std::set<double> top;
    size_t count = 0;
    for (auto it = avgs.rbegin(); it != avgs.rend(); ++it) {
        if (count++ >= topN) break;
        top.insert(*it);
    }
    for (size_t i = 0; i < ok.size(); ++i)
        if (ok[i] && !top.count(avg[i])) ok[i] = false;
}

int rankBench(size_t nthPlace, std::vector<bool> &ok, const std::vector<double> &avg) {
    std::map<double, size_t> byRate;
    for (size_t i = 0; i < ok.size(); ++i)
        if (ok[i]) byRate[avg[i]] = i;
    size_t count = 0;
    for (auto it = byRate.rbegin(); it != byRate.rend(); ++it)
        if (nthPlace == count++) return (int)it->second;
    return -1;
}

void printBench(size_t numberTrials, const std::vector<std::vector<size_t>> &pargs, const std::vector<bool> &ok,
                const std::vector<size_t> &time, const std::vector<double> &avg, const std::vector<double> &var,
                const std::vector<std::vector<size_t>> &extra) {
    std::map<size_t, size_t> byTime;
    for (size_t i = 0; i < pargs.size(); ++i)
        if (ok[i]) byTime[time[i]] = i;
    size_t count = 0;
    for (const auto &kv : byTime) {
        const size_t idx = kv.second;
        std::cout << "[" << count++ << "] " << kv.first << " usec"
                  << "\tavg: " << avg[idx] << "\tstddev: " << std::sqrt(var[idx] / numberTrials) << "\t";
        print_point(pargs[idx], extra[idx]);
    }
}

}  // namespace AppUtil

}  // namespace host
}  // namespace gatlas

// Autotuner for the grouped engine's tile width per size bucket.
//
// The successor to the reference's search (benchMatmul.cpp:258-300 driving
// AppUtil::benchLoop, GatlasAppUtil.cpp:188-270): one seeded synthetic group
// mixes the shapes of every bucket; bucket by bucket (coordinate descent), it
// times the whole group at each candidate tile width for that bucket, the
// other buckets at their current widths, and keeps the fastest.  Every candidate is recorded in the same
// crash journal with the same run states (GatlasBenchmark.cpp:185-288):
// build in progress, build ok, run in progress, run ok, microseconds.  A
// resumed search replays recorded times without touching the device and
// skips candidates that crashed while building or hung while running.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <iostream>
#include <string>
#include <vector>

#include "../../../include/gatlas.h"
#include "../common.cuh"
#include "bench.hpp"

namespace gatlas {
namespace host {

namespace {

constexpr int kCandidates[3] = {64, 128, 256};
constexpr int kTuneInstances = 48;

// n range of each bucket (multiples of 16)
void bucket_range(int b, int64_t *lo, int64_t *hi) {
    static const int64_t r[4][2] = {{16, 64}, {80, 128}, {144, 256}, {272, 4096}};
    *lo = r[b][0];
    *hi = r[b][1];
}

// log-uniform integer in [lo, hi], rounded to a multiple of 16
int64_t log_uniform16(uint64_t *state, int64_t lo, int64_t hi) {
    *state = splitmix64(*state);
    const double u = (double)(*state >> 11) * 0x1.0p-53;
    const double v = std::exp(std::log((double)lo) + u * (std::log((double)hi) - std::log((double)lo)));
    int64_t x = (int64_t)std::llround(v / 16.0) * 16;
    if (x < lo) x = lo;
    if (x > hi) x = hi;
    return x;
}

}  // namespace

// Shapes of the synthetic group for one bucket (deterministic in seed).
std::vector<gatlas_grouped_instance> tune_shapes(int bucket, uint64_t seed) {
    int64_t lo, hi;
    bucket_range(bucket, &lo, &hi);
    uint64_t st = seed * 0x9E3779B97F4A7C15ull + (uint64_t)bucket;
    std::vector<gatlas_grouped_instance> v(kTuneInstances);
    for (auto &q : v) {
        std::memset(&q, 0, sizeof(q));
        q.m = log_uniform16(&st, 16, 4096);
        q.n = log_uniform16(&st, lo, hi);
        q.k = log_uniform16(&st, 16, 4096);
        st = splitmix64(st);
        q.trans_a = (int32_t)(st & 1);
        q.trans_b = (int32_t)((st >> 1) & 1);
        q.alpha = 1.0;
    }
    return v;
}

}  // namespace host
}  // namespace gatlas

extern "C" int gatlas_grouped_autotune(int engine, const char *journal_path, int32_t trials, uint64_t seed,
                                       int32_t *out_table) {
    using namespace gatlas;
    using namespace gatlas::host;
    if (engine != GATLAS_ENGINE_TC_BF16 && engine != GATLAS_ENGINE_TC_SPLIT3)
        return set_error(GATLAS_ERR_UNSUPPORTED, "grouped autotune: engine %d has no grouped kernel", engine);
    if (trials < 1) trials = 1;
    const std::string name = engine == GATLAS_ENGINE_TC_SPLIT3 ? "groupedtcsplit3" : "groupedtcbf16";
    Journal journal(journal_path ? journal_path : "");
    const bool use_journal = journal_path && *journal_path;
    if (use_journal) journal.loadMemo();
    int32_t table[GATLAS_GROUPED_BUCKETS];
    int rc = gatlas_grouped_get_tile_table(engine, table, GATLAS_GROUPED_BUCKETS);
    if (rc) return rc;

    // One mixed group: the synthetic shapes of every bucket together.  A tile
    // width is worth what it does beside the other buckets' instances, which
    // supply the parallelism that small tiles would otherwise buy alone.
    std::vector<gatlas_grouped_instance> inst;
    std::vector<int> bucket_of;
    for (int b = 0; b < GATLAS_GROUPED_BUCKETS; ++b) {
        const std::vector<gatlas_grouped_instance> part = tune_shapes(b, seed);
        inst.insert(inst.end(), part.begin(), part.end());
        bucket_of.insert(bucket_of.end(), part.size(), b);
    }
    size_t na = 0, nb = 0, nc = 0;
    for (const auto &q : inst) {
        na += ((size_t)q.m * q.k + 15) / 16 * 16;
        nb += ((size_t)q.k * q.n + 15) / 16 * 16;
        nc += ((size_t)q.m * q.n + 15) / 16 * 16;
    }
    float *dA = nullptr, *dB = nullptr, *dC = nullptr;
    if (cudaMalloc(&dA, na * 4) != cudaSuccess || cudaMalloc(&dB, nb * 4) != cudaSuccess ||
        cudaMalloc(&dC, nc * 4) != cudaSuccess) {
        cudaGetLastError();
        cudaFree(dA);
        cudaFree(dB);
        cudaFree(dC);
        return set_error(GATLAS_ERR_NOMEM, "grouped autotune: operands");
    }
    cudaStream_t stream = nullptr;
    gatlas_fill_f32(dA, na, GATLAS_DIST_UNIFORM, seed + 1, 0, 0.0f, stream);
    gatlas_fill_f32(dB, nb, GATLAS_DIST_UNIFORM, seed + 2, 0, 0.0f, stream);
    size_t oa = 0, ob = 0, oc = 0;
    for (auto &q : inst) {
        q.a = dA + oa;
        q.b = dB + ob;
        q.c = dC + oc;
        oa += ((size_t)q.m * q.k + 15) / 16 * 16;
        ob += ((size_t)q.k * q.n + 15) / 16 * 16;
        oc += ((size_t)q.m * q.n + 15) / 16 * 16;
    }
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
        cudaFree(dA);
        cudaFree(dB);
        cudaFree(dC);
        return set_error(GATLAS_ERR_CUDA, "grouped autotune: events");
    }

    // Times the mixed group with `t` as the table; 0 when the point failed.
    // Recorded under the bucket and width being tried plus the whole table.
    auto measure = [&](int b, const int32_t *t) -> size_t {
        const std::vector<size_t> params = {(size_t)b,    (size_t)t[b], (size_t)inst.size(), (size_t)seed,
                                            (size_t)t[0], (size_t)t[1], (size_t)t[2],        (size_t)t[3]};
        const int state = use_journal ? journal.memoRunState(name, params) : (int)Journal::MISSING;
        if (state == Journal::RUN_OK) {
            const int v = journal.memoTime(name, params, 0);
            return v > 0 ? (size_t)v : 0;
        }
        if (state != Journal::MISSING) return 0;  // crashed while building or hung while running earlier
        for (size_t i = 0; i < inst.size(); ++i) inst[i].tile_n = t[bucket_of[i]];
        if (use_journal) journal.takeMemo(name, params, Journal::BUILD_IN_PROGRESS);
        gatlas_grouped_plan *plan = nullptr;
        if (gatlas_grouped_create(engine, inst.data(), (int32_t)inst.size(), nullptr, 0, &plan) != GATLAS_OK)
            return 0;
        if (use_journal) journal.takeMemo(name, params, Journal::BUILD_OK);
        if (use_journal) journal.takeMemo(name, params, Journal::RUN_IN_PROGRESS);
        int f0 = 0, f1 = 0;
        gatlas_device_faults(&f0, 0);
        int r = gatlas_grouped_prepare(plan, stream);
        if (!r) r = gatlas_grouped_run(plan, stream);  // warm-up
        cudaEventRecord(e0, stream);
        for (int k = 0; k < trials && !r; ++k) r = gatlas_grouped_run(plan, stream);
        cudaEventRecord(e1, stream);
        const bool synced = cudaEventSynchronize(e1) == cudaSuccess;
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, e0, e1);
        gatlas_device_faults(&f1, 0);
        gatlas_grouped_destroy(plan);
        const bool ok = !r && synced && f1 == f0;
        size_t usec = ok ? (size_t)std::llround(1000.0 * ms) : 0;
        if (ok && usec == 0) usec = 1;
        if (use_journal) {
            journal.takeMemo(name, params, Journal::RUN_OK);
            journal.takeMemo(name, params, (int)usec);
        }
        return usec;
    };

    // one pass of coordinate descent over the buckets
    for (int b = 0; b < GATLAS_GROUPED_BUCKETS; ++b) {
        size_t best = 0;
        int best_bn = table[b];
        for (int bn : kCandidates) {
            int32_t t[GATLAS_GROUPED_BUCKETS];
            std::memcpy(t, table, sizeof(t));
            t[b] = bn;
            const size_t usec = measure(b, t);
            if (usec && (!best || usec < best)) {
                best = usec;
                best_bn = bn;
            }
        }
        table[b] = best_bn;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(dA);
    cudaFree(dB);
    cudaFree(dC);
    rc = gatlas_grouped_set_tile_table(engine, table, GATLAS_GROUPED_BUCKETS);
    if (rc) return rc;
    if (out_table) std::memcpy(out_table, table, sizeof(table));
    return GATLAS_OK;
}

// Serving loop: mixed GEMM / GEMV / SAXPY requests replayed in real time
// with continuous batching under a device-memory admission budget.
//
// No reference counterpart (the reference benchmarks one kernel at a time,
// GatlasBenchmark.cpp:178-289).  Design:
//  * one device arena of `budget_bytes` holds every admitted request's
//    operands, result and packed pieces (first fit, coalescing frees);
//    admission is FIFO and stops at the first request that does not fit, so
//    requests wait for memory instead of overtaking one another;
//  * an admitted request's operands are generated on the prep stream from
//    its seed (seeded uniform[-1,1) streams, as a client upload would land);
//  * GEMMs are batched continuously: whenever fewer than two GEMM batches
//    are on the device, every admitted GEMM not yet batched (in arrival
//    order, up to max_batch or the batch time target) goes into one grouped
//    tcgen05 launch (pack + contraction) whose tables are built on the host
//    and copied asynchronously from pinned staging;
//  * GEMVs and SAXPYs are launched as they are admitted on a second compute
//    stream, so memory-bound work overlaps the tensor-core batches;
//  * completion times come from CUDA events on the device timeline.
// The serial comparator runs one request at a time: wait for its arrival,
// generate its operands, one engine call, synchronise.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstring>
#include <deque>
#include <map>
#include <thread>
#include <vector>

#include "../../../include/gatlas.h"
#include "../kernels/grouped.hpp"
#include "../status.hpp"

namespace gatlas {

namespace {

constexpr size_t kAlign = 1024;

size_t up(size_t x) { return (x + kAlign - 1) / kAlign * kAlign; }

int64_t now_ns() {
    return std::chrono::duration_cast<std::chrono::nanoseconds>(std::chrono::steady_clock::now().time_since_epoch())
        .count();
}

// Best-fit arena with coalescing frees over one device allocation: free
// blocks indexed by offset (for coalescing) and by size (for O(log n) fits).
class Arena {
  public:
    ~Arena() { cudaFree(raw_); }
    int init(size_t bytes) {
        size_ = bytes / kAlign * kAlign;
        if (cudaMalloc(&raw_, size_ + kAlign) != cudaSuccess) {
            cudaGetLastError();
            raw_ = nullptr;
            return set_error(GATLAS_ERR_NOMEM, "server: arena of %zu bytes", size_);
        }
        // every block starts on a 1024-byte boundary (tensor-core workspaces)
        base_ = raw_ + (kAlign - reinterpret_cast<uintptr_t>(raw_) % kAlign) % kAlign;
        insert(0, size_);
        return GATLAS_OK;
    }
    uint8_t *alloc(size_t bytes) {
        bytes = up(bytes ? bytes : 1);
        auto it = by_size_.lower_bound(bytes);
        if (it == by_size_.end()) return nullptr;
        const size_t off = it->second, have = it->first;
        by_size_.erase(it);
        by_off_.erase(off);
        if (have > bytes) insert(off + bytes, have - bytes);
        used_ += bytes;
        peak_ = std::max(peak_, used_);
        return base_ + off;
    }
    void release(uint8_t *p, size_t bytes) {
        bytes = up(bytes ? bytes : 1);
        size_t off = (size_t)(p - base_);
        used_ -= bytes;
        ++epoch_;
        auto next = by_off_.lower_bound(off);
        if (next != by_off_.end() && off + bytes == next->first) {
            bytes += next->second;
            erase(next->first, next->second);
            next = by_off_.lower_bound(off);
        }
        if (next != by_off_.begin()) {
            auto prev = std::prev(next);
            if (prev->first + prev->second == off) {
                off = prev->first;
                bytes += prev->second;
                erase(prev->first, prev->second);
            }
        }
        insert(off, bytes);
    }
    size_t size() const { return size_; }
    size_t peak() const { return peak_; }
    size_t used() const { return used_; }
    uint64_t epoch() const { return epoch_; }  // counts releases

  private:
    void insert(size_t off, size_t bytes) {
        by_off_[off] = bytes;
        by_size_.emplace(bytes, off);
    }
    void erase(size_t off, size_t bytes) {
        by_off_.erase(off);
        auto range = by_size_.equal_range(bytes);
        for (auto it = range.first; it != range.second; ++it)
            if (it->second == off) {
                by_size_.erase(it);
                break;
            }
    }
    uint8_t *raw_ = nullptr, *base_ = nullptr;
    size_t size_ = 0, used_ = 0, peak_ = 0;
    uint64_t epoch_ = 0;
    std::map<size_t, size_t> by_off_;
    std::multimap<size_t, size_t> by_size_;
};

struct Slot {  // double-buffered grouped tables
    void *dev = nullptr, *host = nullptr;
    size_t cap = 0;
    bool busy = false;
};

}  // namespace

struct Server {
    gatlas_server_config cfg;
    Arena arena;
    cudaStream_t prep = nullptr, sg = nullptr, sm = nullptr;
    cudaEvent_t start = nullptr;
    std::vector<cudaEvent_t> event_pool;
    Slot slots[2];
    std::map<float *, std::pair<uint8_t *, size_t>> retained;  // result -> allocation
    int64_t batches = 0, batched_gemms = 0, host_busy_ns = 0, iterations = 0;
    int64_t phase_ns[5] = {0, 0, 0, 0, 0};
    int64_t generate_ns = 0, generate_launches = 0;
    int device = 0;

    cudaEvent_t get_event() {
        if (!event_pool.empty()) {
            cudaEvent_t e = event_pool.back();
            event_pool.pop_back();
            return e;
        }
        cudaEvent_t e = nullptr;
        cudaEventCreate(&e);
        return e;
    }
    void put_event(cudaEvent_t e) { event_pool.push_back(e); }
    ~Server() {
        cudaDeviceSynchronize();
        for (auto e : event_pool) cudaEventDestroy(e);
        for (auto &s : slots) {
            cudaFree(s.dev);
            cudaFreeHost(s.host);
        }
        if (start) cudaEventDestroy(start);
        for (cudaStream_t s : {prep, sg, sm})
            if (s) cudaStreamDestroy(s);
    }
};

namespace {

// Device memory of one request: operands, result and engine scratch.
struct Layout {
    size_t a = 0, b = 0, c = 0, ws = 0, total = 0;  // byte offsets / sizes
};

int request_layout(const Server &S, const gatlas_request &r, int serial, Layout *L) {
    switch (r.kind) {
        case GATLAS_REQ_GEMM: {
            if (r.m < 0 || r.n < 0 || r.k < 0) return set_error(GATLAS_ERR_INVALID, "server: negative GEMM dimension");
            const size_t a = up((size_t)r.m * r.k * 4), b = up((size_t)r.k * r.n * 4), c = up((size_t)r.m * r.n * 4);
            size_t ws = 0;
            if (serial) {
                gatlas_matmul_desc d;
                std::memset(&d, 0, sizeof(d));
                d.engine = S.cfg.gemm_engine;
                d.m = r.m, d.n = r.n, d.k = r.k, d.trans_a = r.trans_a, d.trans_b = r.trans_b;
                ws = up(gatlas_matmul_workspace_size(&d));
            } else {
                gatlas_grouped_instance q;
                std::memset(&q, 0, sizeof(q));
                q.m = r.m, q.n = r.n, q.k = r.k, q.trans_a = r.trans_a, q.trans_b = r.trans_b;
                const int rc = grouped_instance_bytes(S.cfg.gemm_engine, q, &ws);
                if (rc) return rc;
                ws = up(ws);
            }
            L->a = 0, L->b = a, L->c = a + b, L->ws = a + b + c, L->total = a + b + c + ws;
            return GATLAS_OK;
        }
        case GATLAS_REQ_GEMV: {
            if (r.m < 0 || r.n < 0) return set_error(GATLAS_ERR_INVALID, "server: negative GEMV dimension");
            gatlas_matvec_desc d;
            std::memset(&d, 0, sizeof(d));
            d.gemv = 1, d.trans_a = r.trans_a, d.m = r.m, d.n = r.n;
            const size_t a = up((size_t)r.m * r.n * 4), x = up((size_t)r.n * 4), y = up((size_t)r.m * 4);
            const size_t ws = up(gatlas_matvec_workspace_size(&d));
            L->a = 0, L->b = a, L->c = a + x, L->ws = a + x + y, L->total = a + x + y + ws;
            return GATLAS_OK;
        }
        case GATLAS_REQ_SAXPY: {
            if (r.n < 0) return set_error(GATLAS_ERR_INVALID, "server: negative SAXPY length");
            const size_t x = up((size_t)r.n * 4);
            L->a = 0, L->b = 0, L->c = x, L->ws = 2 * x, L->total = 2 * x;  // x at a, y (result) at c
            return GATLAS_OK;
        }
        default: return set_error(GATLAS_ERR_INVALID, "server: unknown request kind %d", r.kind);
    }
}

int64_t result_elems(const gatlas_request &r) {
    return r.kind == GATLAS_REQ_GEMM ? r.m * r.n : r.kind == GATLAS_REQ_GEMV ? r.m : r.n;
}

// Operands from the request's seed: streams 4*seed + {0, 1, 2} for the
// first operand, the second operand and the initial result.
int generate(const gatlas_request &r, uint8_t *mem, const Layout &L, cudaStream_t s) {
    float *p0 = reinterpret_cast<float *>(mem + L.a), *p1 = reinterpret_cast<float *>(mem + L.b);
    float *pc = reinterpret_cast<float *>(mem + L.c);
    const uint64_t sd = r.seed * 4;
    int rc = GATLAS_OK;
    if (r.kind == GATLAS_REQ_GEMM) {
        rc = gatlas_fill_f32(p0, (size_t)r.m * r.k, GATLAS_DIST_UNIFORM, sd, 0, 0.0f, s);
        if (!rc) rc = gatlas_fill_f32(p1, (size_t)r.k * r.n, GATLAS_DIST_UNIFORM, sd + 1, 0, 0.0f, s);
        if (!rc && r.beta != 0.0) rc = gatlas_fill_f32(pc, (size_t)r.m * r.n, GATLAS_DIST_UNIFORM, sd + 2, 0, 0.0f, s);
    } else if (r.kind == GATLAS_REQ_GEMV) {
        rc = gatlas_fill_f32(p0, (size_t)r.m * r.n, GATLAS_DIST_UNIFORM, sd, 0, 0.0f, s);
        if (!rc) rc = gatlas_fill_f32(p1, (size_t)r.n, GATLAS_DIST_UNIFORM, sd + 1, 0, 0.0f, s);
        if (!rc && r.beta != 0.0) rc = gatlas_fill_f32(pc, (size_t)r.m, GATLAS_DIST_UNIFORM, sd + 2, 0, 0.0f, s);
    } else {
        rc = gatlas_fill_f32(p0, (size_t)r.n, GATLAS_DIST_UNIFORM, sd, 0, 0.0f, s);
        if (!rc) rc = gatlas_fill_f32(pc, (size_t)r.n, GATLAS_DIST_UNIFORM, sd + 2, 0, 0.0f, s);
    }
    return rc;
}

// Fill launches generate() makes for a request.
int generate_launch_count(const gatlas_request &r) {
    if (r.kind == GATLAS_REQ_SAXPY) return 2;
    return r.beta != 0.0 ? 3 : 2;
}

// One request through its single-instance engine call (GEMV, SAXPY, and
// the serial comparator's GEMM).
int launch_single(const Server &S, const gatlas_request &r, uint8_t *mem, const Layout &L, cudaStream_t s) {
    float *p0 = reinterpret_cast<float *>(mem + L.a), *p1 = reinterpret_cast<float *>(mem + L.b);
    float *pc = reinterpret_cast<float *>(mem + L.c);
    void *ws = mem + L.ws;
    if (r.kind == GATLAS_REQ_GEMM) {
        gatlas_matmul_desc d;
        std::memset(&d, 0, sizeof(d));
        d.engine = S.cfg.gemm_engine;
        d.gemm = 1;
        d.m = r.m, d.n = r.n, d.k = r.k, d.trans_a = r.trans_a, d.trans_b = r.trans_b;
        d.alpha = r.alpha, d.beta = r.beta;
        return gatlas_matmul_f32(&d, p0, p1, pc, ws, L.total - L.ws, s);
    }
    if (r.kind == GATLAS_REQ_GEMV) {
        gatlas_matvec_desc d;
        std::memset(&d, 0, sizeof(d));
        d.gemv = 1, d.trans_a = r.trans_a, d.m = r.m, d.n = r.n;
        d.alpha = r.alpha, d.beta = r.beta;
        return gatlas_matvec_f32(&d, p0, p1, pc, ws, L.total - L.ws, s);
    }
    return gatlas_saxpy_f32(GATLAS_ENGINE_BUFFER, (size_t)r.n, (float)r.alpha, p0, pc, pc, s);
}

double request_flops(const gatlas_request &r) {
    if (r.kind == GATLAS_REQ_GEMM) return 2.0 * r.m * r.n * r.k;
    if (r.kind == GATLAS_REQ_GEMV) return 2.0 * r.m * r.n;
    return 2.0 * r.n;
}

struct RState {
    uint8_t *mem = nullptr;
    Layout L;
};

void finish(Server &S, const gatlas_request &r, RState &st, gatlas_request_result &res) {
    if (r.retain && st.mem) {
        res.result = reinterpret_cast<float *>(st.mem + st.L.c);
        res.result_elems = result_elems(r);
        S.retained[res.result] = {st.mem, st.L.total};
    } else if (st.mem) {
        S.arena.release(st.mem, st.L.total);
    }
    st.mem = nullptr;
}

int64_t elapsed_ns(const Server &S, cudaEvent_t e) {
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, S.start, e);
    return (int64_t)((double)ms * 1e6);
}

// Waits until host time t0 + target_ns, sleeping while far away.
void wait_until(int64_t t0, int64_t target_ns) {
    for (;;) {
        const int64_t left = target_ns - (now_ns() - t0);
        if (left <= 0) return;
        if (left > 200000) std::this_thread::sleep_for(std::chrono::nanoseconds(left - 100000));
        else std::this_thread::yield();
    }
}

int ensure_slot(Slot &s, size_t bytes) {
    if (s.cap >= bytes) return GATLAS_OK;
    cudaFree(s.dev);
    cudaFreeHost(s.host);
    s.dev = s.host = nullptr;
    const size_t cap = std::max(bytes, s.cap * 2);
    if (cudaMalloc(&s.dev, cap) != cudaSuccess || cudaHostAlloc(&s.host, cap, cudaHostAllocDefault) != cudaSuccess) {
        cudaGetLastError();
        s.cap = 0;
        return set_error(GATLAS_ERR_NOMEM, "server: batch tables of %zu bytes", cap);
    }
    s.cap = cap;
    return GATLAS_OK;
}

// Host and device timelines share their origin: the start event is recorded
// and completed before the host clock starts, so a completion measured on the
// device from the start event is never earlier, on the host's clock, than the
// arrival it follows (latencies can only be overstated, by the microseconds
// the synchronisation takes to return).
int64_t start_clocks(Server &S) {
    cudaEventRecord(S.start, S.sg);
    cudaEventSynchronize(S.start);
    return now_ns();
}

int run_serial(Server &S, const gatlas_request *rq, int32_t count, gatlas_request_result *res) {
    const int64_t t0 = start_clocks(S);
    cudaEvent_t ev = S.get_event();
    for (int i = 0; i < count; ++i) {
        const gatlas_request &r = rq[i];
        wait_until(t0, r.arrival_ns);
        RState st;
        int rc = request_layout(S, r, 1, &st.L);
        if (!rc) {
            st.mem = S.arena.alloc(st.L.total);
            if (!st.mem) rc = set_error(GATLAS_ERR_NOMEM, "server: request %d needs %zu bytes", i, st.L.total);
        }
        res[i].admit_ns = now_ns() - t0;
        res[i].batch = -1;
        if (!rc) rc = generate(r, st.mem, st.L, S.sg);
        if (!rc) rc = launch_single(S, r, st.mem, st.L, S.sg);
        cudaEventRecord(ev, S.sg);
        cudaEventSynchronize(ev);
        res[i].done_ns = elapsed_ns(S, ev);
        res[i].start_ns = res[i].admit_ns;
        res[i].status = rc;
        finish(S, r, st, res[i]);
    }
    S.put_event(ev);
    return GATLAS_OK;
}

int run_continuous(Server &S, const gatlas_request *rq, int32_t count, gatlas_request_result *res) {
    struct Flight {
        cudaEvent_t ev;
        std::vector<int> reqs;
        int slot;  // table slot of a GEMM batch, -1 otherwise
    };
    std::vector<RState> st(count);
    std::deque<int> waiting;
    std::vector<int> ready_gemm, ready_mem;
    // work completes in launch order on each stream: harvest from the fronts
    std::deque<Flight> flights_g, flights_m;
    cudaEvent_t prep_ev = S.get_event();
    const int64_t t0 = start_clocks(S);
    int next = 0, done = 0, gemm_inflight = 0;
    int blocked_head = -1;
    uint64_t blocked_epoch = 0;
    const double est_rate = (S.cfg.gemm_tflops_estimate > 0 ? S.cfg.gemm_tflops_estimate : 300.0) * 1e12;
    const double target_s = (S.cfg.batch_target_ms > 0 ? S.cfg.batch_target_ms : 20.0) * 1e-3;
    const int max_batch = S.cfg.max_batch > 0 ? S.cfg.max_batch : 256;
    while (done < count) {
        bool progress = false;
        const int64_t now = now_ns() - t0;
        ++S.iterations;
        while (next < count && rq[next].arrival_ns <= now) waiting.push_back(next++);
        int64_t tp = now_ns();
        auto phase = [&](int i) {
            const int64_t t1 = now_ns();
            S.phase_ns[i] += t1 - tp;
            tp = t1;
        };
        // 1. harvest completed work
        for (std::deque<Flight> *fl : {&flights_g, &flights_m}) {
            while (!fl->empty()) {
                Flight &f = fl->front();
                const cudaError_t q = cudaEventQuery(f.ev);
                if (q == cudaErrorNotReady) break;
                const int64_t t = elapsed_ns(S, f.ev);
                for (int r : f.reqs) {
                    res[r].done_ns = t;
                    if (q != cudaSuccess && res[r].status == GATLAS_OK) res[r].status = GATLAS_ERR_CUDA;
                    finish(S, rq[r], st[r], res[r]);
                    ++done;
                }
                if (f.slot >= 0) {
                    S.slots[f.slot].busy = false;
                    --gemm_inflight;
                }
                S.put_event(f.ev);
                fl->pop_front();
                progress = true;
            }
        }
        phase(0);
        // 2. FIFO admission under the memory budget (a head that did not fit is
        // retried only after some memory was released)
        bool admitted = false;
        while (!waiting.empty()) {
            const bool idle = flights_g.empty() && flights_m.empty() && ready_gemm.empty();
            if (waiting.front() == blocked_head && S.arena.epoch() == blocked_epoch && !idle) break;
            const int r = waiting.front();
            RState &s = st[r];
            int rc = request_layout(S, rq[r], 0, &s.L);
            if (!rc && s.L.total > S.arena.size())
                rc = set_error(GATLAS_ERR_NOMEM, "server: request %d needs %zu bytes, budget %zu", r, s.L.total,
                               S.arena.size());
            if (rc) {
                res[r].status = rc;
                res[r].admit_ns = res[r].done_ns = now;
                waiting.pop_front();
                ++done;
                progress = true;
                continue;
            }
            s.mem = S.arena.alloc(s.L.total);
            if (!s.mem) {
                if (flights_g.empty() && flights_m.empty() && ready_gemm.empty()) {
                    // nothing on the device will free memory (retained results hold it)
                    res[r].status = set_error(GATLAS_ERR_NOMEM, "server: request %d does not fit beside the retained "
                                                                "results", r);
                    res[r].admit_ns = res[r].done_ns = now;
                    waiting.pop_front();
                    ++done;
                    progress = true;
                    continue;
                }
                blocked_head = r;
                blocked_epoch = S.arena.epoch();
                break;  // wait for memory; later arrivals do not overtake
            }
            waiting.pop_front();
            res[r].admit_ns = now;
            const int64_t g0 = now_ns();
            rc = generate(rq[r], s.mem, s.L, S.prep);
            S.generate_ns += now_ns() - g0;
            S.generate_launches += generate_launch_count(rq[r]);
            res[r].status = rc;
            if (rc) {
                res[r].done_ns = now;
                finish(S, rq[r], s, res[r]);
                ++done;
            } else if (rq[r].kind == GATLAS_REQ_GEMM) {
                ready_gemm.push_back(r);
            } else {
                ready_mem.push_back(r);
            }
            admitted = true;
            progress = true;
        }
        if (admitted) {
            cudaEventRecord(prep_ev, S.prep);
            cudaStreamWaitEvent(S.sg, prep_ev, 0);
            cudaStreamWaitEvent(S.sm, prep_ev, 0);
        }
        phase(1);
        // 3. memory-bound requests run as admitted, beside the GEMM batches
        for (int r : ready_mem) {
            res[r].start_ns = now;
            res[r].batch = -1;
            const int rc = launch_single(S, rq[r], st[r].mem, st[r].L, S.sm);
            if (rc) res[r].status = rc;
            Flight f{S.get_event(), {r}, -1};
            cudaEventRecord(f.ev, S.sm);
            flights_m.push_back(std::move(f));
        }
        ready_mem.clear();
        phase(2);
        // 4. next GEMM batch while fewer than two are on the device
        if (!ready_gemm.empty() && gemm_inflight < 2) {
            int slot = S.slots[0].busy ? 1 : 0;
            size_t take = 0;
            double est = 0.0;
            while (take < ready_gemm.size() && (int)take < max_batch && (take == 0 || est < target_s)) {
                // BF16 runs one product where split3 runs three
                est += request_flops(rq[ready_gemm[take]]) * (S.cfg.gemm_engine == GATLAS_ENGINE_TC_SPLIT3 ? 1.0 : 1.0 / 3) /
                       est_rate;
                ++take;
            }
            std::vector<gatlas_grouped_instance> inst(take);
            std::vector<uint8_t *> packed(take);
            std::vector<int> ids(ready_gemm.begin(), ready_gemm.begin() + take);
            for (size_t j = 0; j < take; ++j) {
                const gatlas_request &r = rq[ids[j]];
                const RState &s = st[ids[j]];
                gatlas_grouped_instance &q = inst[j];
                std::memset(&q, 0, sizeof(q));
                q.a = reinterpret_cast<const float *>(s.mem + s.L.a);
                q.b = reinterpret_cast<const float *>(s.mem + s.L.b);
                q.c = reinterpret_cast<float *>(s.mem + s.L.c);
                q.m = r.m, q.n = r.n, q.k = r.k, q.trans_a = r.trans_a, q.trans_b = r.trans_b;
                q.gemm = 1, q.alpha = r.alpha, q.beta = r.beta;
                packed[j] = s.mem + s.L.ws;
            }
            GroupedTables t;
            int rc = grouped_build(S.cfg.gemm_engine, inst.data(), (int32_t)take, nullptr, packed.data(), &t);
            const size_t tb = rc ? 0 : grouped_tables_bytes(t);
            if (!rc) rc = ensure_slot(S.slots[slot], tb);
            if (!rc) {
                grouped_tables_serialise(t, S.slots[slot].host);
                if (cudaMemcpyAsync(S.slots[slot].dev, S.slots[slot].host, tb, cudaMemcpyHostToDevice, S.sg) !=
                    cudaSuccess)
                    rc = set_error(GATLAS_ERR_CUDA, "server: table upload");
            }
            phase(3);
            const GroupedDevice d = grouped_tables_device(t, S.slots[slot].dev);
            if (!rc) rc = grouped_launch_pack(t, d, S.sg);
            if (!rc) rc = grouped_launch_contract(t, d, S.sg);
            Flight f{S.get_event(), ids, slot};
            cudaEventRecord(f.ev, S.sg);
            for (int r : ids) {
                res[r].start_ns = now;
                res[r].batch = (int32_t)S.batches;
                if (rc) res[r].status = rc;
            }
            S.slots[slot].busy = true;
            ++gemm_inflight;
            ++S.batches;
            S.batched_gemms += (int64_t)take;
            flights_g.push_back(std::move(f));
            ready_gemm.erase(ready_gemm.begin(), ready_gemm.begin() + take);
            progress = true;
            phase(4);
        }
        if (progress) S.host_busy_ns += now_ns() - t0 - now;
        if (!progress) {
            // nothing changed: wait a little for the device or the next arrival
            const int64_t nxt = next < count ? rq[next].arrival_ns - (now_ns() - t0) : INT64_MAX;
            if (flights_g.empty() && flights_m.empty() && next < count && nxt > 200000)
                wait_until(t0, rq[next].arrival_ns);
            else std::this_thread::yield();
        }
    }
    S.put_event(prep_ev);
    cudaStreamSynchronize(S.prep);
    return GATLAS_OK;
}

}  // namespace

}  // namespace gatlas

extern "C" {

int gatlas_server_create(const gatlas_server_config *cfg, gatlas_server **out) {
    using namespace gatlas;
    clear_error();
    if (!cfg || !out) return set_error(GATLAS_ERR_INVALID, "server: null argument");
    *out = nullptr;
    if (cfg->gemm_engine != GATLAS_ENGINE_TC_SPLIT3 && cfg->gemm_engine != GATLAS_ENGINE_TC_BF16)
        return set_error(GATLAS_ERR_UNSUPPORTED, "server: GEMM engine %d has no grouped kernel", cfg->gemm_engine);
    if (cfg->budget_bytes < kAlign) return set_error(GATLAS_ERR_INVALID, "server: budget below %zu bytes", kAlign);
    Server *S = new Server();
    S->cfg = *cfg;
    cudaGetDevice(&S->device);
    int rc = S->arena.init(cfg->budget_bytes);
    if (!rc && (cudaStreamCreateWithFlags(&S->prep, cudaStreamNonBlocking) != cudaSuccess ||
                cudaStreamCreateWithFlags(&S->sg, cudaStreamNonBlocking) != cudaSuccess ||
                cudaStreamCreateWithFlags(&S->sm, cudaStreamNonBlocking) != cudaSuccess ||
                cudaEventCreate(&S->start) != cudaSuccess))
        rc = set_error(GATLAS_ERR_CUDA, "server: streams");
    // table slots sized for a few thousand tiles up front, so that the first
    // batches do not pay for device and pinned allocations
    for (Slot &sl : S->slots)
        if (!rc) rc = ensure_slot(sl, 8u << 20);
    if (rc) {
        delete S;
        return rc;
    }
    *out = reinterpret_cast<gatlas_server *>(S);
    return GATLAS_OK;
}

int gatlas_server_run(gatlas_server *srv, const gatlas_request *reqs, int32_t count, int32_t mode,
                      gatlas_request_result *results) {
    using namespace gatlas;
    clear_error();
    if (!srv || (count > 0 && (!reqs || !results)) || count < 0)
        return set_error(GATLAS_ERR_INVALID, "server: invalid run arguments");
    for (int i = 1; i < count; ++i)
        if (reqs[i].arrival_ns < reqs[i - 1].arrival_ns)
            return set_error(GATLAS_ERR_INVALID, "server: arrivals must be non-decreasing");
    Server &S = *reinterpret_cast<Server *>(srv);
    for (int i = 0; i < count; ++i) {
        std::memset(&results[i], 0, sizeof(results[i]));
        results[i].batch = -1;
    }
    if (mode == GATLAS_SERVE_SERIAL) return run_serial(S, reqs, count, results);
    if (mode == GATLAS_SERVE_CONTINUOUS) return run_continuous(S, reqs, count, results);
    return set_error(GATLAS_ERR_INVALID, "server: unknown mode %d", mode);
}

int gatlas_server_release(gatlas_server *srv, float *result) {
    using namespace gatlas;
    clear_error();
    if (!srv) return set_error(GATLAS_ERR_INVALID, "server: null server");
    Server &S = *reinterpret_cast<Server *>(srv);
    auto it = S.retained.find(result);
    if (it == S.retained.end()) return set_error(GATLAS_ERR_INVALID, "server: not a retained result");
    S.arena.release(it->second.first, it->second.second);
    S.retained.erase(it);
    return GATLAS_OK;
}

int gatlas_server_read(gatlas_server *srv, const float *result, float *host_dst, int64_t elems) {
    using namespace gatlas;
    clear_error();
    if (!srv || !host_dst || elems < 0) return set_error(GATLAS_ERR_INVALID, "server: invalid read arguments");
    Server &S = *reinterpret_cast<Server *>(srv);
    if (!S.retained.count(const_cast<float *>(result))) return set_error(GATLAS_ERR_INVALID, "server: not a retained result");
    if (cudaMemcpy(host_dst, result, (size_t)elems * 4, cudaMemcpyDeviceToHost) != cudaSuccess)
        return set_error(GATLAS_ERR_CUDA, "server: result copy");
    return GATLAS_OK;
}

int gatlas_server_stats(const gatlas_server *srv, gatlas_server_stats_t *out) {
    using namespace gatlas;
    clear_error();
    if (!srv || !out) return set_error(GATLAS_ERR_INVALID, "server: null argument");
    const Server &S = *reinterpret_cast<const Server *>(srv);
    out->budget_bytes = S.arena.size();
    out->peak_bytes = S.arena.peak();
    out->used_bytes = S.arena.used();
    out->gemm_batches = S.batches;
    out->batched_gemms = S.batched_gemms;
    out->host_busy_ns = S.host_busy_ns;
    out->iterations = S.iterations;
    for (int i = 0; i < 5; ++i) out->phase_ns[i] = S.phase_ns[i];
    out->generate_ns = S.generate_ns;
    out->generate_launches = S.generate_launches;
    return GATLAS_OK;
}

void gatlas_server_destroy(gatlas_server *srv) { delete reinterpret_cast<gatlas::Server *>(srv); }

}  // extern "C"

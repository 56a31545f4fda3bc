// Work-group scheduler for the reference's generated kernels on the host CPU.
//
// TEST INFRASTRUCTURE (see clshim.hpp).  Work groups run in parallel over the
// host's cores (OpenMP, one group per thread at a time); the work items of a
// group run one after another on that thread.  A kernel with barrier() runs
// its work items as fibers: each runs until its next barrier, then the next
// item runs, so every item of the group reaches a barrier before any passes
// it.  Local memory is one buffer per __local argument per thread, reused by
// every group that thread runs.
#include <omp.h>
#include <stdlib.h>

#include <vector>

#include "clshim.hpp"
#include "refk.h"

namespace clshim {

thread_local WorkItem *tl_item = nullptr;
thread_local GroupScheduler *tl_group = nullptr;

namespace {

thread_local refk_body tl_body = nullptr;
thread_local void *tl_arg = nullptr;
thread_local void *tl_local[2] = {nullptr, nullptr};

void trampoline() {
    tl_body(tl_arg, tl_local[0], tl_local[1]);
    tl_item->done = 1;  // returning resumes the scheduler (uc_link)
}

constexpr size_t kStackBytes = 64 * 1024;

}  // namespace
}  // namespace clshim

extern "C" int refk_run_groups(const refk_launch *L, refk_body body, void *arg) {
    using namespace clshim;
    size_t gb[2], ge[2], ngroups[2];
    for (int d = 0; d < 2; ++d) {
        if (L->local[d] == 0 || L->global[d] % L->local[d]) return -1;
        ngroups[d] = L->global[d] / L->local[d];
        gb[d] = L->group_begin[d];
        ge[d] = L->group_end[d] ? L->group_end[d] : ngroups[d];
        if (gb[d] > ge[d] || ge[d] > ngroups[d]) return -1;
    }
    const size_t span0 = ge[0] - gb[0], span1 = ge[1] - gb[1];
    const long total = (long)(span0 * span1);
    const size_t items = L->local[0] * L->local[1];
    const int threads = L->threads > 0 ? L->threads : omp_get_max_threads();
    int failed = 0;
#pragma omp parallel num_threads(threads)
    {
        std::vector<unsigned char> local0(L->local_bytes[0] + 64), local1(L->local_bytes[1] + 64);
        std::vector<WorkItem> wi(items);
        std::vector<unsigned char> stacks;
        if (L->uses_barrier) stacks.resize(items * kStackBytes);
        GroupScheduler group;
        tl_group = &group;
        tl_body = body;
        tl_arg = arg;
        tl_local[0] = L->local_bytes[0] ? local0.data() : nullptr;
        tl_local[1] = L->local_bytes[1] ? local1.data() : nullptr;
#pragma omp for schedule(dynamic, 1)
        for (long g = 0; g < total; ++g) {
            const size_t grp[2] = {gb[0] + (size_t)g % span0, gb[1] + (size_t)g / span0};
            for (size_t i = 0; i < items; ++i) {
                WorkItem &w = wi[i];
                const size_t lid[2] = {i % L->local[0], i / L->local[0]};
                for (int d = 0; d < 2; ++d) {
                    w.local_id[d] = lid[d];
                    w.group_id[d] = grp[d];
                    w.global_id[d] = grp[d] * L->local[d] + lid[d];
                    w.local_size[d] = L->local[d];
                    w.global_size[d] = L->global[d];
                }
                w.done = 0;
            }
            if (!L->uses_barrier) {
                for (size_t i = 0; i < items; ++i) {
                    tl_item = &wi[i];
                    body(arg, tl_local[0], tl_local[1]);
                }
                continue;
            }
            for (size_t i = 0; i < items; ++i) {
                WorkItem &w = wi[i];
                if (getcontext(&w.ctx) != 0) {
#pragma omp atomic write
                    failed = 1;
                    continue;
                }
                w.ctx.uc_stack.ss_sp = stacks.data() + i * kStackBytes;
                w.ctx.uc_stack.ss_size = kStackBytes;
                w.ctx.uc_link = &group.sched;
                makecontext(&w.ctx, trampoline, 0);
            }
            // every pass runs each unfinished item up to its next barrier
            for (bool pending = true; pending;) {
                pending = false;
                for (size_t i = 0; i < items; ++i) {
                    if (wi[i].done) continue;
                    tl_item = &wi[i];
                    swapcontext(&group.sched, &wi[i].ctx);
                    if (!wi[i].done) pending = true;
                }
            }
        }
    }
    return failed ? -1 : 0;
}

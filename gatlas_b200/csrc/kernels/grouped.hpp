// Grouped tensor-core matmul (grouped.cu): internal interface.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include "../status.hpp"

namespace gatlas {

constexpr int kGroupedBuckets = GATLAS_GROUPED_BUCKETS;

struct GroupedPlan;

int32_t grouped_bucket(int64_t m, int64_t n, int64_t k);
int grouped_set_tile_table(int engine, const int32_t *t, int32_t nb);
int grouped_get_tile_table(int engine, int32_t *t, int32_t nb);
size_t grouped_workspace_bytes(int engine, const gatlas_grouped_instance *in, int32_t count);
int grouped_create(int engine, const gatlas_grouped_instance *in, int32_t count, void *ws, size_t ws_bytes,
                   GroupedPlan **out);
int grouped_prepare(GroupedPlan *p, cudaStream_t stream);
int grouped_run(GroupedPlan *p, cudaStream_t stream);
int grouped_launch_graph(GroupedPlan *p, int with_prepare, cudaStream_t stream);
int grouped_run_each(GroupedPlan *p, cudaStream_t stream);
int grouped_info(const GroupedPlan *p, int64_t *tiles, int32_t *ctas, double *flops, int64_t *items);
void grouped_destroy(GroupedPlan *p);

}  // namespace gatlas

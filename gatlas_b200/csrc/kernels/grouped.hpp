// Grouped tensor-core matmul (grouped.cu): internal interface.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include "../status.hpp"

#include <vector>

namespace gatlas {

constexpr int kGroupedBuckets = GATLAS_GROUPED_BUCKETS;

namespace grp {

// Per-instance device record.
struct Inst {
    const float *src_a, *src_b;
    uint8_t *pa[2], *pb[2];  // packed pieces
    float *C;
    int64_t M, N, K, lda, ldb, ldc;
    int32_t ta, tb, gemm, bn, mt, nt, kt, pad;  // kt: pack items (64 K elements) per row block
    float alpha, beta;
};

// Self-contained record of one output tile, in the order its CTA runs it:
// the producer, the MMA issuer and the epilogue read nothing else.
struct TileRec {
    const uint8_t *a[2];  // piece tiles of this row block: [kt][128 rows x one K slice]
    const uint8_t *b[2];  // piece tiles of this column block: [kt][bn rows x one K slice]
    float *C;             // C at the tile's origin
    int64_t ldc;
    int32_t kt, bn, rows, cols;  // K slices; tile width; valid rows / columns of the tile
    float alpha, beta;
    int32_t gemm, pad;
};
static_assert(sizeof(TileRec) == 80, "tile record layout");

}  // namespace grp

// Resolved geometry of one instance.
struct InstPlan {
    int64_t M, N, K, lda, ldb, ldc;
    int bn, mt, nt, kt;
    size_t a_piece, b_piece;  // bytes per piece
};

// Host tables of one group: instance records and pack segments (pack pass),
// output tile records in CTA order and each CTA's range (contraction).
struct GroupedTables {
    int engine = 0, np = 1, mode = 0;
    bool pair = false;  // 256-row tiles on CTA pairs; `grid` and `cta` count clusters
    bool vec = false;   // every instance's C takes 8-byte vector accesses
    std::vector<InstPlan> ip;
    std::vector<grp::Inst> inst;
    std::vector<int64_t> seg;
    std::vector<grp::TileRec> tiles;
    std::vector<int32_t> cta;
    int grid = 0, nseg = 0;
    int64_t nitems = 0, ntiles = 0;
    double flops = 0;
    size_t packed_bytes = 0;
};

// Device copies of the tables.
struct GroupedDevice {
    const grp::Inst *inst = nullptr;
    const int64_t *seg = nullptr;
    const grp::TileRec *tiles = nullptr;
    const int32_t *cta = nullptr;
};

// Packed bytes of one instance for the engine (0 and an error on invalid input).
int grouped_instance_bytes(int engine, const gatlas_grouped_instance &in, size_t *bytes);
// Builds the tables.  Instance i's packed pieces start at packed[i] when
// `packed` is given, otherwise consecutively from `base` (1024-byte aligned).
int grouped_build(int engine, const gatlas_grouped_instance *in, int32_t count, uint8_t *base,
                  uint8_t *const *packed, GroupedTables *t);
// Pack pass and contraction over device tables.
int grouped_launch_pack(const GroupedTables &t, const GroupedDevice &d, cudaStream_t stream);
int grouped_launch_contract(const GroupedTables &t, const GroupedDevice &d, cudaStream_t stream);
// The tables as one device image: bytes, host serialisation, device views.
size_t grouped_tables_bytes(const GroupedTables &t);
void grouped_tables_serialise(const GroupedTables &t, void *host_dst);
GroupedDevice grouped_tables_device(const GroupedTables &t, const void *dev_base);

struct GroupedPlan;

int32_t grouped_bucket(int64_t m, int64_t n, int64_t k);
// Tiling of grouped contractions: 0 128-row tiles on single CTAs (the
// default), 1 256-row tiles on CTA pairs.
int grouped_set_pair(int mode);
int grouped_get_pair();
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

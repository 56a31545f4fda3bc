// SIMT SGEMM instantiations, no transposes: the tuning grid work group
// {8,16}x{8,16} x inner blocking {4,8}x{4,8} x vector width {1,2,4}
// (part a of 2; split for parallel compilation).
#include "gemm_simt_inst.cuh"

#define E(GH, GW, BH, BW, VL) GATLAS_SIMT_ENTRY(float, 0, 0, 0, GH, GW, BH, BW, VL)
#define ROW_VL(GH, GW, BH, BW) E(GH, GW, BH, BW, 1), E(GH, GW, BH, BW, 2), E(GH, GW, BH, BW, 4)
#define ROW_B(GH, GW) ROW_VL(GH, GW, 4, 4), ROW_VL(GH, GW, 4, 8), ROW_VL(GH, GW, 8, 4), ROW_VL(GH, GW, 8, 8)

namespace gatlas {
namespace simt {

static const Entry kTable[] = {ROW_B(8, 8), ROW_B(8, 16)};

const Entry *table_f32_nn_a(size_t *n) {
    *n = sizeof(kTable) / sizeof(kTable[0]);
    return kTable;
}

}  // namespace simt
}  // namespace gatlas

// SIMT SGEMM instantiations for the transposed layouts (A^T B, A B^T, A^T B^T).
#include "gemm_simt_inst.cuh"

#define E(TA, TB, GH, GW, BH, BW, VL) GATLAS_SIMT_ENTRY(float, 0, TA, TB, GH, GW, BH, BW, VL)
#define POINTS(TA, TB) E(TA, TB, 16, 16, 8, 8, 4), E(TA, TB, 16, 16, 4, 4, 4), \
                       E(TA, TB, 16, 16, 8, 8, 1), E(TA, TB, 8, 8, 8, 8, 4)

namespace gatlas {
namespace simt {

static const Entry kTable[] = {POINTS(0, 1), POINTS(1, 0), POINTS(1, 1)};

const Entry *table_f32_tx(size_t *n) {
    *n = sizeof(kTable) / sizeof(kTable[0]);
    return kTable;
}

}  // namespace simt
}  // namespace gatlas

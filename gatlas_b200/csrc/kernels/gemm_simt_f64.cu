// SIMT DGEMM instantiations (all four layouts).
#include "gemm_simt_inst.cuh"

#define E(TA, TB, GH, GW, BH, BW, VL) GATLAS_SIMT_ENTRY(double, 1, TA, TB, GH, GW, BH, BW, VL)
// 8 x 16 threads with 8 x 8 doubles each is the fastest measured point on
// B200 (20.3 TFLOP/s at 4096^3, against 12.5 for 16 x 16 x 8 x 4) and the
// default for double.
#define POINTS(TA, TB) E(TA, TB, 16, 16, 4, 4, 2), E(TA, TB, 16, 16, 4, 4, 1), \
                       E(TA, TB, 16, 16, 8, 4, 2), E(TA, TB, 16, 16, 8, 8, 2), \
                       E(TA, TB, 8, 16, 8, 8, 2), E(TA, TB, 16, 8, 8, 8, 2), E(TA, TB, 8, 8, 8, 8, 2)

namespace gatlas {
namespace simt {

static const Entry kTable[] = {POINTS(0, 0), POINTS(0, 1), POINTS(1, 0), POINTS(1, 1)};

const Entry *table_f64(size_t *n) {
    *n = sizeof(kTable) / sizeof(kTable[0]);
    return kTable;
}

}  // namespace simt
}  // namespace gatlas

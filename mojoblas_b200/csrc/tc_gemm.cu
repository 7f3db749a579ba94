// Tensor-core (tcgen05) GEMM paths — placeholder until the kernels land.
#include "mbg_internal.cuh"

namespace mbg {

int sgemm_split_tc(int, char, char, i64, i64, i64, float, const float*, i64, const float*, i64,
                   float, float*, i64, char) {
    set_error_msg("split-precision sgemm is not built yet");
    return MBG_ERR_UNSUPPORTED;
}
int dgemm_ozaki_tc(int, char, char, i64, i64, i64, double, const double*, i64, const double*, i64,
                   double, double*, i64) {
    set_error_msg("Ozaki dgemm is not built yet");
    return MBG_ERR_UNSUPPORTED;
}

}  // namespace mbg

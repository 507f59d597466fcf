// trace_ks_mixed.cu — the mixed-precision Kerr-Schild trace kernels (FP32
// dual-number right-hand side, FP64 state, projection and island), one per
// register budget and launch form.
#include "tracer.cuh"

namespace sirius {
namespace eng {

TraceFn pick_ks_mixed(int minb, bool uni) {
    constexpr int KS = SIRIUS_METRIC_KERR_SCHILD;
    if (uni) {
        switch (minb) {
            case 3: return trace_kernel<true, 3, KS, true>;
            case 4: return trace_kernel<true, 4, KS, true>;
            default: return trace_kernel<true, 2, KS, true>;
        }
    }
    switch (minb) {
        case 3: return trace_kernel<true, 3, KS, false>;
        case 4: return trace_kernel<true, 4, KS, false>;
        default: return trace_kernel<true, 2, KS, false>;
    }
}

}  // namespace eng
}  // namespace sirius

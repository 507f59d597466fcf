// trace_ks_fp64.cu — the all-FP64 Kerr-Schild trace kernels (the plain FP64
// GPU integrator), one per register budget and launch form.
#include "tracer.cuh"

namespace sirius {
namespace eng {

TraceFn pick_ks_fp64(int minb, bool uni) {
    constexpr int KS = SIRIUS_METRIC_KERR_SCHILD;
    if (uni) {
        switch (minb) {
            case 3: return trace_kernel<false, 3, KS, true>;
            case 4: return trace_kernel<false, 4, KS, true>;
            default: return trace_kernel<false, 2, KS, true>;
        }
    }
    switch (minb) {
        case 3: return trace_kernel<false, 3, KS, false>;
        case 4: return trace_kernel<false, 4, KS, false>;
        default: return trace_kernel<false, 2, KS, false>;
    }
}

}  // namespace eng
}  // namespace sirius

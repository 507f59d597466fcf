// trace_ks_fp64.cu — the all-FP64 Kerr-Schild trace kernels (the plain FP64
// GPU integrator), one per register budget and launch form.
#include "tracer.cuh"

namespace sirius {
namespace eng {

template <int INT>
TraceFn pick_budget(int minb, bool uni) {
    constexpr int KS = SIRIUS_METRIC_KERR_SCHILD;
    if (uni) {
        switch (minb) {
            case 3: return trace_kernel<false, 3, KS, true, INT>;
            case 4: return trace_kernel<false, 4, KS, true, INT>;
            default: return trace_kernel<false, 2, KS, true, INT>;
        }
    }
    switch (minb) {
        case 3: return trace_kernel<false, 3, KS, false, INT>;
        case 4: return trace_kernel<false, 4, KS, false, INT>;
        default: return trace_kernel<false, 2, KS, false, INT>;
    }
}

TraceFn pick_ks_fp64(int minb, bool uni, bool symp) {
    return symp ? pick_budget<SIRIUS_INTEGRATOR_SYMPLECTIC>(minb, uni) : pick_budget<SIRIUS_INTEGRATOR_DP45>(minb, uni);
}

}  // namespace eng
}  // namespace sirius

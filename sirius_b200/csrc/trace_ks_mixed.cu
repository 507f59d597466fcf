// trace_ks_mixed.cu — the mixed-precision Kerr-Schild trace kernels (FP32
// dual-number right-hand side, FP64 state, projection and island), one per
// register budget and launch form, with one ray per thread (tracer.cuh) or two
// rays per thread in packed FP32 pairs (tracer_pair.cuh).
#include "tracer_pair.cuh"

namespace sirius {
namespace eng {

template <int INT>
TraceFn pick_budget(int minb, bool uni) {
    constexpr int KS = SIRIUS_METRIC_KERR_SCHILD;
    if (uni) {
        switch (minb) {
            case 3: return trace_kernel<true, 3, KS, true, INT>;
            case 4: return trace_kernel<true, 4, KS, true, INT>;
            default: return trace_kernel<true, 2, KS, true, INT>;
        }
    }
    switch (minb) {
        case 3: return trace_kernel<true, 3, KS, false, INT>;
        case 4: return trace_kernel<true, 4, KS, false, INT>;
        default: return trace_kernel<true, 2, KS, false, INT>;
    }
}

TraceFn pick_ks_mixed(int minb, bool uni, bool symp) {
    return symp ? pick_budget<SIRIUS_INTEGRATOR_SYMPLECTIC>(minb, uni) : pick_budget<SIRIUS_INTEGRATOR_DP45>(minb, uni);
}

TraceFn pick_ks_mixed_pair(int minb, bool uni) {
    if (uni) return minb == 3 ? trace_pair_kernel<3, true> : trace_pair_kernel<2, true>;
    return minb == 3 ? trace_pair_kernel<3, false> : trace_pair_kernel<2, false>;
}

}  // namespace eng
}  // namespace sirius

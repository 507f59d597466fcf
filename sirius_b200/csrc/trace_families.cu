// trace_families.cu — the trace kernels of the Morris-Thorne and Alcubierre
// families, and the generic kernel that dispatches on each ray's family (the
// persistent queue over a heterogeneous batch).
#include "tracer.cuh"

namespace sirius {
namespace eng {

TraceFn pick_family(bool mixed, int fam) {
    switch (fam) {
        case SIRIUS_METRIC_MORRIS_THORNE:
            return mixed ? trace_kernel<true, 2, SIRIUS_METRIC_MORRIS_THORNE, false, kAnyIntegrator>
                         : trace_kernel<false, 2, SIRIUS_METRIC_MORRIS_THORNE, false, kAnyIntegrator>;
        case SIRIUS_METRIC_ALCUBIERRE:
            return mixed ? trace_kernel<true, 2, SIRIUS_METRIC_ALCUBIERRE, false, kAnyIntegrator>
                         : trace_kernel<false, 2, SIRIUS_METRIC_ALCUBIERRE, false, kAnyIntegrator>;
        default:
            return mixed ? trace_kernel<true, 2, kAnyFamily, false, kAnyIntegrator> : trace_kernel<false, 2, kAnyFamily, false, kAnyIntegrator>;
    }
}

}  // namespace eng
}  // namespace sirius

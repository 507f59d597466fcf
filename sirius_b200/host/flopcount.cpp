// flopcount.cpp — sirius_cuda_flop_count (include/sirius_cuda.h): the
// algorithmic operation count of the kernels' own formulation, obtained by
// instantiating the device metric templates on the host with a counting scalar.
// Host-only translation unit; no device is needed.
#include "../csrc/flopcount.h"
#include "../csrc/spacetime.cuh"

using namespace sirius;

extern "C" {

// Operations of one DP45 attempt besides its six right-hand sides, as written in
// dp45_attempt(): stage points sum_{s=2..6} 8 (2s - 1) = 280, the fifth-order
// combination 8 x 9 = 72 and its FP64 accumulation 8 x 2 = 16, the error
// estimate 4 x 11 + 4 x 5 + 2 = 66.
static constexpr double kStageAlgebraFlops = 280 + 72 + 16 + 66;
// FP64 constraint re-projection of an accepted step: inv_form (46) and
// project_null (3 bilinear forms of 24, the root and the update: 90).
static constexpr double kProjectionFlops = 136;

int sirius_cuda_flop_count(const sirius_metric* metric, double* rhs_flops, double* attempt_flops,
                           double* accepted_step_flops) {
    if (!metric || !rhs_flops || !attempt_flops || !accepted_step_flops) return SIRIUS_ERR_INVALID_ARGUMENT;
    if (metric->family < 0 || metric->family > 2) return SIRIUS_ERR_INVALID_ARGUMENT;
    const MetricDev m = metric_dev(*metric);
    Counted x[4], p[4], k[4], f[4];
    // a generic point off the symmetry planes and a generic covector
    const double xv[4] = {0.0, 7.1, -3.3, 2.9}, pv[4] = {-1.0, 0.3, -0.6, 0.2};
    for (int i = 0; i < 4; ++i) { x[i] = xv[i]; p[i] = pv[i]; }
    if (m.family == SIRIUS_METRIC_MORRIS_THORNE) { x[1] = 8.0; x[2] = 1.1; x[3] = 0.4; }
    FlopCounter::n() = 0;
    rhs<Counted>(m, x, p, k, f);
    const double c = double(FlopCounter::n());
    *rhs_flops = c;
    *attempt_flops = 6.0 * c + kStageAlgebraFlops;
    *accepted_step_flops = *attempt_flops + kProjectionFlops;
    return SIRIUS_OK;
}

}  // extern "C"

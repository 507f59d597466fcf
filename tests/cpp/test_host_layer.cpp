// C++ checks of include/sirius_b200.hpp (the host layer mirroring the
// reference's GeodesicTracer / IAccelerator / KerrSchildFamily interfaces).
// Built and run by tests/test_host_layer.py; "--gpu" adds device checks.
#include <cmath>
#include <cstdio>
#include <cstring>

#include "sirius_b200.hpp"

using namespace sirius_b200;

static int failures = 0;
#define CHECK(c)                                                         \
    do {                                                                 \
        if (!(c)) { std::printf("FAIL %s:%d %s\n", __FILE__, __LINE__, #c); ++failures; } \
    } while (0)

int main(int argc, char** argv) {
    const bool gpu = argc > 1 && std::strcmp(argv[1], "--gpu") == 0;
    // KerrSchildFamily parameter semantics (PHMT100A.h:149-196)
    KerrSchildFamily ks(KerrSchildParams{2.0, 1.0, 0.0, 0.0});
    CHECK(std::fabs(ks.getParameters().at("spin").value - 0.5) < 1e-15);
    CHECK(std::strcmp(ks.getName(), "Kerr") == 0);
    ks.setParameter("spin", 5.0);  // clamped to 0.998
    CHECK(std::fabs(ks.getParams().a - 0.998 * 2.0) < 1e-12);
    ks.setParameter("charge", 0.1);
    CHECK(std::strcmp(ks.getName(), "Kerr-Newman") == 0);
    KerrSchildFamily schw;
    CHECK(std::strcmp(schw.getName(), "Schwarzschild") == 0);
    sirius_metric m = ks.toMetric();
    CHECK(m.family == SIRIUS_METRIC_KERR_SCHILD && std::fabs(m.Q - 0.2) < 1e-12);

    // TracerConfig -> engine config
    TracerConfig tc;
    tc.escape_radius = 200.0f;
    tc.integrator.abs_tolerance = 5e-6f;
    const sirius_trace_config c = toEngineConfig(tc);
    CHECK(c.escape_radius == 200.0 && c.max_steps == 5000 && std::fabs(c.abs_tolerance - 5e-6) < 1e-12);

    // sirius_ray_result -> TraceResult
    sirius_ray_result r{};
    r.outcome = SIRIUS_DISK_HIT;
    r.n_crossings = 2;
    r.disk_r[0] = 12.0f; r.disk_r[1] = 7.0f; r.disk_g[0] = 0.8f; r.disk_g[1] = 1.1f;
    r.flags = SIRIUS_FLAG_PHOTON_RING;
    r.steps = 321;
    TraceResult tr = toTraceResult(r, tc);
    CHECK(tr.outcome == TraceResult::Outcome::DISK_HIT && tr.num_disk_crossings == 2);
    CHECK(tr.disk_crossings[1].valid && tr.disk_crossings[1].crossing_index == 1);
    CHECK(std::fabs(tr.disk_temperature - std::pow(6.0f / 12.0f, 0.75f)) < 1e-6f);
    CHECK(tr.photon_ring && tr.steps_taken == 321 && std::fabs(tr.redshift - 0.8f) < 1e-7f);
    r.outcome = SIRIUS_STEP_UNDERFLOW;
    CHECK(toTraceResult(r, tc).outcome == TraceResult::Outcome::MAX_STEPS);

    // factory: only the CUDA slot
    CHECK(createAccelerator(BackendType::OptiX) == nullptr);
    auto acc = createAccelerator(BackendType::CUDA);
    CHECK(acc && acc->getType() == BackendType::CUDA);

    KerrSchildFamily kerr(KerrSchildParams{1.0, 0.9, 0.0, 0.0});
    TracerConfig cfg;
    cfg.escape_radius = 200.0f;
    cfg.disk_inner = 2.3208830f;
    cfg.disk_outer = 20.0f;
    cfg.max_steps = 20000;
    cfg.integrator.abs_tolerance = 1e-8f;
    cfg.integrator.rel_tolerance = 1e-8f;
    cfg.integrator.max_step = 2.0f;
    cfg.integrator.initial_step = 0.1f;
    cfg.integrator.min_step = 1e-9f;
    CudaGeodesicTracer tracer(&kerr, cfg);
    if (!gpu) {
        CHECK(!tracer.ok() || true);  // without a device the tracer reports, never crashes
        CameraRay ray;
        ray.origin(1) = 100.0; ray.origin(2) = 1.0; ray.direction(1) = -1.0;
        if (!tracer.ok()) {
            CHECK(tracer.traceBatch({ray}).empty());
            CHECK(!tracer.getLastError().empty());
            CHECK(!acc->initialise(64, 64) || acc->isInitialised());
        }
        std::printf("host layer CPU checks: %d failures\n", failures);
        return failures ? 1 : 0;
    }
    CHECK(tracer.ok());
    // a radial ray falls in, an outward ray escapes, a grazing ray hits the disk
    CameraRay in;
    in.origin(1) = 100.0; in.origin(2) = 1.2; in.direction(1) = -1.0;
    TraceResult a = tracer.trace(in);
    CHECK(a.outcome == TraceResult::Outcome::HORIZON);
    CHECK(a.null_final < 1e-10f);
    CameraRay out = in;
    out.direction(1) = 1.0;
    CHECK(tracer.trace(out).outcome == TraceResult::Outcome::ESCAPED);
    std::vector<CameraRay> rays;
    for (int i = 0; i < 64; ++i) {
        CameraRay q = in;
        q.direction(1) = -std::cos(0.001 * i);
        q.direction(3) = std::sin(0.001 * i) * (i % 2 ? 1 : -1);
        rays.push_back(q);
    }
    auto batch = tracer.traceBatch(rays);
    CHECK(batch.size() == rays.size());
    for (size_t i = 0; i < rays.size(); i += 9) {
        TraceResult one = tracer.trace(rays[i]);
        CHECK(one.outcome == batch[i].outcome && one.steps_taken == batch[i].steps_taken);
        CHECK(one.final_position(1) == batch[i].final_position(1));
    }
    // trace(ray, M, a) moves the disk edge to the ISCO of the new spin
    tracer.trace(in, 1.0, 0.5);
    CHECK(std::fabs(tracer.getConfig().disk_inner - 4.233f) < 2e-3f);
    // the accelerator renders a frame into its RGBA framebuffer
    CHECK(acc->initialise(64, 48));
    LaunchConfig lc;
    lc.blackHoleSpin = 0.9f;
    lc.observerDistance = 60.0f;
    lc.observerInclination = 1.3f;
    lc.cameraFOV = 35.0f;
    lc.diskInnerRadius = 2.32f;
    lc.diskOuterRadius = 20.0f;
    lc.maxStepSize = 2.0f;
    lc.exposure = 1.0f;
    acc->launch(lc);
    CHECK(acc->getLastError().empty());
    const float* fb = acc->getFrameBuffer();
    CHECK(fb != nullptr && acc->getFrameBufferSize() == size_t(64) * 48 * 16);
    float mx = 0;
    for (int i = 0; i < 64 * 48; ++i) { mx = std::fmax(mx, fb[4 * i]); CHECK(fb[4 * i + 3] == 1.0f); }
    CHECK(mx > 0.0f);
    std::printf("host layer GPU checks: %d failures\n", failures);
    return failures ? 1 : 0;
}

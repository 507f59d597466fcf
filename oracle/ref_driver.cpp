// ref_driver.cpp — C entry points around the reference's OWN CPU implementation
// of the path (GeodesicTracer + Geodesic + TensorOps), compiled from the
// reference's sources where they lie, by oracle/Makefile, into oracle/_ref/.
//
// TEST INFRASTRUCTURE ONLY: used to pin the oracle (golden fixtures, compat
// parity) and as the timed CPU baseline ("reference" kind) of bench.py. The
// reference source tree is read at build time only; the built library travels
// with the repository snapshot.
//
// The thread pool below reproduces RenderSession's CPU pattern: an atomic pixel
// queue over N worker threads, one GeodesicTracer per thread sharing one
// read-only metric (src/Sirius.Infrastructure/Session/SNRS001A.cpp:174-190,871-911).
#include <algorithm>
#include <atomic>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

#include "GTRC001A.h"
#include "PHAD001A.h"

using namespace Sirius;

extern "C" {

// Flat record of one TraceResult (the fields the parity tests compare).
struct ref_trace_record {
    int32_t outcome;
    int32_t steps_taken;
    int32_t numerical_failure;
    int32_t num_disk_crossings;
    double final_position[4];
    double final_direction[4];
    float disk_r[4];
    float disk_phi[4];
    float disk_redshift[4];
    float disk_temperature[4];
    int32_t equatorial_crossings;
    int32_t image_order;
    float total_phi_change;
    float min_radius;
    float redshift;
    float magnification;
    float impact_parameter;
    float optical_depth;
    float volumetric_emission;
    int32_t photon_ring;
};

// Mirror of the TracerConfig/IntegratorConfig fields a caller may set.
struct ref_tracer_config {
    float escape_radius, horizon_factor;
    int32_t max_steps;
    int32_t enable_disk;
    float disk_inner, disk_outer, disk_temperature_inner;
    int32_t enable_volumetric;
    float abs_tolerance, rel_tolerance, min_step, max_step, initial_step, safety_factor, step_grow_max,
        step_shrink_min;
};

static TracerConfig make_config(const ref_tracer_config& c) {
    TracerConfig t;
    t.escape_radius = c.escape_radius;
    t.horizon_factor = c.horizon_factor;
    t.max_steps = c.max_steps;
    t.enable_disk = c.enable_disk != 0;
    t.disk_inner = c.disk_inner;
    t.disk_outer = c.disk_outer;
    t.disk_temperature_inner = c.disk_temperature_inner;
    t.enable_volumetric = c.enable_volumetric != 0;
    t.integrator.abs_tolerance = c.abs_tolerance;
    t.integrator.rel_tolerance = c.rel_tolerance;
    t.integrator.min_step = c.min_step;
    t.integrator.max_step = c.max_step;
    t.integrator.initial_step = c.initial_step;
    t.integrator.safety_factor = c.safety_factor;
    t.integrator.step_grow_max = c.step_grow_max;
    t.integrator.step_shrink_min = c.step_shrink_min;
    t.integrator.use_rk45 = true;
    return t;
}

static void fill(const TraceResult& r, ref_trace_record& o) {
    std::memset(&o, 0, sizeof(o));
    o.outcome = int32_t(r.outcome);
    o.steps_taken = r.steps_taken;
    o.numerical_failure = r.numerical_failure;
    o.num_disk_crossings = r.num_disk_crossings;
    for (int i = 0; i < 4; ++i) {
        o.final_position[i] = r.final_position(i);
        o.final_direction[i] = r.final_direction(i);
        o.disk_r[i] = r.disk_crossings[i].r;
        o.disk_phi[i] = r.disk_crossings[i].phi;
        o.disk_redshift[i] = r.disk_crossings[i].redshift;
        o.disk_temperature[i] = r.disk_crossings[i].temperature;
    }
    o.equatorial_crossings = r.equatorial_crossings;
    o.image_order = r.image_order;
    o.total_phi_change = r.total_phi_change;
    o.min_radius = r.min_radius;
    o.redshift = r.redshift;
    o.magnification = r.magnification;
    o.impact_parameter = r.impact_parameter;
    o.optical_depth = r.optical_depth;
    o.volumetric_emission = r.volumetric_emission[0];
    o.photon_ring = r.photon_ring;
}

int ref_sizeof_record() { return int(sizeof(ref_trace_record)); }

// Kerr-Schild metric (M, a, Q, Lambda): g (16) and dg (64, only .real) at n points.
int ref_ks_evaluate(double M, double a, double Q, double Lambda, const double* pos, int64_t n, double* g,
                    double* dg) {
    KerrSchildFamily metric(KerrSchildParams{M, a, Q, Lambda});
    for (int64_t i = 0; i < n; ++i) {
        Tensor<double, 4> x;
        for (int j = 0; j < 4; ++j) x(j) = pos[4 * i + j];
        Metric4D gg;
        Tensor<Dual<double>, 4, 4, 4> dd;
        metric.evaluate(x, gg, dd);
        for (int p = 0; p < 4; ++p)
            for (int q = 0; q < 4; ++q) {
                g[16 * i + 4 * p + q] = gg(p, q).real;
                for (int l = 0; l < 4; ++l) dg[64 * i + 16 * l + 4 * p + q] = dd(l, p, q).real;
            }
    }
    return 0;
}

// Pinhole camera rays (PinholeCamera::generateRay) for pixels (px[i], py[i]).
int ref_camera_rays(double r, double theta, double phi, float fov, int width, int height, float yaw, float pitch,
                    float roll, const int32_t* px, const int32_t* py, int64_t n, double* origin, double* dir) {
    CameraConfig cc;
    cc.r = r; cc.theta = theta; cc.phi = phi; cc.fov = fov; cc.width = width; cc.height = height;
    cc.yaw = yaw; cc.pitch = pitch; cc.roll = roll;
    PinholeCamera cam(cc);
    for (int64_t i = 0; i < n; ++i) {
        CameraRay ray = cam.generateRay(px[i], py[i]);
        for (int j = 0; j < 4; ++j) {
            origin[4 * i + j] = ray.origin(j);
            dir[4 * i + j] = ray.direction(j);
        }
    }
    return 0;
}

// PinholeCamera::generateRay(x, y, u, v) with a sub-pixel position per ray
// (the stratified samples of RenderSession::shadePixel, SNRS001A.cpp:480-497).
int ref_camera_rays_uv(double r, double theta, double phi, float fov, int width, int height, float yaw, float pitch,
                       float roll, const int32_t* px, const int32_t* py, const float* u, const float* v, int64_t n,
                       double* origin, double* dir) {
    CameraConfig cc;
    cc.r = r; cc.theta = theta; cc.phi = phi; cc.fov = fov; cc.width = width; cc.height = height;
    cc.yaw = yaw; cc.pitch = pitch; cc.roll = roll;
    PinholeCamera cam(cc);
    for (int64_t i = 0; i < n; ++i) {
        CameraRay ray = cam.generateRay(px[i], py[i], u[i], v[i]);
        for (int j = 0; j < 4; ++j) {
            origin[4 * i + j] = ray.origin(j);
            dir[4 * i + j] = ray.direction(j);
        }
    }
    return 0;
}

// One Geodesic::integrateStepRK45 call per Lightray (position, velocity, h).
// Returns success flags and terminated codes; updates pos/vel/h in place.
int ref_rk45_step(double M, double a, const ref_tracer_config* c, double* pos, double* vel, float* h,
                  int32_t* success, int32_t* terminated, int64_t n) {
    KerrSchildFamily metric(KerrSchildParams::Kerr(M, a));
    TracerConfig tc = make_config(*c);
    for (int64_t i = 0; i < n; ++i) {
        Lightray ray{};
        for (int j = 0; j < 4; ++j) { ray.position(j) = pos[4 * i + j]; ray.velocity(j) = vel[4 * i + j]; }
        ray.step_size = h[i];
        ray.terminated = 0;
        success[i] = Geodesic::integrateStepRK45(ray, &metric, tc.integrator) ? 1 : 0;
        terminated[i] = ray.terminated;
        for (int j = 0; j < 4; ++j) { pos[4 * i + j] = ray.position(j); vel[4 * i + j] = ray.velocity(j); }
        h[i] = ray.step_size;
    }
    return 0;
}

// GeodesicTracer::trace for host camera rays, RenderSession-style thread pool.
int ref_trace_rays(double M, double a, const ref_tracer_config* c, const double* origin, const double* dir,
                   int64_t n, ref_trace_record* out, int threads) {
    KerrSchildFamily metric(KerrSchildParams::Kerr(M, a));
    TracerConfig tc = make_config(*c);
    std::atomic<int64_t> next{0};
    auto worker = [&]() {
        GeodesicTracer tracer(&metric, tc);
        for (;;) {
            const int64_t i = next.fetch_add(1);
            if (i >= n) break;
            CameraRay ray;
            for (int j = 0; j < 4; ++j) { ray.origin(j) = origin[4 * i + j]; ray.direction(j) = dir[4 * i + j]; }
            fill(tracer.trace(ray), out[i]);
        }
    };
    threads = std::max(1, threads);
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; ++t) pool.emplace_back(worker);
    for (auto& t : pool) t.join();
    return 0;
}

// Pinhole frame: camera rays generated per pixel inside the worker, as
// RenderSession::shadePixel does (SNRS001A.cpp:480-558, 1 spp at the centre).
int ref_trace_frame(double M, double a, const ref_tracer_config* c, double r_obs, double theta, double phi, float fov,
                    int width, int height, int64_t first, int64_t count, ref_trace_record* out, int threads) {
    KerrSchildFamily metric(KerrSchildParams::Kerr(M, a));
    TracerConfig tc = make_config(*c);
    CameraConfig cc;
    cc.r = r_obs; cc.theta = theta; cc.phi = phi; cc.fov = fov; cc.width = width; cc.height = height;
    PinholeCamera cam(cc);
    std::atomic<int64_t> next{0};
    auto worker = [&]() {
        GeodesicTracer tracer(&metric, tc);
        for (;;) {
            const int64_t i = next.fetch_add(1);
            if (i >= count) break;
            const int64_t pix = first + i;
            CameraRay ray = cam.generateRay(int(pix % width), int(pix / width));
            TraceResult r = tracer.trace(ray);
            if (out) fill(r, out[i]);
        }
    };
    threads = std::max(1, threads);
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; ++t) pool.emplace_back(worker);
    for (auto& t : pool) t.join();
    return 0;
}

double ref_isco(double a_star) { return AccretionDiskD::computeISCO(a_star); }

double ref_nt_flux_q(double r, double a_star) {
    // Page-Thorne Q(r) = F / F_newt of AccretionDiskD::flux (PHAD001A.h:321-361)
    AccretionDiskD::Config cfg;
    cfg.M = 1.0;
    cfg.a_star = a_star;
    cfg.r_outer = 1000.0;
    AccretionDiskD disk(cfg);
    const double F = disk.flux(r);
    const double rs = disk.schwarzschildRadius();
    const double rp = r * rs / 2.0;
    const double Mdot = cfg.Mdot * 1.98847e30 / (365.25 * 24 * 3600);
    (void)Mdot;
    return F * rp * rp * rp;  // proportional to Q(r)/1 with a constant SI prefactor
}

}  // extern "C"

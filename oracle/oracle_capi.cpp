// oracle_capi.cpp — C entry points of the CPU oracle (liboracle.so).
//
// TEST INFRASTRUCTURE ONLY: called by tests/, __graft_entry__.smoke() and the
// CPU-baseline leg of bench.py, as the checker. The product never links it.
#include <algorithm>
#include <atomic>
#include <thread>
#include <vector>

#include "oracle.hpp"

using namespace oracle;

namespace {

template <class R>
void trace_pixels(const sirius_frame& f, const sirius_trace_config& cfg, int64_t first, int64_t count,
                  sirius_ray_result* out, double* bins, int threads) {
    TraceContext ctx;
    ctx.metric = f.metric;
    ctx.cfg = cfg;
    const double astar = f.metric.M != 0 ? f.metric.a / f.metric.M : 0.0;
    ctx.disk_inner = f.disk_inner > 0 ? f.disk_inner : isco(astar) * f.metric.M;
    ctx.disk_outer = f.disk_outer;
    const int nb = std::min(cfg.n_bins, SIRIUS_MAX_BINS);
    // pixel indices are relative to the frame's row window (row_count 0: the whole image)
    const int64_t row0 = f.row_count > 0 ? f.row_begin : 0;
    std::atomic<int64_t> next{0};
    auto worker = [&]() {
        for (;;) {
            const int64_t i = next.fetch_add(1);
            if (i >= count) break;
            const int64_t pix = row0 * f.camera.width + first + i;
            const int px = int(pix % f.camera.width), py = int(pix / f.camera.width);
            double o[4], d[4];
            camera_ray(f.camera, px, py, o, d);
            trace_ray<R>(ctx, o, d, out[i], bins ? bins + i * nb : nullptr);
        }
    };
    threads = std::max(1, threads);
    if (threads == 1) { worker(); return; }
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; ++t) pool.emplace_back(worker);
    for (auto& t : pool) t.join();
}

}  // namespace

extern "C" {

int oracle_version() { return SIRIUS_CUDA_ABI_VERSION; }
int oracle_sizeof_result() { return int(sizeof(sirius_ray_result)); }
int oracle_sizeof_config() { return int(sizeof(sirius_trace_config)); }
int oracle_sizeof_frame() { return int(sizeof(sirius_frame)); }

// Trace pixels [first, first+count) of one frame (row-major pixel index within
// the frame's row window).
// precision: 0 = double, 1 = long double.
int oracle_trace_frame(const sirius_frame* f, const sirius_trace_config* cfg, int64_t first, int64_t count,
                       sirius_ray_result* out, double* bins, int threads, int precision) {
    if (!f || !cfg || !out || count < 0) return 1;
    if (precision == 1) trace_pixels<long double>(*f, *cfg, first, count, out, bins, threads);
    else trace_pixels<double>(*f, *cfg, first, count, out, bins, threads);
    return 0;
}

// Trace host-generated camera rays through one metric.
int oracle_trace_rays(const sirius_metric* m, double disk_inner, double disk_outer, const sirius_trace_config* cfg,
                      const sirius_camera_ray* rays, int64_t n, sirius_ray_result* out, int threads) {
    if (!m || !cfg || !rays || !out) return 1;
    TraceContext ctx;
    ctx.metric = *m;
    ctx.cfg = *cfg;
    const double astar = m->M != 0 ? m->a / m->M : 0.0;
    ctx.disk_inner = disk_inner > 0 ? disk_inner : isco(astar) * m->M;
    ctx.disk_outer = disk_outer;
    std::atomic<int64_t> next{0};
    auto worker = [&]() {
        for (;;) {
            const int64_t i = next.fetch_add(1);
            if (i >= n) break;
            trace_ray<double>(ctx, rays[i].origin, rays[i].direction, out[i], nullptr);
        }
    };
    threads = std::max(1, threads);
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; ++t) pool.emplace_back(worker);
    for (auto& t : pool) t.join();
    return 0;
}

// the camera mapping in FP64 at a fractional pixel position (u, v in pixel units)
int oracle_camera_ray_exact(const sirius_camera* cam, double u, double v, double* origin, double* dir) {
    camera_ray_exact(*cam, u, v, origin, dir);
    return 0;
}

// PinholeCamera::generateRay(x, y, u, v) (CMBS001A.h:120): the ray through sub-pixel (u, v)
int oracle_camera_ray_uv(const sirius_camera* cam, int px, int py, float u, float v, double* origin, double* dir) {
    camera_ray(*cam, px, py, origin, dir, u, v);
    return 0;
}

int oracle_camera_ray(const sirius_camera* cam, int px, int py, double* origin, double* dir) {
    camera_ray(*cam, px, py, origin, dir);
    return 0;
}

// g: n x 16, dg: n x 64 (dg[l*16 + m*4 + n] = d_l g_mn)
int oracle_metric_evaluate(const sirius_metric* m, const double* pos, int64_t n, double* g, double* dg) {
    for (int64_t i = 0; i < n; ++i) {
        double gg[4][4], dd[4][4][4];
        metric_evaluate(*m, pos + 4 * i, gg, dd);
        for (int a = 0; a < 4; ++a)
            for (int b = 0; b < 4; ++b) {
                g[16 * i + 4 * a + b] = gg[a][b];
                for (int l = 0; l < 4; ++l) dg[64 * i + 16 * l + 4 * a + b] = dd[l][a][b];
            }
    }
    return 0;
}

int oracle_invert4x4(const double* m, double* inv) {
    double a[4][4], b[4][4];
    for (int i = 0; i < 16; ++i) a[i / 4][i % 4] = m[i];
    invert4x4(a, b);
    for (int i = 0; i < 16; ++i) inv[i] = b[i / 4][i % 4];
    return 0;
}

// state: n x 8 (x, p) -> derivative n x 8 (k, dp)
int oracle_rhs(const sirius_metric* m, const double* state, int64_t n, double* out, int compat) {
    for (int64_t i = 0; i < n; ++i) rhs(*m, state + 8 * i, state + 8 * i + 4, out + 8 * i, out + 8 * i + 4, compat != 0);
    return 0;
}

// One DP45 attempt per state (fresh stage 1). state/h updated in place on accept.
int oracle_dp45_step(const sirius_metric* m, const sirius_trace_config* cfg, double* state, double* h,
                     int32_t* accepted, double* err, int64_t n) {
    for (int64_t i = 0; i < n; ++i) {
        double* s = state + 8 * i;
        double k1x[4], k1p[4], xn[4], pn[4], k7x[4], k7p[4];
        rhs(*m, s, s + 4, k1x, k1p, false);
        const double e = dp45_attempt(*m, *cfg, s, s + 4, h[i], k1x, k1p, xn, pn, k7x, k7p, false);
        err[i] = e;
        accepted[i] = (e <= 1.0) ? 1 : 0;
        if (accepted[i])
            for (int j = 0; j < 4; ++j) { s[j] = xn[j]; s[4 + j] = pn[j]; }
        h[i] = optimal_step(h[i], e, *cfg, false);
    }
    return 0;
}

// Geodesic::integrateStepRK45 as written, per Lightray (pos, vel: n x 4; h float).
int oracle_rk45_step_compat(const sirius_metric* m, const sirius_trace_config* cfg, double* pos, double* vel, float* h,
                            int32_t* success, int32_t* terminated, int64_t n) {
    for (int64_t i = 0; i < n; ++i) {
        double hh = double(h[i]);
        int term = 0;
        success[i] = compat_rk45_step(*m, *cfg, pos + 4 * i, vel + 4 * i, hh, term) ? 1 : 0;
        terminated[i] = term;
        h[i] = float(hh);
    }
    return 0;
}

// E/L_z-preserving projection along dr; returns the null value before projection.
double oracle_project_null(const sirius_metric* m, const double* x, double* p) { return project_null(*m, x, p); }
double oracle_null_value(const sirius_metric* m, const double* x, const double* p) { return null_value(*m, x, p); }
int oracle_invariants(const sirius_metric* m, const double* x, const double* p, double* out3) {
    invariants(*m, x, p, out3[0], out3[1], out3[2]);
    return 0;
}
double oracle_radial(const sirius_metric* m, const double* x, double* grad) { return radial(*m, x, grad); }
double oracle_isco(double a_star) { return isco(a_star); }
double oracle_r_photon(double M, double a, int prograde) { return r_photon(M, a, prograde != 0); }
double oracle_r_plus(const sirius_metric* m) { return r_plus(*m); }
double oracle_nt_flux(double r, double a_star, double r_in, double r_out) { return nt_flux(r, a_star, r_in, r_out); }

// Initial state (x, p) of a camera ray; compat selects the reference's float roundings.
int oracle_init_state(const sirius_metric* m, const sirius_trace_config* cfg, const double* origin, const double* dir,
                      double* x, double* p, double* k) {
    TraceContext ctx;
    ctx.metric = *m;
    ctx.cfg = *cfg;
    ctx.disk_inner = 0;
    ctx.disk_outer = 0;
    init_state<double>(ctx, origin, dir, x, p, k);
    return 0;
}

}  // extern "C"

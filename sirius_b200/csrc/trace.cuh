// trace.cuh — the per-ray state machine of the geodesic engine (device code).
//
// One thread owns one ray at a time. A ray is initialised from its pixel
// (PinholeCamera::generateRay + GeodesicTracer::initializeLightray,
// CMBS001A.h:120-185, GTRC001A.cpp:15-134), advanced by Dormand-Prince 5(4)
// steps on (x^mu, p_mu) (Geodesic::integrateStepRK45, PHGD001A.cpp:530-641)
// with retry-on-reject, re-projected onto the null cone in FP64 after
// accepted steps, and checked for the reference's terminations in its order
// (GeodesicTracer::trace, GTRC001A.cpp:264-556): failure, spiral, horizon,
// escape, volumetric segment, thin-disk crossing.
#pragma once

#include <stdint.h>

#include "packed.cuh"
#include "spacetime.cuh"

#include <type_traits>

namespace sirius {

constexpr double kPi = 3.14159265358979323846;

// Per-frame constants prepared on the host (double precision, host libm).
struct FrameDev {
    MetricDev m;
    long long ray_offset, n_rays;
    int width, height, projection, has_horizon, gate;
    int flux_slot;  // index of this frame's disk flux table (its position in the launch)
    int row0;       // first camera row of the frame's row window (pixel row of its ray 0)
    // camera
    double cam_t, cam_r, cam_st, cam_ct, cam_sp, cam_cp, cam_th, cam_ph;
    float aspect, tan_half_fov, cY, sY, cP, sP, cR, sR;
    // radii
    double disk_in, disk_out, r_hor, r_plus, island_r, a_star, isco, r_ph_pro;
    double sqrt_m_gtt_cam;
    float fsqrt_m_gtt_cam, fdisk_in, fdisk_out, fr_ph_pro;  // FP32 copies
    // observer (enum sirius_observer); for the zero-angular-momentum observer:
    // the camera's Kerr-Schild position and the four tetrad vectors e_(t),
    // e_(r), e_(theta), e_(phi) in Kerr-Schild contravariant components
    int observer;
    float sub_u, sub_v;  // sub-pixel position of the ray through a pixel (0.5, 0.5: the centre)
    double zx[4];
    double ze[16];  // ze[4 i + mu]: vector i, component mu
};

// The observer's energy normalisation in the redshift of an emitter: the
// static observer sees E / sqrt(-g_tt(camera)); the zero-angular-momentum
// observer sees frequency 1 by construction, so the factor is E itself.
template <class T>
__device__ __forceinline__ T observer_factor(const FrameDev& F, T E) {
    return F.observer == SIRIUS_OBSERVER_ZAMO ? E : cst<T>(F.sqrt_m_gtt_cam, F.fsqrt_m_gtt_cam);
}

struct CfgDev {
    double atol, rtol, hmin, hmax, h0, safety, grow, shrink;
    double escape_r, decay;
    int max_steps, enable_disk, enable_vol, nbins, vol_sub, proj_period, spiral, compat;
    int integrator, symp_order;
    double symp_step, crit_band;
    double vol_j0, vol_aoj, vol_hz, vol_s;
    // FP32 copies for the single-precision paths
    float fatol, frtol, fsafety, fgrow, fshrink, fvol_j0, fvol_aoj, fvol_hz, fvol_s;
    int npair;                       // bin pairs, (nbins + 1) / 2
    float2 nu_l2[SIRIUS_MAX_BINS / 2];  // -nu^-s / ln 2 of bins (2j, 2j + 1); 0 pads an odd last pair
    int nu_desc;                        // 1: |nu_l2| falls along the bins (spectral index >= 0)
};

// ---------------------------------------------------------------------------
// Page-Thorne flux (AccretionDiskD::flux / fullPageThorneFlux, PHAD001A.h:112-361)
// in geometric units F = 3/(8 pi r^3) Q(r); 16-point Gauss-Legendre on [r_isco, r]
// (nodes/weights: Abramowitz & Stegun table 25.4).
// ---------------------------------------------------------------------------
__device__ __forceinline__ double pt_E(double r, double a) {
    const double s = sqrt(r), d = r * sqrt(r * r - 3.0 * r + 2.0 * a * s);
    return fabs(d) < 1e-15 ? 1.0 : (r * r - 2.0 * r + a * s) / d;
}
__device__ __forceinline__ double pt_L(double r, double a) {
    const double s = sqrt(r), d = r * sqrt(r * r - 3.0 * r + 2.0 * a * s);
    return fabs(d) < 1e-15 ? 0.0 : (r * r - 2.0 * a * s + a * a) / d;
}
__device__ __forceinline__ double pt_Om(double r, double a) { return 1.0 / (r * sqrt(r) + a); }
__device__ __forceinline__ double pt_dLdr(double r, double a) {
    if (r <= 0) return 0;
    const double sr = sqrt(r);
    const double N = r * r - 2.0 * a * sr + a * a, D = r * r - 3.0 * r + 2.0 * a * sr;
    if (D <= 1e-15) return 0;
    const double sD = sqrt(D), q = a / sr;
    const double dN = 2.0 * r - q, dD = 2.0 * r - 3.0 + q;
    const double drsD = (2.0 * D + r * dD) / (2.0 * sD), rsD = r * sD, den = rsD * rsD;
    if (fabs(den) < 1e-30) return 0;
    return (dN * rsD - N * drsD) / den;
}
__device__ __forceinline__ double pt_dOm(double r, double a) {
    if (r <= 0) return 0;
    const double den = r * sqrt(r) + a;
    return -3.0 * sqrt(r) / (2.0 * den * den);
}

static __device__ __noinline__ double nt_flux(double r, double a, double isco, double r_in, double r_out) {
    const double gx[8] = {0.0950125098376374, 0.2816035507792589, 0.4580167776572274, 0.6178762444026438,
                          0.7554044083550030, 0.8656312023878318, 0.9445750230732326, 0.9894009349916499};
    const double gw[8] = {0.1894506104550685, 0.1826034150449236, 0.1691565193950025, 0.1495959888165767,
                          0.1246289712555339, 0.0951585116824928, 0.0622535239386479, 0.0271524594117541};
    if (r < r_in || r > r_out || r <= isco) return 0.0;
    const double Fn = 3.0 / (8.0 * kPi * r * r * r);
    if (r > 1.5 * isco) {
        const double hw = 0.5 * (r - isco), mid = 0.5 * (r + isco);
        double I = 0;
        for (int sgn = -1; sgn <= 1; sgn += 2)
            for (int i = 0; i < 8; ++i) {
                const double rr = mid + hw * sgn * gx[i];
                I += gw[i] * (pt_E(rr, a) - pt_Om(rr, a) * pt_L(rr, a)) * pt_dLdr(rr, a);
            }
        I *= hw;
        const double EmOL = pt_E(r, a) - pt_Om(r, a) * pt_L(r, a);
        if (fabs(EmOL) >= 1e-15) {
            const double F = Fn * (-pt_dOm(r, a) / (EmOL * EmOL)) * I;
            if (isfinite(F) && F > 0) return F;
        }
    }
    const double it = 1.0 - sqrt(isco / r);
    if (it <= 0) return 0.0;
    const double y = sqrt(r), den = y * y * y * (y - 3.0 / y + 2.0 * a / (y * y));
    double Q = fabs(den) > 1e-10 ? 1.0 / den : 1.0;
    if (!isfinite(Q) || Q <= 0) Q = 1.0;
    Q = fmin(fmax(Q, 0.1), 10.0);
    return Fn * it * Q;
}

// ---------------------------------------------------------------------------
// Camera ray for pixel (px, py). The pinhole arithmetic is the reference's
// float arithmetic (CMBS001A.h:130-181) with every operation rounded
// individually (no contraction), the trigonometric constants taken from the host.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void camera_dir(const FrameDev& F, int px, int py, double dir[4]) {
    dir[0] = 0.0;
    if (F.projection == SIRIUS_CAMERA_EQUIRECTANGULAR) {
        const double psi = (2.0 * (px + double(F.sub_u)) / F.width - 1.0) * kPi;
        const double chi = (1.0 - 2.0 * (py + double(F.sub_v)) / F.height) * (0.5 * kPi);
        double sc, cc, sps, cps;
        sincos(chi, &sc, &cc);
        sincos(psi, &sps, &cps);
        dir[1] = -cc * cps;
        dir[2] = -sc;
        dir[3] = cc * sps;
        return;
    }
    const float w = float(F.width), hgt = float(F.height);
    const float pxn = __fmul_rn(__fsub_rn(__fdiv_rn(__fmul_rn(2.0f, __fadd_rn(float(px), F.sub_u)), w), 1.0f), F.aspect);
    const float pyn = __fsub_rn(1.0f, __fdiv_rn(__fmul_rn(2.0f, __fadd_rn(float(py), F.sub_v)), hgt));
    const float dx = __fmul_rn(pxn, F.tan_half_fov), dy = __fmul_rn(pyn, F.tan_half_fov), dz = -1.0f;
    const float rx = __fsub_rn(__fmul_rn(dx, F.cR), __fmul_rn(dy, F.sR));
    const float ry = __fadd_rn(__fmul_rn(dx, F.sR), __fmul_rn(dy, F.cR));
    const float ry2 = __fsub_rn(__fmul_rn(ry, F.cP), __fmul_rn(dz, F.sP));
    const float rz = __fadd_rn(__fmul_rn(ry, F.sP), __fmul_rn(dz, F.cP));
    const float rx2 = __fadd_rn(__fmul_rn(rx, F.cY), __fmul_rn(rz, F.sY));
    const float rz2 = __fadd_rn(__fmul_rn(-rx, F.sY), __fmul_rn(rz, F.cY));
    const float len = __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(rx2, rx2), __fmul_rn(ry2, ry2)), __fmul_rn(rz2, rz2)));
    dir[1] = double(__fdiv_rn(rz2, len));
    dir[2] = double(__fdiv_rn(-ry2, len));
    dir[3] = double(__fdiv_rn(rx2, len));
}

// TensorOps::normalizeNull (MTTN001A.cpp:171-237) for k^0, given g_0mu, g_ij.
__device__ __forceinline__ double null_k0(const double g[16], const double k[4]) {
    const double A = g[0];
    double B = 0, C = 0;
    for (int i = 1; i < 4; ++i) B += 2.0 * g[i] * k[i];
    for (int i = 1; i < 4; ++i)
        for (int j = 1; j < 4; ++j) C += g[4 * i + j] * k[i] * k[j];
    if (fabs(A) < 1e-15) return fabs(B) > 1e-15 ? -C / B : 1.0;
    const double d = B * B - 4.0 * A * C;
    if (d < 0.0) return 1.0;
    const double sd = sqrt(d);
    const double kp = (-B + sd) / (2.0 * A), km = (-B - sd) / (2.0 * A);
    if (kp > 0.0) return kp;
    if (km > 0.0) return km;
    return fmax(kp, km);
}

// k^0 from the null condition, then p_mu = g_mu_nu k^nu.
__device__ __forceinline__ void null_momentum(const double g[16], double k[4], double p[4]) {
    k[0] = 0.0;
    k[0] = null_k0(g, k);
    for (int mu = 0; mu < 4; ++mu) {
        double s = 0;
        for (int nu = 0; nu < 4; ++nu) s += g[4 * mu + nu] * k[nu];
        p[mu] = s;
    }
}

// Initial state from a camera ray (GTRC001A.cpp:15-134 without float roundings):
// spherical map of the camera position, spherical -> Cartesian velocity,
// normalizeNull for k^0, p = g k.
__device__ __forceinline__ void init_state(const FrameDev& F, const double dir[4], double x[4], double p[4]) {
    if (F.observer == SIRIUS_OBSERVER_ZAMO) {
        // k = e_(t) + n^r e_(r) + n^theta e_(theta) + n^phi e_(phi), n = dir (a unit vector)
        double k[4], g[16];
        for (int mu = 0; mu < 4; ++mu) {
            x[mu] = F.zx[mu];
            k[mu] = F.ze[mu] + dir[1] * F.ze[4 + mu] + dir[2] * F.ze[8 + mu] + dir[3] * F.ze[12 + mu];
        }
        metric_g(F.m, x, g);
        for (int mu = 0; mu < 4; ++mu) {
            double s = 0;
            for (int nu = 0; nu < 4; ++nu) s += g[4 * mu + nu] * k[nu];
            p[mu] = s;
        }
        return;
    }
    const double r = F.cam_r, st = F.cam_st, ct = F.cam_ct, sp = F.cam_sp, cp = F.cam_cp;
    const double vr = dir[1], vth = dir[2] / r;
    double vph = dir[3] / (r * st);
    if (fabs(st) < 1e-10) vph = 0.0;
    double k[4];
    double g[16];
    if (F.m.family == SIRIUS_METRIC_MORRIS_THORNE) {
        x[0] = F.cam_t; x[1] = r; x[2] = F.cam_th; x[3] = F.cam_ph;
        metric_g(F.m, x, g);
        k[1] = vr / sqrt(g[5]); k[2] = vth; k[3] = vph;
    } else {
        x[0] = F.cam_t; x[1] = r * st * cp; x[2] = r * st * sp; x[3] = r * ct;
        k[1] = vr * st * cp + r * vth * ct * cp - r * vph * st * sp;
        k[2] = vr * st * sp + r * vth * ct * sp + r * vph * st * cp;
        k[3] = vr * ct - r * vth * st;
        metric_g(F.m, x, g);
    }
    null_momentum(g, k, p);
}

// Kerr-Schild camera position of a frame (the x of init_state's Cartesian branch).
__device__ __forceinline__ void camera_position_ks(const FrameDev& F, double x[4]) {
    const double r = F.cam_r, st = F.cam_st, ct = F.cam_ct, sp = F.cam_sp, cp = F.cam_cp;
    x[0] = F.cam_t; x[1] = r * st * cp; x[2] = r * st * sp; x[3] = r * ct;
}

// init_state's Cartesian (Kerr-Schild family) branch with the metric at the
// camera already evaluated: the same operations in the same order, for kernels
// that start many rays from one camera.
__device__ __forceinline__ void init_state_ks(const FrameDev& F, const double dir[4], const double g[16],
                                              double x[4], double p[4]) {
    const double r = F.cam_r, st = F.cam_st, ct = F.cam_ct, sp = F.cam_sp, cp = F.cam_cp;
    const double vr = dir[1], vth = dir[2] / r;
    double vph = dir[3] / (r * st);
    if (fabs(st) < 1e-10) vph = 0.0;
    double k[4];
    camera_position_ks(F, x);
    k[1] = vr * st * cp + r * vth * ct * cp - r * vph * st * sp;
    k[2] = vr * st * sp + r * vth * ct * sp + r * vph * st * cp;
    k[3] = vr * ct - r * vth * st;
    null_momentum(g, k, p);
}

// ---------------------------------------------------------------------------
// Dormand-Prince 5(4) tableau (Dormand & Prince 1980; PHGD001A.cpp:16-79) in
// sliding-window form: DP_A[j][s] = a_{j+2+s, j+1}, the weight of k_{j+1} in
// the input of stage j+2+s (row 7 = the fifth-order weights b, first same as
// last); DP_E[j] = b_{j+1} - b*_{j+1}. Rows are read with a warp-uniform index
// (constant-cache broadcast).
// ---------------------------------------------------------------------------
template <class T>
struct DPTable {
    T A[6][6];
    T E[7];
};
#define SIRIUS_DP45_TABLE(T)                                                                                      \
    {{{T(1.0 / 5.0), T(3.0 / 40.0), T(44.0 / 45.0), T(19372.0 / 6561.0), T(9017.0 / 3168.0), T(35.0 / 384.0)},      \
      {T(9.0 / 40.0), T(-56.0 / 15.0), T(-25360.0 / 2187.0), T(-355.0 / 33.0), T(0), T(0)},                        \
      {T(32.0 / 9.0), T(64448.0 / 6561.0), T(46732.0 / 5247.0), T(500.0 / 1113.0), T(0), T(0)},                    \
      {T(-212.0 / 729.0), T(49.0 / 176.0), T(125.0 / 192.0), T(0), T(0), T(0)},                                     \
      {T(-5103.0 / 18656.0), T(-2187.0 / 6784.0), T(0), T(0), T(0), T(0)},                                          \
      {T(11.0 / 84.0), T(0), T(0), T(0), T(0), T(0)}},                                                              \
     {T(35.0 / 384.0 - 5179.0 / 57600.0), T(0), T(500.0 / 1113.0 - 7571.0 / 16695.0),                              \
      T(125.0 / 192.0 - 393.0 / 640.0), T(-2187.0 / 6784.0 + 92097.0 / 339200.0), T(11.0 / 84.0 - 187.0 / 2100.0),  \
      T(-1.0 / 40.0)}}
static __constant__ DPTable<float> kDPf = SIRIUS_DP45_TABLE(float);
static __constant__ DPTable<double> kDPd = SIRIUS_DP45_TABLE(double);

template <class T>
__device__ __forceinline__ const DPTable<T>& dp_table();
template <>
__device__ __forceinline__ const DPTable<float>& dp_table<float>() { return kDPf; }
template <>
__device__ __forceinline__ const DPTable<double>& dp_table<double>() { return kDPd; }

// One DP45 attempt on y = (x^mu, p_mu) with the stage arithmetic in T (float:
// the FP32 bulk; double: FP64). The state stays in FP64; stage inputs are
// x + h acc where acc = sum_j a_sj k_j accumulates in T in a sliding window, so
// the six right-hand sides share one call site (a compact loop body keeps the
// instruction stream in cache). The p_0 component is not accumulated: every
// family's metric is static, so dp_0/dl = 0 and p_0 (the conserved -E) carries
// through the attempt unchanged. On entry k1 = f(x, p); on exit (xn, pn) is the
// fifth-order solution and k7 = f(xn, pn) (first same as last). Returns the
// scaled RMS error of the position components (computeRK45ErrorNorm,
// PHGD001A.cpp:508-517).
// The FP32 attempt of dp45_attempt with its stage accumulators in packed pairs
// of components ((x0, x1), (x2, x3), (p1, p2), (p3, -); p_0 is constant): every
// fold of a stage derivative is one f32x2 FMA per pair (1024^2 bench frame
// 22.7 -> 22.4 ms; images move by ~1e-8 of the peak, FP32 contraction order).
// The Dormand-Prince tableau as lane pairs (a, a), read with one 64-bit constant
// load (the two-ray kernel folds two rays' derivatives with it).
struct DPTablePair {
    float2 A[6][6];
    float2 E[7];
};
#define SIRIUS_X2(v) {float(v), float(v)}
static __constant__ DPTablePair kDPpair = {
    {{SIRIUS_X2(1.0 / 5.0), SIRIUS_X2(3.0 / 40.0), SIRIUS_X2(44.0 / 45.0), SIRIUS_X2(19372.0 / 6561.0),
      SIRIUS_X2(9017.0 / 3168.0), SIRIUS_X2(35.0 / 384.0)},
     {SIRIUS_X2(9.0 / 40.0), SIRIUS_X2(-56.0 / 15.0), SIRIUS_X2(-25360.0 / 2187.0), SIRIUS_X2(-355.0 / 33.0),
      SIRIUS_X2(0), SIRIUS_X2(0)},
     {SIRIUS_X2(32.0 / 9.0), SIRIUS_X2(64448.0 / 6561.0), SIRIUS_X2(46732.0 / 5247.0), SIRIUS_X2(500.0 / 1113.0),
      SIRIUS_X2(0), SIRIUS_X2(0)},
     {SIRIUS_X2(-212.0 / 729.0), SIRIUS_X2(49.0 / 176.0), SIRIUS_X2(125.0 / 192.0), SIRIUS_X2(0), SIRIUS_X2(0),
      SIRIUS_X2(0)},
     {SIRIUS_X2(-5103.0 / 18656.0), SIRIUS_X2(-2187.0 / 6784.0), SIRIUS_X2(0), SIRIUS_X2(0), SIRIUS_X2(0),
      SIRIUS_X2(0)},
     {SIRIUS_X2(11.0 / 84.0), SIRIUS_X2(0), SIRIUS_X2(0), SIRIUS_X2(0), SIRIUS_X2(0), SIRIUS_X2(0)}},
    {SIRIUS_X2(35.0 / 384.0 - 5179.0 / 57600.0), SIRIUS_X2(0), SIRIUS_X2(500.0 / 1113.0 - 7571.0 / 16695.0),
     SIRIUS_X2(125.0 / 192.0 - 393.0 / 640.0), SIRIUS_X2(-2187.0 / 6784.0 + 92097.0 / 339200.0),
     SIRIUS_X2(11.0 / 84.0 - 187.0 / 2100.0), SIRIUS_X2(-1.0 / 40.0)}};
#undef SIRIUS_X2

template <int FAM>
__device__ __forceinline__ double dp45_attempt_x2(const MetricDev& m, const CfgDev& c, const double x[4],
                                                  const double p[4], double h, const float k1[8], double xn[4],
                                                  double pn[4], float k7[8]) {
    const DPTablePair& D = kDPpair;
    const float ht = float(h);
    const float2 X[4] = {make_float2(float(x[0]), float(x[1])), make_float2(float(x[2]), float(x[3])),
                         make_float2(float(p[1]), float(p[2])), make_float2(float(p[3]), 0.f)};
    const float p0 = float(p[0]);
    float2 acc[6][4];
    float2 eacc[2];
    float kc[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) kc[i] = k1[i];
#pragma unroll
    for (int s = 0; s < 6; ++s)
#pragma unroll
        for (int q = 0; q < 4; ++q) acc[s][q] = make_float2(0.f, 0.f);
    eacc[0] = eacc[1] = make_float2(0.f, 0.f);
#pragma unroll 1
    for (int j = 0; j < 6; ++j) {
        const float2 k2[4] = {make_float2(kc[0], kc[1]), make_float2(kc[2], kc[3]), make_float2(kc[5], kc[6]),
                              make_float2(kc[7], 0.f)};
#pragma unroll
        for (int s = 0; s < 6; ++s) {
            const float2 a = D.A[j][s];
#pragma unroll
            for (int q = 0; q < 4; ++q) acc[s][q] = fma2(a, k2[q], acc[s][q]);
        }
        eacc[0] = fma2(D.E[j], k2[0], eacc[0]);
        eacc[1] = fma2(D.E[j], k2[1], eacc[1]);
        float xs[4], ps[4];
        if (j == 5) {  // stage 7 is the solution point
            const float a[8] = {acc[0][0].x, acc[0][0].y, acc[0][1].x, acc[0][1].y,
                                0.f, acc[0][2].x, acc[0][2].y, acc[0][3].x};
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                xn[i] = x[i] + h * double(a[i]);
                pn[i] = i == 0 ? p[0] : p[i] + h * double(a[4 + i]);
                xs[i] = float(xn[i]);
                ps[i] = float(pn[i]);
            }
        } else {
            const float2 h2 = make_float2(ht, ht);
            const float2 s0 = fma2(h2, acc[0][0], X[0]), s1 = fma2(h2, acc[0][1], X[1]);
            const float2 s2 = fma2(h2, acc[0][2], X[2]), s3 = fma2(h2, acc[0][3], X[3]);
            xs[0] = s0.x; xs[1] = s0.y; xs[2] = s1.x; xs[3] = s1.y;
            ps[0] = p0; ps[1] = s2.x; ps[2] = s2.y; ps[3] = s3.x;
        }
        rhs<float, FAM>(m, xs, ps, kc, kc + 4);
#pragma unroll
        for (int s = 0; s < 5; ++s)
#pragma unroll
            for (int q = 0; q < 4; ++q) acc[s][q] = acc[s + 1][q];
#pragma unroll
        for (int q = 0; q < 4; ++q) acc[5][q] = make_float2(0.f, 0.f);
    }
    float en = 0.f;
    const float ex[4] = {eacc[0].x + D.E[6].x * kc[0], eacc[0].y + D.E[6].x * kc[1], eacc[1].x + D.E[6].x * kc[2],
                         eacc[1].y + D.E[6].x * kc[3]};
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        k7[i] = kc[i];
        k7[4 + i] = kc[4 + i];
        const float e = ht * ex[i] * rcp_(c.fatol + c.frtol * fabsf(float(xn[i])));
        en += e * e;
    }
    return double(sqrtp_(tmax(0.25f * en, 1e-30f)));
}

template <class T, int FAM = kAnyFamily>
__device__ __forceinline__ double dp45_attempt(const MetricDev& m, const CfgDev& c, const double x[4], const double p[4],
                                               double h, const T k1[8], double xn[4], double pn[4], T k7[8]) {
    if constexpr (std::is_same<T, float>::value) return dp45_attempt_x2<FAM>(m, c, x, p, h, k1, xn, pn, k7);
    const DPTable<T>& D = dp_table<T>();
    const T ht = T(h);
    T X[8];
#pragma unroll
    for (int i = 0; i < 4; ++i) { X[i] = T(x[i]); X[4 + i] = T(p[i]); }
    T acc[6][8];
    T eacc[4];
    T kc[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        kc[i] = k1[i];
#pragma unroll
        for (int s = 0; s < 6; ++s) acc[s][i] = T(0);
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) eacc[i] = T(0);
#pragma unroll 1
    for (int j = 0; j < 6; ++j) {
        // fold k_{j+1} into the inputs of every later stage, and into the error
#pragma unroll
        for (int s = 0; s < 6; ++s) {
            const T a = D.A[j][s];
#pragma unroll
            for (int i = 0; i < 8; ++i)
                if (i != 4) acc[s][i] += a * kc[i];
        }
        const T e = D.E[j];
#pragma unroll
        for (int i = 0; i < 4; ++i) eacc[i] += e * kc[i];
        T xs[4], ps[4];
        if (j == 5) {  // stage 7 is the solution point
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                xn[i] = x[i] + h * double(acc[0][i]);
                pn[i] = i == 0 ? p[0] : p[i] + h * double(acc[0][4 + i]);
                xs[i] = T(xn[i]);
                ps[i] = T(pn[i]);
            }
        } else {
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                xs[i] = X[i] + ht * acc[0][i];
                ps[i] = i == 0 ? X[4] : X[4 + i] + ht * acc[0][4 + i];
            }
        }
        rhs<T, FAM>(m, xs, ps, kc, kc + 4);
        // slide the window: the next stage's input moves to slot 0
#pragma unroll
        for (int s = 0; s < 5; ++s)
#pragma unroll
            for (int i = 0; i < 8; ++i)
                if (i != 4) acc[s][i] = acc[s + 1][i];
#pragma unroll
        for (int i = 0; i < 8; ++i) acc[5][i] = T(0);
    }
    T en = T(0);
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        k7[i] = kc[i];
        k7[4 + i] = kc[4 + i];
        const T ex = eacc[i] + D.E[6] * kc[i];
        if constexpr (sizeof(T) == sizeof(double)) {
            const double e = h * double(ex) / (c.atol + c.rtol * fabs(xn[i]));
            en += e * e;
        } else {  // the estimate needs a few digits only
            const float e = ht * ex * rcp_(c.fatol + c.frtol * fabsf(float(xn[i])));
            en += e * e;
        }
    }
    if constexpr (sizeof(T) == sizeof(double)) return sqrt(0.25 * en);
    else return double(sqrtp_(tmax(T(0.25) * en, T(1e-30))));  // 1e-15 when the estimate vanishes
}

// The same DP45 attempt in FP64 with the stage derivatives in a thread-local
// array indexed at run time (L1-resident local memory instead of registers): the
// rare FP64 island steps of the mixed path then do not set its register budget.
// Butcher form: stage s input = x + h sum_{j<s} a_sj k_j, with the tableau rows
// of DP_A read back as a_{s, j+1} = A[j][s-1-j].
template <int FAM = kAnyFamily>
__device__ __forceinline__ double dp45_attempt_lowreg(const MetricDev& m, const CfgDev& c, const double x[4],
                                                      const double p[4], double h, const double k1[8], double xn[4],
                                                      double pn[4], double k7[8]) {
    const DPTable<double>& D = kDPd;
    double K[7][8];
#pragma unroll
    for (int i = 0; i < 8; ++i) K[0][i] = k1[i];
#pragma unroll 1
    for (int s = 1; s < 7; ++s) {
        double sx[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) sx[i] = 0.0;
#pragma unroll 1
        for (int j = 0; j < s; ++j) {
            const double a = D.A[j][s - 1 - j];
#pragma unroll
            for (int i = 0; i < 8; ++i) sx[i] += a * K[j][i];
        }
        double xs[4], ps[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            xs[i] = x[i] + h * sx[i];
            ps[i] = p[i] + h * sx[4 + i];
        }
        if (s == 6) {
#pragma unroll
            for (int i = 0; i < 4; ++i) { xn[i] = xs[i]; pn[i] = ps[i]; }
        }
        rhs<double, FAM>(m, xs, ps, K[s], K[s] + 4);
    }
    double en = 0.0;
#pragma unroll 1
    for (int i = 0; i < 4; ++i) {
        double ex = 0.0;
#pragma unroll 1
        for (int j = 0; j < 7; ++j) ex += D.E[j] * K[j][i];
        const double e = h * ex / (c.atol + c.rtol * fabs(xn[i]));
        en += e * e;
    }
#pragma unroll
    for (int i = 0; i < 8; ++i) k7[i] = K[6][i];
    return sqrt(0.25 * en);
}

// Event location of the equatorial crossing inside an accepted step: DP45
// sub-steps from the step's start state (x0, p0) with f(x0, p0) recomputed in
// T, the sub-step length corrected by Newton on z(l) (dz/dl = k^z), seeded by
// the cubic Hermite root; two sub-steps and a final first-order correction.
// LOWREG (FP64 only) takes the sub-steps with the local-array attempt, for the
// mixed path's rare FP64 steps: with the register-resident attempt, the 48 FP64
// stage accumulators of this rare path set the mixed kernel's register count.
template <class T, int FAM = kAnyFamily, bool LOWREG = false>
__device__ __forceinline__ void locate_equator(const MetricDev& m, const CfgDev& c, const double x0[4],
                                            const double p0[4], double hs, double& xc1, double& xc2) {
    static_assert(!LOWREG || sizeof(T) == sizeof(double), "the low-register attempt is FP64");
    T xk[4], pk[4], k0[8], k7[8];
    for (int i = 0; i < 4; ++i) { xk[i] = T(x0[i]); pk[i] = T(p0[i]); }
    rhs<T, FAM>(m, xk, pk, k0, k0 + 4);
    double xn[4], pn[4];
    auto attempt = [&](double hh) {
        if constexpr (LOWREG) dp45_attempt_lowreg<FAM>(m, c, x0, p0, hh, k0, xn, pn, k7);
        else dp45_attempt<T, FAM>(m, c, x0, p0, hh, k0, xn, pn, k7);
    };
    attempt(hs);
    hs -= xn[3] / double(k7[3]);
    attempt(hs);
    const double dl = -xn[3] / double(k7[3]);
    xc1 = xn[1] + dl * double(k7[1]);
    xc2 = xn[2] + dl * double(k7[2]);
}

// The mixed path's event location: one FP32 DP45 sub-step of length hs from
// the step's start state with its stored f(x0, p0), then the first-order
// correction along k. FP32 stages bound the location at ~1e-7 relative, which a
// second sub-step would not improve.
template <int FAM = kAnyFamily>
__device__ __forceinline__ void locate_equator_f32(const MetricDev& m, const CfgDev& c, const double x0[4],
                                                const double p0[4], const float k0[8], double hs, double& xc1,
                                                double& xc2) {
    double xn[4], pn[4];
    float k7[8];
    dp45_attempt<float, FAM>(m, c, x0, p0, hs, k0, xn, pn, k7);
    const double dl = -xn[3] / double(k7[3]);
    xc1 = xn[1] + dl * double(k7[1]);
    xc2 = xn[2] + dl * double(k7[2]);
}

// Geodesic::computeOptimalStep (PHGD001A.cpp:471-483).
__device__ __forceinline__ double optimal_step(double h, double err, const CfgDev& c) {
    if (err < 1e-15) return fmin(h * c.grow, c.hmax);
    double fac = c.safety * pow(1.0 / err, 0.2);
    fac = fmax(c.shrink, fmin(c.grow, fac));
    return fmax(c.hmin, fmin(c.hmax, h * fac));
}

// ---------------------------------------------------------------------------
// Symplectic integration (SymplecticIntegratorD, PHSI001A.h:43-80, 136-215,
// 430-455) on H = 1/2 g^{mu nu} p_mu p_nu: a Yoshida composition (orders 4, 6,
// 8; Yoshida 1990) of the kick-drift-kick leapfrog
//   p += h/2 f(x, p);  x += h k(x, p);  p += h/2 f(x, p)
// (k = g^{-1} p, f = 1/2 d g k k). The three phases share one RHS call site;
// the right-hand sides run in T, the state accumulates in FP64.
// ---------------------------------------------------------------------------
static __constant__ double kYoshida[3][15] = {
    {1.3512071919596576, -1.7024143839193153, 1.3512071919596576},
    {0.78451361047756, 0.23557321335936, -1.17767998417887, 1.31518632068391, -1.17767998417887,
     0.23557321335936, 0.78451361047756},
    {0.74167036435061, -0.40910082580003, 0.19075471029623, -0.57386247111608, 0.29906418130365,
     0.33462491824529, 0.31529309239676, -0.79688793935291, 0.31529309239676, 0.33462491824529,
     0.29906418130365, -0.57386247111608, 0.19075471029623, -0.40910082580003, 0.74167036435061}};

template <class T, int FAM = kAnyFamily>
__device__ __forceinline__ void symplectic_step(const MetricDev& m, int order, double h, double x[4], double p[4]) {
    const int row = order >= 8 ? 2 : (order >= 6 ? 1 : 0);
    const int n = row == 2 ? 15 : (row == 1 ? 7 : 3);
#pragma unroll 1
    for (int s = 0; s < n; ++s) {
        const double hs = kYoshida[row][s] * h;
#pragma unroll 1
        for (int ph = 0; ph < 3; ++ph) {
            T X[4], P[4], k[4], f[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) { X[i] = T(x[i]); P[i] = T(p[i]); }
            rhs<T, FAM>(m, X, P, k, f);
            if (ph == 1) {
#pragma unroll
                for (int i = 0; i < 4; ++i) x[i] += hs * double(k[i]);
            } else {
#pragma unroll
                for (int i = 0; i < 4; ++i) p[i] += 0.5 * hs * double(f[i]);
            }
        }
    }
}

// The Kerr-Schild radius r(x, y, z) (r^4 - (R^2 - a^2) r^2 - a^2 z^2 = 0), FP64.
__device__ __forceinline__ double ks_radius(const MetricDev& m, const double x[4]) {
    const double R2 = x[1] * x[1] + x[2] * x[2] + x[3] * x[3], Rm2 = R2 - m.a2;
    const double sd = sqrt(fmax(Rm2 * Rm2 + 4.0 * m.a2 * x[3] * x[3], 1e-20));
    return sqrt(fmax(0.5 * (Rm2 + sd), 1e-10));
}

// Step control in FP32 for the mixed path (the factor needs a few digits only).
__device__ __forceinline__ double optimal_step_fast(double h, double err, const CfgDev& c) {
    if (err < 1e-15) return fmin(h * c.grow, c.hmax);
    float fac = c.fsafety * exp2f(-0.2f * __log2f(float(err)));
    fac = fmaxf(c.fshrink, fminf(c.fgrow, fac));
    return fmax(c.hmin, fmin(c.hmax, h * double(fac)));
}

// Gauss-Legendre points and weights on [0, 1] for n = 1..4 (Abramowitz & Stegun
// 25.4), ordered along the step: the volumetric quadrature of one step.
static __constant__ float kGLx[4][4] = {{0.5f, 0, 0, 0},
                                 {0.21132486540518713f, 0.78867513459481287f, 0, 0},
                                 {0.11270166537925831f, 0.5f, 0.88729833462074169f, 0},
                                 {0.069431844202973713f, 0.33000947820757187f, 0.66999052179242813f,
                                  0.93056815579702629f}};
static __constant__ float kGLw[4][4] = {{1.0f, 0, 0, 0},
                                 {0.5f, 0.5f, 0, 0},
                                 {0.27777777777777778f, 0.44444444444444444f, 0.27777777777777778f, 0},
                                 {0.17392742256872693f, 0.32607257743127307f, 0.32607257743127307f,
                                  0.17392742256872693f}};

// Emission beyond this many scale heights (e^-18 of the peak) is dropped.
constexpr double kVolCutoff = 6.0;

// Largest affine step near the emitting volume, so that the per-step
// quadrature, and hence the spectra, do not depend on the step sequence: half
// the local scale height hz r over the spatial speed |dx/dl| inside the emitting
// region (r_in <= r <= r_out, |z| <= kVolCutoff hz r), and outside it the
// distance to that region, so that no step jumps into its interior.
__device__ __forceinline__ double volume_step_cap(double r, double z, double vx, double vy, double vz, double hz,
                                                  double r_in, double r_out) {
    const double H = hz * fmin(fmax(r, r_in), r_out);
    const double dist = fmax(fmax(r_in - r, r - r_out), fabs(z) - kVolCutoff * H);
    const double v = sqrt(vx * vx + vy * vy + vz * vz);
    return fmax(0.5 * H, dist) / fmax(v, 1e-3);
}

// The same cap in FP32 for the mixed path (a step-size bound needs a few digits).
__device__ __forceinline__ float volume_step_cap_f(float r, float z, float vx, float vy, float vz, float hz,
                                                   float r_in, float r_out) {
    const float H = hz * fminf(fmaxf(r, r_in), r_out);
    const float dist = fmaxf(fmaxf(r_in - r, r - r_out), fabsf(z) - float(kVolCutoff) * H);
    return fmaxf(0.5f * H, dist) * rsqrtf(fmaxf(vx * vx + vy * vy + vz * vz, 1e-6f));
}

// Cubic Hermite interpolation of z over the accepted step; bisection for z = 0.
__device__ __forceinline__ double hermite_root(double z0, double z1, double dz0, double dz1, double h) {
    double lo = 0.0, hi = 1.0, flo = z0;
    for (int it = 0; it < 60; ++it) {
        const double s = 0.5 * (lo + hi), s2 = s * s, s3 = s2 * s;
        const double f = (2.0 * s3 - 3.0 * s2 + 1.0) * z0 + (s3 - 2.0 * s2 + s) * h * dz0 +
                         (-2.0 * s3 + 3.0 * s2) * z1 + (s3 - s2) * h * dz1;
        if ((f < 0.0) == (flo < 0.0)) { lo = s; flo = f; } else { hi = s; }
    }
    return 0.5 * (lo + hi);
}

// Keplerian emitter at BL radius rbl seen from the camera: g = (p.u_obs)/(p.u_em),
// u_em = u^t (d_t + Omega d_phi) with u^t from the Killing norms at the point
// (g_tt = -1 + H, g_t,phi = H (l.xi), g_phi,phi = x^2 + y^2 + H (l.xi)^2 in KS).
// rbl is the Kerr-Schild r of (x, y, z): H and l follow from it without derivatives.
template <class T>
__device__ __forceinline__ T kepler_g(const MetricDev& m, T x, T y, T z, T rbl, T E, T Lz, T sqrt_m_gtt_cam) {
    const T a = cst<T>(m.a, m.fa), a2 = cst<T>(m.a2, m.fa2), sqrtM = cst<T>(m.sqrtM, m.fsqrtM);
    const T r2 = rbl * rbl, iden = rcp_(r2 + a2);
    const T l1 = (rbl * x + a * y) * iden, l2 = (rbl * y - a * x) * iden;
    const T H = (cst<T>(2.0 * m.M, m.fM2) * rbl - cst<T>(m.Q2, m.fQ2)) * r2 * rcp_(r2 * r2 + a2 * z * z);
    const T lxi = -y * l1 + x * l2;
    T gtt = -T(1) + H;
    if (m.has_lambda) gtt -= cst<T>(m.lam3, m.flam3) * (x * x + y * y + z * z);
    const T gtp = H * lxi, gpp = x * x + y * y + H * lxi * lxi;
    const T Om = sqrtM * rcp_(rbl * sqrtp_(rbl) + a * sqrtM);
    const T n = -(gtt + T(2) * Om * gtp + Om * Om * gpp);
    if (!(n > T(0))) return T(0);
    const T ut = rsqrt_(n);
    const T den = sqrt_m_gtt_cam * ut * (T(1) - Om * Lz * rcp_(E));
    return den > T(0) ? rcp_(den) : T(0);
}

}  // namespace sirius

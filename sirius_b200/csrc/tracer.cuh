// tracer.cuh — the per-ray state machine of the trace kernels (device code
// shared by the translation units that instantiate them).
//
// trace_kernel<MIXED, MINB, FAM, UNI> is one thread per ray (or a persistent
// queue of rays) running GeodesicTracer::trace (GTRC001A.cpp:139-592) on the
// device: begin_ray initialises the ray from its pixel, advance takes one
// DP45 (or symplectic) step with the termination checks, end_ray writes the
// outputs. Each instantiation lives in one translation unit
// (trace_ks_mixed.cu, trace_ks_fp64.cu, trace_families.cu), so the library
// builds in parallel; engine.cu picks them through the pick_* functions.
#pragma once

#include <stdint.h>

#include <type_traits>

#include "packed.cuh"
#include "trace.cuh"

namespace sirius {
namespace eng {
constexpr unsigned kFull = 0xffffffffu;

constexpr unsigned kListSkip = 0xFFFFFFFFu;  // a list entry that names no ray

struct Params {
    const FrameDev* frames;
    int n_frames;
    long long total;
    sirius_ray_result* results;
    float* image;
    float* spectra;
    const sirius_camera_ray* host_rays;  // optional: explicit camera rays (device copy)
    const unsigned* list;                 // optional: trace only these ray indices (total = list length;
                                          // kListSkip entries are padding)
    const float* flux;                    // optional: per-frame disk flux tables (mixed path), kFluxN each
    unsigned long long* queue;            // [0] ray cursor
    unsigned long long* counters;         // [0] accepted, [1] rejected, [2] fp64 steps
    int* status;                          // [0] watchdog flag
    int persistent;
    int refill_threshold;
    int family;                           // >= 0: trace only the rays of frames of this family
    const int2* blocks;                   // multi-frame launch: per frame of the launch, x: its first block,
    int n_block_frames;                   // y: its index; a block traces one pixel tile of one frame
                                          // (tile_ray's layout, edge tiles cut by the frame)
    int tiled;                            // one-frame launch in pixel tiles: each warp traces an 8 x 4
                                          // pixel tile (tile_ray), edge tiles cut by the frame
    int block0;                           // tiled launch: the tile of block 0 (a launch of a run of tile rows)
    unsigned long long* clock0;           // launch start on the device clock (first warp stamps it)
    unsigned long long watchdog_ns;       // globaltimer bound for the whole launch, per warp
    CfgDev c;
    FrameDev f0;                          // the frame of a one-frame launch (read from the parameter bank)
};

// The frame of ray state s: a one-frame launch (UNI) reads it, metric included,
// from the kernel's parameter bank, whose constants the arithmetic takes as
// operands instead of loading them from global memory.
template <bool UNI>
__device__ __forceinline__ const FrameDev& frame_of(const Params& P, int frame) {
    if constexpr (UNI) return P.f0;
    else return P.frames[frame];
}

__device__ __forceinline__ unsigned long long globaltimer() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ int find_frame(const FrameDev* frames, int n, long long idx) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (frames[mid].ray_offset <= idx) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// Per-ray state held in registers between steps. K is the storage type of the
// first-same-as-last derivative f(x, p): float on the mixed path (the FP64
// island recomputes it in FP64), double on the all-FP64 path.
template <bool MIXED>
struct Ray {
    using K = typename std::conditional<MIXED, float, double>::type;
    double x[4], p[4];
    K k[8];
    double h;
    double intensity;
    float min_r, null_max, tphi, prev_z;
    float prev_r;  // r at the start of the step (volumetric early-out)
    int steps, rejected, attempts, ncross, eq, fp64_steps;
    int frame;
    int crit;  // mixed path: the ray skims the photon region, every step in FP64
    long long idx;
};

// Kerr-Newman radial potential of a null ray, R(r) = ((r^2+a^2) E - a L)^2 -
// Delta (Q + (L - a E)^2), Delta = r^2 - 2 M r + a^2 + Q_e^2: a double root marks
// the critical curve. Returns min R / (E^2 r^4) over the photon region
// r in [1.0001 r_+, 4.5 M] (48 samples).
__device__ __forceinline__ double radial_potential_gap(const MetricDev& m, double rp, double E, double L, double Q) {
    double best = 1e300;
    const double r0 = 1.0001 * rp, r1 = 4.5 * m.M;
    for (int i = 0; i < 48; ++i) {
        const double r = r0 + (r1 - r0) * (i / 47.0);
        const double A = (r * r + m.a2) * E - m.a * L;
        const double D = r * r - 2.0 * m.M * r + m.a2 + m.Q2;
        const double La = L - m.a * E;
        const double R = (A * A - D * (Q + La * La)) / (E * E * r * r * r * r);
        best = fmin(best, R);
    }
    return best;
}

__device__ __forceinline__ void write_default_crossings(sirius_ray_result* R) {
#pragma unroll
    for (int i = 0; i < SIRIUS_MAX_CROSSINGS; ++i) {
        R->disk_r[i] = 0.f; R->disk_phi[i] = 0.f; R->disk_g[i] = 1.f; R->disk_flux[i] = 0.f;
    }
}

static __device__ void invariants(const MetricDev& m, const InvForm& F, const double x[4], const double p[4], double& E,
                           double& Lz, double& Q) {
    E = -p[0];
    if (m.family == SIRIUS_METRIC_MORRIS_THORNE) {
        const double s = sin(x[2]), c = cos(x[2]);
        Lz = p[3];
        Q = p[2] * p[2] + c * c * p[3] * p[3] / (s * s);
        return;
    }
    const double L = x[1] * p[2] - x[2] * p[1];
    Lz = L;
    const double r = F.r;
    const double ct = fmin(fmax(x[3] / r, -1.0), 1.0);
    const double st = sqrt(fmax(1.0 - ct * ct, 1e-30));
    const double pth = (ct / st) * (x[1] * p[1] + x[2] * p[2]) - r * st * p[3];
    const double e = -p[0];
    Q = pth * pth + ct * ct * (-m.a2 * e * e + L * L / (st * st));
}

template <bool MIXED, int FAM, bool UNI>
__device__ __forceinline__ void begin_ray(const Params& P, Ray<MIXED>& s, long long idx, int frame, float2* vol) {
    using K = typename Ray<MIXED>::K;
    s.idx = idx;
    s.frame = frame;
    const FrameDev& F = frame_of<UNI>(P, s.frame);
    double dir[4];
    if (P.host_rays) {
        const sirius_camera_ray& cr = P.host_rays[idx];
        for (int i = 0; i < 4; ++i) dir[i] = cr.direction[i];
    } else {
        const long long pix = idx - F.ray_offset;
        camera_dir(F, int(pix % F.width), F.row0 + int(pix / F.width), dir);
    }
    init_state(F, dir, s.x, s.p);
    K xk[4], pk[4];
    for (int i = 0; i < 4; ++i) { xk[i] = K(s.x[i]); pk[i] = K(s.p[i]); }
    rhs<K, FAM>(F.m, xk, pk, s.k, s.k + 4);
    s.h = P.c.h0;
    s.intensity = 0.0;
    s.min_r = 1e10f;
    s.null_max = 0.f;
    s.tphi = 0.f;
    s.prev_z = float(s.x[3]);
    s.prev_r = float(ks_radius(F.m, s.x));
    s.steps = s.rejected = s.attempts = s.ncross = s.eq = s.fp64_steps = 0;
    s.crit = 0;
    if (MIXED && F.gate && P.c.crit_band > 0.0) {
        InvForm GF;
        inv_form(F.m, s.x, GF);
        double E, L, Q;
        invariants(F.m, GF, s.x, s.p, E, L, Q);
        s.crit = fabs(radial_potential_gap(F.m, F.r_plus, E, L, Q)) < P.c.crit_band;
    }
    if (P.results) {
        sirius_ray_result* R = P.results + idx;
        write_default_crossings(R);
        InvForm IF;
        inv_form(F.m, s.x, IF);
        double E, L, Q;
        invariants(F.m, IF, s.x, s.p, E, L, Q);
        R->E0 = E; R->Lz0 = L; R->Carter0 = Q;
        // impact parameter heuristic (GTRC001A.cpp:208-233)
        float b = 0.f;
        if (!is_family<FAM>(F.m, SIRIUS_METRIC_MORRIS_THORNE)) {
            const double k1 = double(s.k[1]), k2 = double(s.k[2]), k3 = double(s.k[3]);
            const double R0 = sqrt(s.x[1] * s.x[1] + s.x[2] * s.x[2] + s.x[3] * s.x[3]);
            const double vm = sqrt(k1 * k1 + k2 * k2 + k3 * k3);
            const double vrad = (k1 * s.x[1] + k2 * s.x[2] + k3 * s.x[3]) / R0;
            b = float(R0 * sqrt(fmax(vm * vm - vrad * vrad, 0.0)) / fmax(vm, 1e-10));
        }
        R->impact_parameter = b;
    }
    if (vol)
        for (int j = 0; j < P.c.npair; ++j) {
            vol[j * blockDim.x] = p2(0.f);
            vol[(P.c.npair + j) * blockDim.x] = p2(1.f);
        }
}

template <bool MIXED, bool UNI>
__device__ __forceinline__ void end_ray(const Params& P, const Ray<MIXED>& s, int outcome, float magnification, int flags,
                                     const float2* vol) {
    const FrameDev& F = frame_of<UNI>(P, s.frame);
    if (P.image) P.image[s.idx] = float(s.intensity);
    if (P.spectra && vol)
        for (int b = 0; b < P.c.nbins; ++b) {
            const float2 I = vol[(b >> 1) * blockDim.x];
            P.spectra[s.idx * P.c.nbins + b] = (b & 1) ? I.y : I.x;
        }
    if (!P.results) return;
    sirius_ray_result* R = P.results + s.idx;
    InvForm IF;
    inv_form(F.m, s.x, IF);
    double E, L, Q;
    invariants(F.m, IF, s.x, s.p, E, L, Q);
    R->outcome = outcome;
    R->steps = s.steps;
    R->rejected = s.rejected;
    R->n_crossings = s.ncross;
    for (int i = 0; i < 4; ++i) {
        R->final_x[i] = s.x[i];
        R->final_p[i] = s.p[i];
        R->final_k[i] = float(s.k[i]);
    }
    R->equatorial_crossings = s.eq;
    R->image_order = s.eq >= 1 ? (s.eq + 1) / 2 : 0;
    R->total_phi_change = s.tphi;
    R->min_radius = s.min_r;
    R->intensity = float(s.intensity);
    R->E = E; R->Lz = L; R->Carter = Q;
    R->null_drift_max = s.null_max;
    R->null_final = float(fabs(inv_apply(F.m, IF, s.p, s.p)));
    R->magnification = magnification;
    float tmin = 1.f;
    if (vol)
        for (int b = 0; b < P.c.nbins; ++b) {
            const float2 T = vol[(P.c.npair + (b >> 1)) * blockDim.x];
            tmin = fminf(tmin, (b & 1) ? T.y : T.x);
        }
    R->optical_depth = tmin > 0.f ? -logf(tmin) : 1e30f;
    R->fp64_steps = s.fp64_steps;
    R->flags = flags;
}

// A point of the step's cubic Hermite interpolant at parameter q in [0, 1].
__device__ __forceinline__ void hermite_xyz(const double x0[4], const double x1[4], const float k0[4],
                                            const float k1[4], double h, double q, float& xs, float& ys, float& zs) {
    const double q2 = q * q, q3 = q2 * q;
    const double h00 = 2.0 * q3 - 3.0 * q2 + 1.0, h10 = (q3 - 2.0 * q2 + q) * h, h01 = -2.0 * q3 + 3.0 * q2,
                 h11 = (q3 - q2) * h;
    xs = float(h00 * x0[1] + h10 * k0[1] + h01 * x1[1] + h11 * k1[1]);
    ys = float(h00 * x0[2] + h10 * k0[2] + h01 * x1[2] + h11 * k1[2]);
    zs = float(h00 * x0[3] + h10 * k0[3] + h01 * x1[3] + h11 * k1[3]);
}

__device__ __forceinline__ float ks_r(const MetricDev& m, float x, float y, float z) {
    const float a2 = m.fa2, R2 = x * x + y * y + z * z, Rm2 = R2 - a2;
    const float sd = sqrtp_(fmaxf(Rm2 * Rm2 + 4.f * a2 * z * z, 1e-20f));
    return sqrtp_(fmaxf(0.5f * (Rm2 + sd), 1e-10f));
}

// A point of the step's cubic Hermite interpolant at parameter q in [0, 1], in
// FP32 relative to the step's start: x(q) = x0 + h10 k0 + h01 (x1 - x0) + h11 k1
// (the mixed path; the step is short against |x0|, so the offset carries the
// digits that matter).
__device__ __forceinline__ void hermite_xyz_f(const float x0[3], const float dx[3], const float k0[4],
                                              const float k1[4], float h, float q, float& xs, float& ys, float& zs) {
    const float q2 = q * q, q3 = q2 * q;
    const float h10 = (q3 - 2.f * q2 + q) * h, h01 = 3.f * q2 - 2.f * q3, h11 = (q3 - q2) * h;
    xs = x0[0] + (h10 * k0[1] + h01 * dx[0] + h11 * k1[1]);
    ys = x0[1] + (h10 * k0[2] + h01 * dx[1] + h11 * k1[2]);
    zs = x0[2] + (h10 * k0[3] + h01 * dx[2] + h11 * k1[3]);
}

// |b| (base-2 exponent of a bin's optical depth) below which the series alone
// is the bin's 1 - e^-x: x = |b| ln 2 < 0.04
constexpr float kSeriesOnlyB = 0.04f / 0.693147180559945309f;

// Volumetric transfer over the accepted segment x0 -> x1 (affine length h):
// Gauss-Legendre points on the step's cubic Hermite interpolant (the reference
// marches the chord with midpoints, GTRC001A.cpp:943-958) over the part of the
// step inside the emitting annulus r_in <= r <= r_out (its edges, where j jumps,
// are located by regula falsi), camera-first accumulation per bin:
// I_b += T_b S (1 - e^-dtau), T_b = e^-tau_b,
//   j = j0 r^-2 exp(-z^2/(2 (h_z r)^2)) nu_em^-s, alpha = c_a j,
//   dtau = alpha (nu_cam/g) dl, S = g^3 / c_a.
// The bins are updated in pairs with packed FP32 arithmetic: vol[j * blockDim]
// holds (I_2j, I_2j+1), vol[(npair + j) * blockDim] (T_2j, T_2j+1). MIXED
// evaluates the interpolant in FP32 (hermite_xyz_f); the FP64 path in FP64.
template <bool MIXED>
__device__ __forceinline__ void volumetric_segment(const Params& P, const FrameDev& F, const double x0[4],
                                                const double x1[4], const float k0[4], const float k1[4],
                                                const double p[4], double h, float r0, float r1, float2* vol) {
    const CfgDev& c = P.c;
    const int nq = c.vol_sub < 1 ? 1 : (c.vol_sub > 4 ? 4 : c.vol_sub);
    const float E = float(-p[0]);
    const float Lz = float(x1[1] * p[2] - x1[2] * p[1]);
    const float nu_cam = E / observer_factor<float>(F, E);
    const float rin = F.fdisk_in, rout = F.fdisk_out;
    const bool in0 = r0 >= rin && r0 <= rout, in1 = r1 >= rin && r1 <= rout;
    float xf0[3], dxf[3];
    if constexpr (MIXED) {
#pragma unroll
        for (int i = 0; i < 3; ++i) { xf0[i] = float(x0[i + 1]); dxf[i] = float(x1[i + 1] - x0[i + 1]); }
    }
    auto point = [&](double q, float& xs, float& ys, float& zs) {
        if constexpr (MIXED) hermite_xyz_f(xf0, dxf, k0, k1, float(h), float(q), xs, ys, zs);
        else hermite_xyz(x0, x1, k0, k1, h, q, xs, ys, zs);
    };
    double fa = 0.0, fb = 1.0;
    if (in0 != in1) {
        // the annulus edge on the step's Hermite interpolant: regula falsi
        // (Illinois) on r(q) - edge over [0, 1], three evaluations
        const float edge = in0 ? (r1 < rin ? rin : rout) : (r0 < rin ? rin : rout);
        double qa = 0.0, qb = 1.0, ga = double(r0) - edge, gb = double(r1) - edge;
        int side = 0;
        for (int it = 0; it < 3; ++it) {
            const double q = (qa * gb - qb * ga) / (gb - ga);
            float xs, ys, zs;
            point(q, xs, ys, zs);
            const double g = double(ks_r(F.m, xs, ys, zs)) - edge;
            if ((g < 0.0) == (ga < 0.0)) {
                qa = q; ga = g;
                if (side == -1) gb *= 0.5;
                side = -1;
            } else {
                qb = q; gb = g;
                if (side == 1) ga *= 0.5;
                side = 1;
            }
        }
        const double qe = (qa * gb - qb * ga) / (gb - ga);
        if (in0) fb = qe;
        else fa = qe;
    }
    const double span = fb - fa;
    const unsigned bd = blockDim.x;
    // 1 - e^-x of two bins from b = -x / ln 2 (the bins' exponents in base 2):
    // the smaller of the three-term series x - x^2/2 + x^3/6 (an upper bound,
    // too large by < x^4/24) and 1 - k 2^b, k = 1 - 2^-20 (1 - e^-x plus a bias
    // of 2^-20 e^-x that covers the rounding of the hardware 2^b, so the series
    // wins wherever x^4/24 is below that bias, x < 0.06). The result lies in
    // (0, 1], with a relative error below 2e-5 at every x.
    constexpr float L = 0.693147180559945309f, L2h = 0.240226506959100712f,  // ln 2, ln^2 2 / 2
        L3s = 0.0555041086648215800f;                                          // ln^3 2 / 6
    auto series = [&](float2 b) {
        const float2 u = fma2(b, p2(-L3s), p2(-L2h));
        return mul2(b, fma2(b, u, p2(-L)));
    };
    auto one_minus_exp = [&](float2 b) {
        const float2 ser = series(b);
        const float2 e = fma2(make_float2(ex2_approx(b.x), ex2_approx(b.y)), p2(-(1.f - 0x1p-20f)), p2(1.f));
        return make_float2(fminf(ser.x, e.x), fminf(ser.y, e.y));
    };
    auto point_at = [&](int s, float& dts, float& Ss) {
        dts = 0.f;
        Ss = 0.f;
        float xs, ys, zs;
        point(fa + span * double(kGLx[nq - 1][s]), xs, ys, zs);
        const float r = ks_r(F.m, xs, ys, zs);
        if (r < rin || r > rout) return;
        const float zr = zs / (c.fvol_hz * r);
        if (fabsf(zr) > float(kVolCutoff)) return;
        const float g = kepler_g<float>(F.m, xs, ys, zs, r, E, Lz, observer_factor<float>(F, E));
        if (!(g > 0.f)) return;
        const float dl = float(h * span) * kGLw[nq - 1][s];
        const float jsp = c.fvol_j0 / (r * r) * __expf(-0.5f * zr * zr);
        const float gs = __powf(g, c.fvol_s);  // nu_em^-s = (g/nu_b)^s
        dts = c.fvol_aoj * jsp * gs * (nu_cam / g) * dl;
        Ss = g * g * g / c.fvol_aoj;
    };
    // the Gauss-Legendre points in step order, each applied to every bin pair
    // (a point outside the emitting region, or with no redshift, leaves the bins
    // as they are)
#pragma unroll 1
    for (int s = 0; s < nq; ++s) {
        float dts, Ss;
        point_at(s, dts, Ss);
        if (dts == 0.f) continue;
        const float2 dt0 = p2(dts), S = p2(Ss);
        // bins in order of falling optical depth (c.nu_desc): once a pair's deeper
        // bin is below x = 0.04, where the minimum above is the series, every
        // later pair takes the series alone (the same values, no exponentials)
        int j = 0;
#pragma unroll 1
        for (; j < c.npair; ++j) {
            const float2 b = mul2(dt0, c.nu_l2[j]);
            if (c.nu_desc && b.x > -kSeriesOnlyB) break;
            const float2 I = vol[j * bd];
            const float2 T = vol[(c.npair + j) * bd];  // transmittance e^-tau to the camera
            const float2 om = one_minus_exp(b);
            vol[j * bd] = fma2(mul2(T, S), om, I);
            vol[(c.npair + j) * bd] = fma2(neg2(T), om, T);
        }
#pragma unroll 1
        for (; j < c.npair; ++j) {
            const float2 I = vol[j * bd];
            const float2 T = vol[(c.npair + j) * bd];
            const float2 om = series(mul2(dt0, c.nu_l2[j]));
            vol[j * bd] = fma2(mul2(T, S), om, I);
            vol[(c.npair + j) * bd] = fma2(neg2(T), om, T);
        }
    }
}

// A disk crossing at the event-located point (xc1, xc2, 0): BL radius, exact
// redshift with the ray's conserved E and L_z (from the state x, p), flux.
// Returns true when the crossing lies on the disk (GTRC001A.cpp:468-555).
// Per-frame table of the Page-Thorne flux for the mixed path: kFluxN samples
// at u = sqrt((r - r_in) / (r_out - r_in)) in [0, 1] (F ~ (r - r_ISCO) near the
// inner edge is smooth in u), read by cubic Lagrange interpolation, followed by
// kFluxN cell flags. The flux as the reference defines it switches to an
// approximate form where the full expression is not positive (PHAD001A.h:321-361),
// which leaves a kink; a cell whose interpolant misses the exact flux at its
// midpoint by more than 1e-6 (relative) is flagged, and a crossing there
// evaluates the 16-point quadrature itself, as the FP64 path does everywhere.
constexpr int kFluxN = 256;
constexpr int kFluxTable = 2 * kFluxN;  // floats per frame: samples, then cell flags

__device__ __forceinline__ double flux_cubic(const float* t, double x) {
    int j = int(x) - 1;
    j = j < 0 ? 0 : (j > kFluxN - 4 ? kFluxN - 4 : j);
    const double f = x - j;  // position within the samples j..j+3, in [0, 3]
    const double w0 = -(f - 1.0) * (f - 2.0) * (f - 3.0) / 6.0, w1 = f * (f - 2.0) * (f - 3.0) / 2.0,
                 w2 = -f * (f - 1.0) * (f - 3.0) / 2.0, w3 = f * (f - 1.0) * (f - 2.0) / 6.0;
    return w0 * t[j] + w1 * t[j + 1] + w2 * t[j + 2] + w3 * t[j + 3];
}


__device__ __forceinline__ double flux_lookup(const float* t, const FrameDev& F, double r) {
    const double u = sqrt(fmin(fmax((r - F.disk_in) / (F.disk_out - F.disk_in), 0.0), 1.0));
    const double x = u * (kFluxN - 1);
    const int cell = min(int(x), kFluxN - 2);
    if (t[kFluxN + cell] != 0.f) return nt_flux(r, F.a_star, F.isco, F.disk_in, F.disk_out);
    return flux_cubic(t, x);
}

struct Vec4v {
    double v[4];
};

// (out of line: rare, and its flux fallback is long)
static __device__ __noinline__ double record_crossing(const Params& P, const FrameDev& F, long long idx, int n, double xc1,
                                               double xc2, const Vec4v xv, const Vec4v pv) {
    const double* x = xv.v;
    const double* p = pv.v;
    const MetricDev& m = F.m;
    const double xc[4] = {0.0, xc1, xc2, 0.0};
    InvForm CF;
    inv_form(m, xc, CF);
    const double rc = CF.r;
    if (!(rc >= F.disk_in && rc <= F.disk_out)) return -1.0;
    const double E = -p[0], Lz = x[1] * p[2] - x[2] * p[1];
    const double g = kepler_g<double>(m, xc1, xc2, 0.0, rc, E, Lz, observer_factor<double>(F, E));
    const double Fl = P.flux ? flux_lookup(P.flux + size_t(F.flux_slot) * kFluxTable, F, rc)
                             : nt_flux(rc, F.a_star, F.isco, F.disk_in, F.disk_out);
    const double dI = exp(-P.c.decay * n) * g * g * g * g * Fl;
    if (P.results) {
        sirius_ray_result* R = P.results + idx;
        R->disk_r[n] = float(rc);
        R->disk_phi[n] = float(atan2(xc2, xc1));
        R->disk_g[n] = float(g);
        R->disk_flux[n] = float(Fl);
    }
    return dI;
}

// The FP64 island of the mixed path is large and rare, so it stays out of line
// (less code in the hot loop). Its arguments and results travel by value: an
// array passed by address would pin the caller's ray state in local memory.
struct IslandStep {
    double xn[4], pn[4];
    float k7[8];
    double err;
};
struct CrossXY {
    double x, y;
};

__device__ __forceinline__ Vec4v vec4v(const double a[4]) { return Vec4v{{a[0], a[1], a[2], a[3]}}; }

// The FP64 island attempt: f(x, p) recomputed in FP64, a DP45 attempt in FP64;
// the derivative at the candidate point returned in float for the FP32 steps
// that may follow.
template <int FAM>
__device__ __noinline__ IslandStep island_attempt(const MetricDev& m, const CfgDev& c, const Vec4v x, const Vec4v p,
                                                  double h) {
    IslandStep o;
    double k1[8], k7[8];
    rhs<double, FAM>(m, x.v, p.v, k1, k1 + 4);
    o.err = dp45_attempt_lowreg<FAM>(m, c, x.v, p.v, h, k1, o.xn, o.pn, k7);
#pragma unroll
    for (int i = 0; i < 8; ++i) o.k7[i] = float(k7[i]);
    return o;
}

// The equatorial crossing of an accepted island step, located in FP64.
template <int FAM>
__device__ __noinline__ CrossXY island_crossing(const MetricDev& m, const CfgDev& c, const Vec4v x, const Vec4v p,
                                                double hs) {
    CrossXY o;
    locate_equator<double, FAM, true>(m, c, x.v, p.v, hs, o.x, o.y);
    return o;
}

// The mixed path's equatorial crossing, located from the step's start state
// with one FP32 sub-step (out of line: it carries its own DP45 attempt).
struct K8f {
    float v[8];
};
template <int FAM>
__device__ __noinline__ CrossXY crossing_f32(const MetricDev& m, const CfgDev& c, const Vec4v x, const Vec4v p,
                                             const K8f k, double hs) {
    CrossXY o;
    locate_equator_f32<FAM>(m, c, x.v, p.v, k.v, hs, o.x, o.y);
    return o;
}

// f(x, p) of the current state in the storage precision of the path.
template <bool MIXED, int FAM>
__device__ __forceinline__ void refresh_derivative(const MetricDev& m, Ray<MIXED>& s) {
    using K = typename Ray<MIXED>::K;
    K xk[4], pk[4];
    for (int i = 0; i < 4; ++i) { xk[i] = K(s.x[i]); pk[i] = K(s.p[i]); }
    rhs<K, FAM>(m, xk, pk, s.k, s.k + 4);
}

// INT selects the integrator at compile time (SIRIUS_INTEGRATOR_DP45 or
// _SYMPLECTIC: the kernel carries one), or kAnyIntegrator (the configuration's).
constexpr int kAnyIntegrator = -1;
template <int INT>
__device__ __forceinline__ bool is_symplectic(const CfgDev& c) {
    if constexpr (INT == kAnyIntegrator) return c.integrator == SIRIUS_INTEGRATOR_SYMPLECTIC;
    else return INT == SIRIUS_INTEGRATOR_SYMPLECTIC;
}

template <bool MIXED, int FAM, bool UNI, int INT>
__device__ __forceinline__ int advance_post(const Params& P, Ray<MIXED>& s, bool island, const double xn[4],
                                            const double pn[4], const typename Ray<MIXED>::K k7[8], double err,
                                            float& magnification, int& flags, float2* vol);

// The volumetric step cap at radius r, height z, spatial velocity k[1..3]: FP32
// on the mixed path, FP64 on the FP64 path.
template <bool MIXED, class K>
__device__ __forceinline__ double vol_cap(double r, double z, const K k[8], const CfgDev& c, const FrameDev& F) {
    if constexpr (MIXED)
        return double(volume_step_cap_f(float(r), float(z), float(k[1]), float(k[2]), float(k[3]), c.fvol_hz,
                                        F.fdisk_in, F.fdisk_out));
    else
        return volume_step_cap(r, z, double(k[1]), double(k[2]), double(k[3]), c.vol_hz, F.disk_in, F.disk_out);
}

// One iteration of the ray state machine: a DP45 attempt, and on acceptance
// the termination checks. Returns -1 while the ray continues, else its outcome.
template <bool MIXED, int FAM, bool UNI, int INT>
__device__ __forceinline__ int advance(const Params& P, Ray<MIXED>& s, float& magnification, int& flags, float2* vol) {
    using K = typename Ray<MIXED>::K;
    const FrameDev& F = frame_of<UNI>(P, s.frame);
    const MetricDev& m = F.m;
    const CfgDev& c = P.c;
    double xn[4], pn[4];
    K k7[8];
    bool island = true;
    double err;
    if constexpr (MIXED) {
        // FP64 island: inside island_factor * r_ph (retrograde) or near the horizon
        const double R2 = s.x[1] * s.x[1] + s.x[2] * s.x[2] + s.x[3] * s.x[3];
        island = s.crit ||
                 (is_family<FAM>(m, SIRIUS_METRIC_MORRIS_THORNE) ? (s.x[1] < F.island_r)
                                                                 : (R2 < F.island_r * F.island_r));
    }
    const bool symp = is_symplectic<INT>(c);
    if (symp) {
        // fixed d-lambda, shrunk near the horizon as SymplecticIntegratorD::integrate
        // does (h0 min(1, ((r - r_+)/r_+)^2), PHSI001A.h:260-263); always accepted
        double hs = c.symp_step;
        if (F.has_horizon) {
            const double q = (ks_radius(m, s.x) - F.r_plus) / F.r_plus;
            hs = fmax(c.hmin, hs * fmin(1.0, q * q));
        }
        s.h = hs;
#pragma unroll
        for (int i = 0; i < 4; ++i) { xn[i] = s.x[i]; pn[i] = s.p[i]; }
        if (MIXED && !island) symplectic_step<float, FAM>(m, c.symp_order, hs, xn, pn);
        else symplectic_step<double, FAM>(m, c.symp_order, hs, xn, pn);
        K xk[4], pk[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) { xk[i] = K(xn[i]); pk[i] = K(pn[i]); }
        rhs<K>(m, xk, pk, k7, k7 + 4);
        err = 0.0;
    } else if constexpr (MIXED) {
        if (island) {
            const IslandStep o = island_attempt<FAM>(m, c, vec4v(s.x), vec4v(s.p), s.h);
#pragma unroll
            for (int i = 0; i < 4; ++i) { xn[i] = o.xn[i]; pn[i] = o.pn[i]; }
#pragma unroll
            for (int i = 0; i < 8; ++i) k7[i] = o.k7[i];
            err = o.err;
        } else {
            err = dp45_attempt<float, FAM>(m, c, s.x, s.p, s.h, s.k, xn, pn, k7);
        }
    } else {
        err = dp45_attempt<double, FAM>(m, c, s.x, s.p, s.h, s.k, xn, pn, k7);
    }
    return advance_post<MIXED, FAM, UNI, INT>(P, s, island, xn, pn, k7, err, magnification, flags, vol);
}

// The rest of one iteration after the attempt: on rejection the step-size
// update; on acceptance the event location of a disk crossing, the constraint
// re-projection and the termination checks (GeodesicTracer::trace's order,
// GTRC001A.cpp:264-556), the volumetric segment and the crossing record.
// (xn, pn, k7, err) is the attempt from s's state; island: it ran in FP64.
template <bool MIXED, int FAM, bool UNI, int INT>
__device__ __forceinline__ int advance_post(const Params& P, Ray<MIXED>& s, bool island, const double xn[4],
                                            const double pn[4], const typename Ray<MIXED>::K k7[8], double err,
                                            float& magnification, int& flags, float2* vol) {
    using K = typename Ray<MIXED>::K;
    const FrameDev& F = frame_of<UNI>(P, s.frame);
    const MetricDev& m = F.m;
    const CfgDev& c = P.c;
    const bool symp = is_symplectic<INT>(c);
    ++s.attempts;
    if (!(err <= 1.0)) {
        ++s.rejected;
        s.h = MIXED ? optimal_step_fast(s.h, isfinite(err) ? err : 1e10, c)
                    : optimal_step(s.h, isfinite(err) ? err : 1e10, c);
        if (c.enable_vol && c.enable_disk && F.has_horizon && is_family<FAM>(m, SIRIUS_METRIC_KERR_SCHILD)) {
            InvForm RF;
            inv_form(m, s.x, RF);
            s.h = fmax(c.hmin, fmin(s.h, vol_cap<MIXED>(RF.r, s.x[3], s.k, c, F)));
        }
        if (s.h <= c.hmin) { ++s.steps; return SIRIUS_STEP_UNDERFLOW; }
        if (s.attempts > c.max_steps * 64 + 1024) return SIRIUS_STEP_UNDERFLOW;
        return -1;
    }
    // accepted
    const double hstep = s.h;
    const bool disk_on = is_family<FAM>(m, SIRIUS_METRIC_KERR_SCHILD) && c.enable_disk && F.has_horizon;
    // equatorial crossing inside the step: locate it from the step's start state
    double xc1 = 0.0, xc2 = 0.0;
    bool cross = disk_on && (s.x[3] * xn[3] < 0.0);
    if (cross) {
        // a crossing that cannot land on the disk needs no location: the chord's
        // crossing point lies within three step lengths of the trajectory's, so
        // Boyer-Lindquist radii (r^2 = x^2 + y^2 - a^2 at z = 0) outside
        // [r_in, r_out] by that margin would fail the disk test in any case
        const float t = float(s.x[3] / (s.x[3] - xn[3]));
        const float dx = float(xn[1] - s.x[1]), dy = float(xn[2] - s.x[2]), dz = float(xn[3] - s.x[3]);
        const float cx = float(s.x[1]) + t * dx, cy = float(s.x[2]) + t * dy;
        const float rho = sqrtp_(fmaxf(cx * cx + cy * cy, 1e-30f));
        const float L3 = 3.f * sqrtp_(fmaxf(dx * dx + dy * dy + dz * dz, 1e-30f));
        const float a2 = m.fa2, rhi = rho + L3, rlo = fmaxf(rho - L3, 0.f);
        if (rlo * rlo - a2 > F.fdisk_out * F.fdisk_out * 1.0001f || rhi * rhi - a2 < F.fdisk_in * F.fdisk_in * 0.9999f)
            cross = false;
    }
    if (cross) {
        const double hs = hermite_root(s.x[3], xn[3], double(s.k[3]), double(k7[3]), hstep) * hstep;
        if constexpr (MIXED) {
            if (island) {
                const CrossXY o = island_crossing<FAM>(m, c, vec4v(s.x), vec4v(s.p), hs);
                xc1 = o.x;
                xc2 = o.y;
            }
            else {
                K8f k0;
#pragma unroll
                for (int i = 0; i < 8; ++i) k0.v[i] = float(s.k[i]);
                const CrossXY o = crossing_f32<FAM>(m, c, vec4v(s.x), vec4v(s.p), k0, hs);
                xc1 = o.x;
                xc2 = o.y;
            }
        } else {
            locate_equator<double, FAM>(m, c, s.x, s.p, hs, xc1, xc2);
        }
    }
    double x0[4];
    float k0f[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) { x0[i] = s.x[i]; k0f[i] = float(s.k[i]); }
    if (!symp) s.h = MIXED ? optimal_step_fast(s.h, err, c) : optimal_step(s.h, err, c);
    ++s.steps;
    if (MIXED && island) ++s.fp64_steps;
    // a NaN or infinity in any component survives the sums (inf - inf is NaN)
    const double sx = ((xn[0] + xn[1]) + (xn[2] + xn[3])) + ((pn[0] + pn[1]) + (pn[2] + pn[3]));
    const K sk = (k7[0] + k7[1]) + (k7[2] + k7[3]);
    const bool bad = !isfinite(sx) || !isfinite(sk);
#pragma unroll
    for (int i = 0; i < 4; ++i) { s.x[i] = xn[i]; s.p[i] = pn[i]; }
#pragma unroll
    for (int i = 0; i < 8; ++i) s.k[i] = k7[i];
    if (bad) { flags |= SIRIUS_FLAG_NUMERICAL_FAILURE; return SIRIUS_NUMERICAL_FAILURE; }

    // constraint re-projection (E, L_z and Carter preserving); the mixed path
    // forms only the null value in FP64 (Kerr-Schild without Lambda)
    double rr;
    const bool project = c.proj_period > 0 && (s.steps % c.proj_period) == 0;
    const bool ks_fast = MIXED && is_family<FAM>(m, SIRIUS_METRIC_KERR_SCHILD) && !m.has_lambda;
    if (project) {
        double pb[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) pb[i] = s.p[i];
        double before;
        if (ks_fast) {
            before = project_null_ks_mixed(m, s.x, s.p, rr);
        } else {
            InvForm IF;
            inv_form(m, s.x, IF);
            rr = IF.r;
            before = project_null(m, IF, s.p);
        }
        s.null_max = fmaxf(s.null_max, float(fabs(before)));
        // a projection that moved p beyond what the stored f(x, p) resolves
        // (1e-10 relative in FP64, 1e-6 with FP32 storage) makes it stale: recompute it
        double dp = 0.0, pm = 0.0;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            dp = fmax(dp, fabs(s.p[i] - pb[i]));
            pm = fmax(pm, fabs(s.p[i]));
        }
        if (dp > (MIXED ? 1e-6 : 1e-10) * pm) refresh_derivative<MIXED, FAM>(m, s);
    } else if (ks_fast) {
        rr = ks_radius(m, s.x);
    } else {
        InvForm IF;
        inv_form(m, s.x, IF);
        rr = IF.r;
    }
    if (float(rr) < s.min_r) s.min_r = float(rr);
    if (disk_on && c.enable_vol && !symp)
        s.h = fmax(c.hmin, fmin(s.h, vol_cap<MIXED>(rr, s.x[3], s.k, c, F)));
    const bool mt = is_family<FAM>(m, SIRIUS_METRIC_MORRIS_THORNE);

    // winding: equatorial crossings and |d phi| (GTRC001A.cpp:294-309); the
    // azimuth sum feeds the spiral check and the per-ray record only
    if (!mt) {
        const float cz = float(s.x[3]);
        if (s.prev_z * cz < 0.f) ++s.eq;
        s.prev_z = cz;
        if (c.spiral || P.results) {
            const float cr = float(x0[1] * s.x[2] - x0[2] * s.x[1]);
            const float dt = float(x0[1] * s.x[1] + x0[2] * s.x[2]);
            s.tphi += fabsf(atan2f(cr, dt));
        }
    }
    // spiral early-out (GTRC001A.cpp:322-352)
    const int sidx = s.steps - 1;
    if (c.spiral && !mt && (sidx % 100) == 0 && sidx > 100) {
        const float ratio = s.min_r / F.fr_ph_pro;
        if (ratio < 1.5f && ratio > 0.9f && s.tphi > 2.f * float(kPi)) {
            const double k1 = double(s.k[1]), k2 = double(s.k[2]), k3 = double(s.k[3]);
            const double Reu = sqrt(s.x[1] * s.x[1] + s.x[2] * s.x[2] + s.x[3] * s.x[3]);
            const double vrad = (s.x[1] * k1 + s.x[2] * k2 + s.x[3] * k3) / Reu;
            const double vt = sqrt(k1 * k1 + k2 * k2 + k3 * k3);
            if (fabs(vrad) / fmax(vt, 1e-10) < 0.3) return s.ncross > 0 ? SIRIUS_DISK_HIT : SIRIUS_SPIRALING;
        }
    }
    // horizon
    if (F.r_hor > 0.0 && rr < F.r_hor) return SIRIUS_HORIZON;
    // throat
    if (mt && s.x[1] <= 1.001 * m.b0 * 1.0001) return SIRIUS_THROAT;
    // escape
    {
        const double R2e = mt ? s.x[1] * fabs(s.x[1]) : s.x[1] * s.x[1] + s.x[2] * s.x[2] + s.x[3] * s.x[3];
        if (R2e > c.escape_r * c.escape_r) {
            const double vrad = mt ? double(s.k[1])
                                   : (s.x[1] * double(s.k[1]) + s.x[2] * double(s.k[2]) + s.x[3] * double(s.k[3]));
            if (vrad > 0.0) {
                const float ratio = s.min_r / F.fr_ph_pro;
                if (ratio < 1.5f) {
                    flags |= SIRIUS_FLAG_PHOTON_RING;
                    magnification = ratio > 1.f ? fminf(1.f + 2.f / fmaxf(ratio - 1.f, 0.1f), 20.f) : 20.f;
                }
                return s.ncross > 0 ? SIRIUS_DISK_HIT : SIRIUS_ESCAPED;
            }
        }
    }
    if (!disk_on) return s.steps >= c.max_steps ? (s.ncross > 0 ? SIRIUS_DISK_HIT : SIRIUS_MAX_STEPS) : -1;
    if (c.enable_vol && vol) {
        // steps that cannot reach the emitting region skip the segment (the
        // step cap keeps a step that starts outside it from jumping in)
        const float r0 = s.prev_r, r1 = float(rr), rin = F.fdisk_in, rout = F.fdisk_out;
        const float zc = float(kVolCutoff * c.vol_hz), z0 = float(x0[3]), z1 = float(s.x[3]);
        const bool beyond = (r0 > rout && r1 > rout) ||
                            (z0 * z1 > 0.f && fabsf(z0) > zc * fminf(fmaxf(r0, rin), rout) &&
                             fabsf(z1) > zc * fminf(fmaxf(r1, rin), rout));
        if (!beyond) {
            float k1f[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) k1f[i] = float(s.k[i]);
            volumetric_segment<MIXED>(P, F, x0, s.x, k0f, k1f, s.p, hstep, r0, r1, vol);
        }
    }
    s.prev_r = float(rr);
    // thin-disk crossing (GTRC001A.h:404-431, GTRC001A.cpp:468-555)
    if (cross && s.ncross < SIRIUS_MAX_CROSSINGS) {
        const double dI = record_crossing(P, F, s.idx, s.ncross, xc1, xc2, vec4v(s.x), vec4v(s.p));
        if (dI >= 0.0) {
            s.intensity += dI;
            ++s.ncross;
            const float ratio = s.min_r / F.fr_ph_pro;
            if (ratio < 1.5f) {
                flags |= SIRIUS_FLAG_PHOTON_RING;
                magnification = ratio > 1.f ? fminf(1.f + 2.f / fmaxf(ratio - 1.f, 0.05f), 100.f) : 100.f;
            }
            if (s.ncross >= SIRIUS_MAX_CROSSINGS) return SIRIUS_DISK_HIT;
        }
    }
    if (s.steps >= c.max_steps) return s.ncross > 0 ? SIRIUS_DISK_HIT : SIRIUS_MAX_STEPS;
    return -1;
}

// The ray (pixel of the frame's row window) of this thread in a tiled launch.
// Each warp traces an 8 x 4 pixel tile (lane l: pixel (l % 8, l / 8) of it);
// a block's warps sit side by side in pairs (block of 32 threads: 8 x 4 pixels,
// 64: 16 x 4, 128: 16 x 8), and blocks cover the window row-major. A warp's rays
// then lie within 8 x 4 pixels instead of 32 x 1, so fewer warps straddle an
// edge of the image (the disk's rim, the photon ring) where neighbouring
// geodesics take different branches, and a block's warps, close together, end
// at about the same time (a block holds its SM slot until its last warp ends).
// Tiles at the frame's right and bottom edges are cut by it: their pixels beyond
// the edge return -1 (no ray).
__device__ __forceinline__ long long tile_ray(int width, int rows, int b) {
    const int nw = int(blockDim.x >> 5), across = nw >= 2 ? 2 : 1, bx = 8 * across, by = 4 * (nw / across);
    const int bpr = (width + bx - 1) / bx, w = int(threadIdx.x >> 5), l = int(threadIdx.x & 31);
    const int x = (b % bpr) * bx + (w % across) * 8 + (l & 7);
    const int y = (b / bpr) * by + (w / across) * 4 + (l >> 3);
    return x < width && y < rows ? (long long)y * width + x : -1;
}

// Persistent tracer. Dynamic shared memory: 2 * npair float2 per thread (volumetric bin pairs).
template <bool MIXED, int FAM, bool UNI, int INT>
__device__ __forceinline__ void trace_body(const Params& P) {
    extern __shared__ float smem[];
    float2* vol = (P.c.enable_vol && P.c.nbins > 0) ? reinterpret_cast<float2*>(smem) + threadIdx.x : nullptr;
    const int lane = threadIdx.x & 31;
    const unsigned lt_mask = (1u << lane) - 1u;
    Ray<MIXED> s;
    bool alive = false;
    float magnification = 1.f;
    int flags = 0;
    unsigned long long acc = 0, rej0 = 0, f64 = 0;
    bool exhausted = false;
    // the watchdog bounds the whole launch: every warp measures from the first warp's start
    unsigned long long t_start = 0;
    if (lane == 0) {
        const unsigned long long now = globaltimer();
        const unsigned long long first = atomicCAS(P.clock0, 0ull, now);
        t_start = first ? first : now;
    }
    t_start = __shfl_sync(kFull, t_start, 0);

    if (!P.persistent) {
        if (!UNI && P.blocks) {
            // this block's frame (the last entry whose first block is at or below it)
            int lo = 0, hi = P.n_block_frames - 1;
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (P.blocks[mid].x <= int(blockIdx.x)) lo = mid;
                else hi = mid - 1;
            }
            const int frame = P.blocks[lo].y, lb = int(blockIdx.x) - P.blocks[lo].x;
            const FrameDev& F = P.frames[frame];
            const long long pix = tile_ray(F.width, int(F.n_rays / F.width), lb);
            if (pix >= 0 && (P.family < 0 || F.m.family == P.family)) {
                begin_ray<MIXED, FAM, UNI>(P, s, F.ray_offset + pix, frame, vol);
                alive = true;
            }
        } else {
            const long long gid = UNI && P.tiled ? tile_ray(P.f0.width, int(P.f0.n_rays / P.f0.width), int(blockIdx.x) + P.block0)
                                                 : (long long)blockIdx.x * blockDim.x + threadIdx.x;
            const unsigned entry = (P.list && gid >= 0 && gid < P.total) ? P.list[gid] : 0u;
            if (gid >= 0 && gid < P.total && entry != kListSkip) {
                const long long idx = P.list ? (long long)entry : gid;
                const int frame = P.n_frames > 1 ? find_frame(P.frames, P.n_frames, idx) : 0;
                if (P.family < 0 || P.frames[frame].m.family == P.family) {
                    begin_ray<MIXED, FAM, UNI>(P, s, idx, frame, vol);
                    alive = true;
                }
            }
        }
        exhausted = true;
    }
    for (unsigned iter = 0;; ++iter) {
        if (P.persistent && !exhausted) {
            const unsigned dead = __ballot_sync(kFull, !alive);
            const int nlive = 32 - __popc(dead);
            if (dead && nlive < P.refill_threshold) {
                unsigned long long base = 0;
                if (lane == 0) base = atomicAdd(P.queue, (unsigned long long)__popc(dead));
                base = __shfl_sync(kFull, base, 0);
                if (base >= (unsigned long long)P.total) exhausted = true;
                if (!alive) {
                    const unsigned long long q = base + __popc(dead & lt_mask);
                    const unsigned entry = (P.list && q < (unsigned long long)P.total) ? P.list[q] : 0u;
                    if (q < (unsigned long long)P.total && entry != kListSkip) {
                        const unsigned long long idx = P.list ? (unsigned long long)entry : q;
                        const int frame = P.n_frames > 1 ? find_frame(P.frames, P.n_frames, (long long)idx) : 0;
                        begin_ray<MIXED, FAM, UNI>(P, s, (long long)idx, frame, vol);
                        alive = true;
                        magnification = 1.f;
                        flags = 0;
                    }
                }
            }
        }
        if ((iter & 255u) == 0) {
            int stop = 0;
            if (lane == 0) {
                if (globaltimer() - t_start > P.watchdog_ns) atomicOr(P.status, 1);
                stop = *((volatile int*)P.status) & 1;
            }
            stop = __shfl_sync(kFull, stop, 0);
            if (stop) {
                // watchdog: abandon the remaining queue and close the live rays
                exhausted = true;
                if (alive) { end_ray<MIXED, UNI>(P, s, SIRIUS_MAX_STEPS, magnification, flags, vol); alive = false; }
            }
        }
        if (__ballot_sync(kFull, alive) == 0) {
            if (!P.persistent || exhausted) break;
            continue;
        }
        if (alive) {
            const int out = advance<MIXED, FAM, UNI, INT>(P, s, magnification, flags, vol);
            if (out >= 0) {
                end_ray<MIXED, UNI>(P, s, out, magnification, flags, vol);
                acc += s.steps;
                rej0 += s.rejected;
                f64 += s.fp64_steps;
                alive = false;
            }
        }
    }
    // warp-aggregated counters
    for (int o = 16; o > 0; o >>= 1) {
        acc += __shfl_down_sync(kFull, acc, o);
        rej0 += __shfl_down_sync(kFull, rej0, o);
        f64 += __shfl_down_sync(kFull, f64, o);
    }
    if (lane == 0) {
        atomicAdd(&P.counters[0], acc);
        atomicAdd(&P.counters[1], rej0);
        atomicAdd(&P.counters[2], f64);
    }
}

// The tracer compiled for MINB resident 128-thread blocks per SM (MINB 2: up to
// 255 registers, 3: 168, 4: 128).
template <bool MIXED, int MINB, int FAM, bool UNI, int INT>
__global__ void __launch_bounds__(128, MINB) trace_kernel(const __grid_constant__ Params P) {
    trace_body<MIXED, FAM, UNI, INT>(P);
}

using TraceFn = void (*)(Params);

// The trace kernel for a register budget (minb resident 128-thread blocks per
// SM: 1 or 2 = up to 255 registers, 3 = 168, 4 = 128) and a launch form
// (uni: one frame, read from the parameter bank).
// Kerr-Schild family, mixed precision / FP64; symp: the symplectic integrator (else DP45)
TraceFn pick_ks_mixed(int minb, bool uni, bool symp);
TraceFn pick_ks_fp64(int minb, bool uni, bool symp);
TraceFn pick_family(bool mixed, int fam);   // Morris-Thorne, Alcubierre, or any family (kAnyFamily)
// Kerr-Schild family, mixed precision, two rays per thread (minb 2: 255 registers, 3: 168)
TraceFn pick_ks_mixed_pair(int minb, bool uni);

}  // namespace eng
}  // namespace sirius

// oracle.hpp — CPU restatement of Sirius's per-pixel geodesic hot path.
//
// TEST INFRASTRUCTURE ONLY. This file is the checker: the parity tests, the
// smoke check and the CPU-baseline leg of the benchmark call it through
// liboracle.so. The product (sirius_b200) never includes, links or calls it.
//
// It restates, in plain templated C++ (R = double or long double), the
// reference's algorithm for the path, following the reference's own structure
// (general metric -> 4x4 Cramer inverse -> 64-term contraction) rather than the
// closed forms the CUDA kernels use, so that the two formulations check each
// other. Two semantics are provided:
//   compat = true : the reference as written — float roundings of the RHS
//                   terms, step sizes and initial state, stop-on-reject,
//                   E-changing normalizeNull, Euclidean horizon/disk radii,
//                   the simplified g-factor and the gray volumetric march;
//   compat = false: the engine's semantics — the same mathematics in full
//                   FP64 with retry-on-reject, an E/L_z/Carter-preserving
//                   re-projection along dr, BL radii, the exact k.u g-factor,
//                   cubic Hermite disk crossings and multi-bin transfer.
// Reference citations are paths inside sunyaisblank/Sirius.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>

#include "../include/sirius_cuda.h"

namespace oracle {

constexpr double kPi = 3.14159265358979323846;

// ---------------------------------------------------------------------------
// Metric evaluation: g_{mu nu} and d_l g_{mu nu} (l = 0..3, d_0 = 0).
// ---------------------------------------------------------------------------

// KerrSchildFamily::evaluate, src/Sirius.Core/Metric/PHMT100A.h:248-396.
// r from r^4 - (R^2 - a^2) r^2 - a^2 z^2 = 0 (:263-273), its gradient (:278-293),
// l_mu = (1, (rx+ay)/(r^2+a^2), (ry-ax)/(r^2+a^2), z/r) and dl (:298-324),
// H = (2Mr - Q^2) r^2 / (r^4 + a^2 z^2) and dH (:329-343),
// g = eta + H l l with the "simplified" -Lambda R^2/3 on g_tt (:349-369), and
// dg (:374-395).
template <class R>
void ks_evaluate(const sirius_metric& m, const R pos[4], R g[4][4], R dg[4][4][4]) {
    const R x = pos[1], y = pos[2], z = pos[3];
    const R M = m.M, a = m.a, Q = m.Q, L = m.Lambda;
    const R a2 = a * a, Q2 = Q * Q;
    const R R2 = x * x + y * y + z * z;
    const R Rm2 = R2 - a2;
    R disc = Rm2 * Rm2 + R(4) * a2 * z * z;
    disc = std::max(disc, R(1e-20));
    const R sd = std::sqrt(disc);
    R r2 = (Rm2 + sd) / R(2);
    r2 = std::max(r2, R(1e-10));
    const R r = std::sqrt(r2);
    // gradient of r: d(r^2)/dx_i = x_i + d(sqrt disc)/dx_i / 2
    const R dsd[4] = {R(0), R(4) * x * Rm2 / (R(2) * sd), R(4) * y * Rm2 / (R(2) * sd),
                      R(4) * z * (R2 + a2) / (R(2) * sd)};
    const R dr2[4] = {R(0), x + dsd[1] / R(2), y + dsd[2] / R(2), z + dsd[3] / R(2)};
    R dr[4];
    for (int i = 0; i < 4; ++i) dr[i] = dr2[i] / (R(2) * r);
    const R den = r2 + a2, den2 = den * den;
    const R l[4] = {R(1), (r * x + a * y) / den, (r * y - a * x) / den, z / r};
    R dl[4][4] = {};  // dl[lambda][mu]
    const R n1 = r * x + a * y, n2 = r * y - a * x;
    dl[1][1] = (r + x * dr[1]) / den - n1 * dr2[1] / den2;
    dl[2][1] = (x * dr[2] + a) / den - n1 * dr2[2] / den2;
    dl[3][1] = (x * dr[3]) / den - n1 * dr2[3] / den2;
    dl[1][2] = (y * dr[1] - a) / den - n2 * dr2[1] / den2;
    dl[2][2] = (r + y * dr[2]) / den - n2 * dr2[2] / den2;
    dl[3][2] = (y * dr[3]) / den - n2 * dr2[3] / den2;
    dl[1][3] = -z * dr[1] / r2;
    dl[2][3] = -z * dr[2] / r2;
    dl[3][3] = R(1) / r - z * dr[3] / r2;
    const R fden = r2 * r2 + a2 * z * z;
    const R num = (R(2) * M * r - Q2) * r2;
    const R H = num / fden;
    R dH[4] = {};
    for (int k = 1; k <= 3; ++k) {
        const R dnum = R(2) * r * dr[k] * (R(3) * M * r - Q2);
        R dfden = R(4) * r2 * r * dr[k];
        if (k == 3) dfden += R(2) * a2 * z;
        dH[k] = (dnum * fden - num * dfden) / (fden * fden);
    }
    for (int mu = 0; mu < 4; ++mu)
        for (int nu = 0; nu < 4; ++nu) {
            const R eta = (mu == nu) ? (mu == 0 ? R(-1) : R(1)) : R(0);
            g[mu][nu] = eta + H * l[mu] * l[nu];
        }
    if (std::abs(L) > R(1e-15)) g[0][0] -= L * R2 / R(3);
    for (int mu = 0; mu < 4; ++mu)
        for (int nu = 0; nu < 4; ++nu) dg[0][mu][nu] = R(0);
    for (int k = 1; k <= 3; ++k)
        for (int mu = 0; mu < 4; ++mu)
            for (int nu = 0; nu < 4; ++nu)
                dg[k][mu][nu] = dH[k] * l[mu] * l[nu] + H * dl[k][mu] * l[nu] + H * l[mu] * dl[k][nu];
    if (std::abs(L) > R(1e-15)) {
        dg[1][0][0] -= R(2) * L * x / R(3);
        dg[2][0][0] -= R(2) * L * y / R(3);
        dg[3][0][0] -= R(2) * L * z / R(3);
    }
}

// Morris-Thorne shape function b(r) and b'(r), PHMT101A.h:195-243 (r clamped to >= b0).
template <class R>
void mt_shape(const sirius_metric& m, R r, R& b, R& db) {
    const R b0 = m.b0;
    r = std::max(r, b0);
    switch (m.shape) {
        case SIRIUS_WORMHOLE_ZERO_TIDAL: b = b0; db = R(0); break;
        case SIRIUS_WORMHOLE_ABSURDLY_BENIGN: b = b0 * (R(2) - b0 / r); db = b0 * b0 / (r * r); break;
        default: b = b0 * b0 / r; db = -b0 * b0 / (r * r); break;  // Ellis
    }
}

// MorrisThorneFamily::evaluate, PHMT101A.h:285-345, spherical (t, r, theta, phi),
// r clamped to >= 1.001 b0 (:293), 1 - b/r regularised at 1e-10 (:307), Phi constant.
// d_r g_rr is written here as the derivative of 1/(1 - b/r); the reference's
// line :334 carries the opposite sign, which its own finite-difference check
// would flag — the oracle follows the mathematics (see the parity notes).
template <class R>
void mt_evaluate(const sirius_metric& m, const R pos[4], R g[4][4], R dg[4][4][4]) {
    R r = std::max(pos[1], R(m.b0) * R(1.001));
    const R th = pos[2];
    const R s = std::sin(th), c = std::cos(th), s2 = s * s, r2 = r * r;
    R b, db;
    mt_shape(m, r, b, db);
    const R e2p = std::exp(R(2) * R(m.Phi0));
    const R f = std::max(R(1) - b / r, R(1e-10));
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) {
            g[i][j] = R(0);
            for (int k = 0; k < 4; ++k) dg[k][i][j] = R(0);
        }
    g[0][0] = -e2p;
    g[1][1] = R(1) / f;
    g[2][2] = r2;
    g[3][3] = r2 * s2;
    const R dfdr = -(db / r - b / r2);
    dg[1][1][1] = -dfdr / (f * f);
    dg[1][2][2] = R(2) * r;
    dg[1][3][3] = R(2) * r * s2;
    dg[2][3][3] = R(2) * r2 * s * c;
}

// WarpDriveFamily::evaluate, PHMT102A.h:136-229: bubble at the origin, static,
// f(rs) = (tanh(s(rs+R)) - tanh(s(rs-R))) / (2 tanh(sR)).
template <class R>
void alc_evaluate(const sirius_metric& m, const R pos[4], R g[4][4], R dg[4][4][4]) {
    const R x = pos[1], y = pos[2], z = pos[3];
    const R vs = m.vs, sg = m.sigma, Rb = m.R;
    R rs = std::sqrt(x * x + y * y + z * z);
    rs = std::max(rs, R(1e-10));
    const R tR = std::tanh(sg * Rb);
    const R f = (std::tanh(sg * (rs + Rb)) - std::tanh(sg * (rs - Rb))) / (R(2) * tR);
    const R chp = R(1) / std::cosh(sg * (rs + Rb)), chm = R(1) / std::cosh(sg * (rs - Rb));
    const R dfdr = sg * (chp * chp - chm * chm) / (R(2) * tR);
    const R df[4] = {R(0), dfdr * x / rs, dfdr * y / rs, dfdr * z / rs};
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) {
            g[i][j] = R(0);
            for (int k = 0; k < 4; ++k) dg[k][i][j] = R(0);
        }
    const R vsf = vs * f;
    g[0][0] = -(R(1) - vsf * vsf);
    g[0][1] = g[1][0] = -vsf;
    g[1][1] = g[2][2] = g[3][3] = R(1);
    for (int k = 1; k <= 3; ++k) {
        dg[k][0][0] = R(2) * vs * vs * f * df[k];
        dg[k][0][1] = dg[k][1][0] = -vs * df[k];
    }
}

template <class R>
void metric_evaluate(const sirius_metric& m, const R pos[4], R g[4][4], R dg[4][4][4]) {
    switch (m.family) {
        case SIRIUS_METRIC_MORRIS_THORNE: mt_evaluate(m, pos, g, dg); break;
        case SIRIUS_METRIC_ALCUBIERRE: alc_evaluate(m, pos, g, dg); break;
        default: ks_evaluate(m, pos, g, dg); break;
    }
}

// ---------------------------------------------------------------------------
// invertMetric4x4, PHGD001A.cpp:84-156: cofactor (Cramer) inverse with a
// Minkowski fallback for |det| < 1e-12 (PHCN001A.h:212) or kappa_inf > 1e12.
// ---------------------------------------------------------------------------
template <class R>
void invert4x4(const R m[4][4], R inv[4][4]) {
    // 2x2 minors of rows 2,3 (lower) and rows 1,3 / 1,2 (upper)
    auto minor = [&](int r0, int r1, int c0, int c1) { return m[r0][c0] * m[r1][c1] - m[r0][c1] * m[r1][c0]; };
    const R s23_23 = minor(2, 3, 2, 3), s23_13 = minor(2, 3, 1, 3), s23_12 = minor(2, 3, 1, 2);
    const R s23_03 = minor(2, 3, 0, 3), s23_02 = minor(2, 3, 0, 2), s23_01 = minor(2, 3, 0, 1);
    const R s13_23 = minor(1, 3, 2, 3), s13_13 = minor(1, 3, 1, 3), s13_12 = minor(1, 3, 1, 2);
    const R s13_03 = minor(1, 3, 0, 3), s13_02 = minor(1, 3, 0, 2), s13_01 = minor(1, 3, 0, 1);
    const R s12_23 = minor(1, 2, 2, 3), s12_13 = minor(1, 2, 1, 3), s12_12 = minor(1, 2, 1, 2);
    const R s12_03 = minor(1, 2, 0, 3), s12_02 = minor(1, 2, 0, 2), s12_01 = minor(1, 2, 0, 1);
    const R c00 = m[1][1] * s23_23 - m[1][2] * s23_13 + m[1][3] * s23_12;
    const R c01 = m[1][0] * s23_23 - m[1][2] * s23_03 + m[1][3] * s23_02;
    const R c02 = m[1][0] * s23_13 - m[1][1] * s23_03 + m[1][3] * s23_01;
    const R c03 = m[1][0] * s23_12 - m[1][1] * s23_02 + m[1][2] * s23_01;
    const R det = m[0][0] * c00 - m[0][1] * c01 + m[0][2] * c02 - m[0][3] * c03;
    auto minkowski = [&]() {
        for (int i = 0; i < 4; ++i)
            for (int j = 0; j < 4; ++j) inv[i][j] = (i == j) ? (i == 0 ? R(-1) : R(1)) : R(0);
    };
    if (std::abs(det) < R(1e-12)) { minkowski(); return; }
    const R id = R(1) / det;
    inv[0][0] = id * c00;
    inv[1][0] = -id * c01;
    inv[2][0] = id * c02;
    inv[3][0] = -id * c03;
    inv[0][1] = -id * (m[0][1] * s23_23 - m[0][2] * s23_13 + m[0][3] * s23_12);
    inv[1][1] = id * (m[0][0] * s23_23 - m[0][2] * s23_03 + m[0][3] * s23_02);
    inv[2][1] = -id * (m[0][0] * s23_13 - m[0][1] * s23_03 + m[0][3] * s23_01);
    inv[3][1] = id * (m[0][0] * s23_12 - m[0][1] * s23_02 + m[0][2] * s23_01);
    inv[0][2] = id * (m[0][1] * s13_23 - m[0][2] * s13_13 + m[0][3] * s13_12);
    inv[1][2] = -id * (m[0][0] * s13_23 - m[0][2] * s13_03 + m[0][3] * s13_02);
    inv[2][2] = id * (m[0][0] * s13_13 - m[0][1] * s13_03 + m[0][3] * s13_01);
    inv[3][2] = -id * (m[0][0] * s13_12 - m[0][1] * s13_02 + m[0][2] * s13_01);
    inv[0][3] = -id * (m[0][1] * s12_23 - m[0][2] * s12_13 + m[0][3] * s12_12);
    inv[1][3] = id * (m[0][0] * s12_23 - m[0][2] * s12_03 + m[0][3] * s12_02);
    inv[2][3] = -id * (m[0][0] * s12_13 - m[0][1] * s12_03 + m[0][3] * s12_01);
    inv[3][3] = id * (m[0][0] * s12_12 - m[0][1] * s12_02 + m[0][2] * s12_01);
    R ng = 0, ni = 0;
    for (int i = 0; i < 4; ++i) {
        R rg = 0, ri = 0;
        for (int j = 0; j < 4; ++j) { rg += std::abs(m[i][j]); ri += std::abs(inv[i][j]); }
        ng = std::max(ng, rg);
        ni = std::max(ni, ri);
    }
    if (ng * ni > R(1e12)) minkowski();
}

// ---------------------------------------------------------------------------
// Hamiltonian right-hand side (PHGD001A.cpp:159-202, 498-505):
//   dx^mu/dl = k^mu = g^{mu nu} p_nu,   dp_mu/dl = 1/2 d_mu g_{rs} k^r k^s.
// compat rounds each term through float as the reference does (:176, :199).
// ---------------------------------------------------------------------------
template <class R>
void rhs(const sirius_metric& m, const R x[4], const R p[4], R kx[4], R kp[4], bool compat) {
    R g[4][4], dg[4][4][4], gi[4][4];
    metric_evaluate(m, x, g, dg);
    invert4x4(g, gi);
    for (int mu = 0; mu < 4; ++mu) {
        R s = 0;
        for (int nu = 0; nu < 4; ++nu) {
            const R t = gi[mu][nu] * p[nu];
            s += compat ? R(float(t)) : t;
        }
        kx[mu] = s;
    }
    for (int mu = 0; mu < 4; ++mu) {
        R s = 0;
        for (int r = 0; r < 4; ++r)
            for (int q = 0; q < 4; ++q) s += dg[mu][r][q] * kx[r] * kx[q];
        kp[mu] = compat ? R(float(R(0.5) * s)) : R(0.5) * s;
    }
}

// p_mu = g_{mu nu} k^nu (computeMomentum, PHGD001A.cpp:486-495)
template <class R>
void lower(const R g[4][4], const R k[4], R p[4]) {
    for (int mu = 0; mu < 4; ++mu) {
        R s = 0;
        for (int nu = 0; nu < 4; ++nu) s += g[mu][nu] * k[nu];
        p[mu] = s;
    }
}

// TensorOps::innerProduct, MTTN001A.cpp:160-169
template <class R>
R inner(const R g[4][4], const R u[4], const R v[4]) {
    R s = 0;
    for (int mu = 0; mu < 4; ++mu)
        for (int nu = 0; nu < 4; ++nu) s += g[mu][nu] * u[mu] * v[nu];
    return s;
}

// TensorOps::normalizeNull, MTTN001A.cpp:171-237: solve g00 (k0)^2 + 2 g0i k0 ki +
// gij ki kj = 0 for a future-directed k0 (compat stores k0 through float).
template <class R>
void normalize_null(const R g[4][4], R k[4], bool compat) {
    const R A = g[0][0];
    R B = 0, C = 0;
    for (int i = 1; i < 4; ++i) B += R(2) * g[0][i] * k[i];
    for (int i = 1; i < 4; ++i)
        for (int j = 1; j < 4; ++j) C += g[i][j] * k[i] * k[j];
    R k0;
    if (std::abs(A) < R(1e-15)) {
        k0 = (std::abs(B) > R(1e-15)) ? -C / B : R(1);
    } else {
        const R d = B * B - R(4) * A * C;
        if (d < R(0)) {
            k0 = R(1);
        } else {
            const R sd = std::sqrt(d);
            const R kp = (-B + sd) / (R(2) * A), km = (-B - sd) / (R(2) * A);
            if (kp > R(0)) k0 = kp;
            else if (km > R(0)) k0 = km;
            else k0 = std::max(kp, km);
        }
    }
    k[0] = compat ? R(float(k0)) : k0;
}

// ---------------------------------------------------------------------------
// Dormand-Prince 5(4) tableau (PHGD001A.cpp:16-79; Dormand & Prince 1980).
// ---------------------------------------------------------------------------
struct DP {
    static constexpr double a21 = 1.0 / 5.0;
    static constexpr double a31 = 3.0 / 40.0, a32 = 9.0 / 40.0;
    static constexpr double a41 = 44.0 / 45.0, a42 = -56.0 / 15.0, a43 = 32.0 / 9.0;
    static constexpr double a51 = 19372.0 / 6561.0, a52 = -25360.0 / 2187.0, a53 = 64448.0 / 6561.0,
                            a54 = -212.0 / 729.0;
    static constexpr double a61 = 9017.0 / 3168.0, a62 = -355.0 / 33.0, a63 = 46732.0 / 5247.0,
                            a64 = 49.0 / 176.0, a65 = -5103.0 / 18656.0;
    static constexpr double b1 = 35.0 / 384.0, b3 = 500.0 / 1113.0, b4 = 125.0 / 192.0,
                            b5 = -2187.0 / 6784.0, b6 = 11.0 / 84.0;
    static constexpr double e1 = 35.0 / 384.0 - 5179.0 / 57600.0, e3 = 500.0 / 1113.0 - 7571.0 / 16695.0,
                            e4 = 125.0 / 192.0 - 393.0 / 640.0, e5 = -2187.0 / 6784.0 + 92097.0 / 339200.0,
                            e6 = 11.0 / 84.0 - 187.0 / 2100.0, e7 = -1.0 / 40.0;
};

// Geodesic::computeOptimalStep, PHGD001A.cpp:471-483 (float arithmetic in compat).
template <class R>
R optimal_step(R h, R err, const sirius_trace_config& c, bool compat) {
    if (compat) {
        const float fh = float(h), fe = float(err);
        if (fe < 1e-15f) return R(std::min(fh * float(c.step_grow_max), float(c.max_step)));
        float fac = float(c.safety_factor) * std::pow(1.0f / fe, 0.2f);
        fac = std::max(float(c.step_shrink_min), std::min(float(c.step_grow_max), fac));
        return R(std::max(float(c.min_step), std::min(float(c.max_step), fh * fac)));
    }
    if (err < R(1e-15)) return std::min(h * R(c.step_grow_max), R(c.max_step));
    R fac = R(c.safety_factor) * std::pow(R(1) / err, R(0.2));
    fac = std::max(R(c.step_shrink_min), std::min(R(c.step_grow_max), fac));
    return std::max(R(c.min_step), std::min(R(c.max_step), h * fac));
}

// One DP45 attempt on y = (x^mu, p_mu). On entry k1 holds f(y) (first-same-as-last).
// Returns the scaled RMS error of the position components (computeRK45ErrorNorm,
// PHGD001A.cpp:508-517) and writes the candidate state and its derivative k7.
// In compat the stage coefficients a_ij h are rounded through float (:549-571).
template <class R>
R dp45_attempt(const sirius_metric& m, const sirius_trace_config& c, const R x[4], const R p[4], R h,
               const R k1x[4], const R k1p[4], R xn[4], R pn[4], R k7x[4], R k7p[4], bool compat) {
    auto cf = [&](double coef) { return compat ? R(float(coef * double(h))) : R(coef) * h; };
    R k2x[4], k2p[4], k3x[4], k3p[4], k4x[4], k4p[4], k5x[4], k5p[4], k6x[4], k6p[4], xs[4], ps[4];
    {
        const R c1 = cf(DP::a21);
        for (int i = 0; i < 4; ++i) { xs[i] = x[i] + k1x[i] * c1; ps[i] = p[i] + k1p[i] * c1; }
        rhs(m, xs, ps, k2x, k2p, compat);
    }
    {
        const R c1 = cf(DP::a31), c2 = cf(DP::a32);
        for (int i = 0; i < 4; ++i) {
            xs[i] = x[i] + k1x[i] * c1 + k2x[i] * c2;
            ps[i] = p[i] + k1p[i] * c1 + k2p[i] * c2;
        }
        rhs(m, xs, ps, k3x, k3p, compat);
    }
    {
        const R c1 = cf(DP::a41), c2 = cf(DP::a42), c3 = cf(DP::a43);
        for (int i = 0; i < 4; ++i) {
            xs[i] = x[i] + k1x[i] * c1 + k2x[i] * c2 + k3x[i] * c3;
            ps[i] = p[i] + k1p[i] * c1 + k2p[i] * c2 + k3p[i] * c3;
        }
        rhs(m, xs, ps, k4x, k4p, compat);
    }
    {
        const R c1 = cf(DP::a51), c2 = cf(DP::a52), c3 = cf(DP::a53), c4 = cf(DP::a54);
        for (int i = 0; i < 4; ++i) {
            xs[i] = x[i] + k1x[i] * c1 + k2x[i] * c2 + k3x[i] * c3 + k4x[i] * c4;
            ps[i] = p[i] + k1p[i] * c1 + k2p[i] * c2 + k3p[i] * c3 + k4p[i] * c4;
        }
        rhs(m, xs, ps, k5x, k5p, compat);
    }
    {
        const R c1 = cf(DP::a61), c2 = cf(DP::a62), c3 = cf(DP::a63), c4 = cf(DP::a64), c5 = cf(DP::a65);
        for (int i = 0; i < 4; ++i) {
            xs[i] = x[i] + k1x[i] * c1 + k2x[i] * c2 + k3x[i] * c3 + k4x[i] * c4 + k5x[i] * c5;
            ps[i] = p[i] + k1p[i] * c1 + k2p[i] * c2 + k3p[i] * c3 + k4p[i] * c4 + k5p[i] * c5;
        }
        rhs(m, xs, ps, k6x, k6p, compat);
    }
    auto cb = [&](double coef) { return compat ? R(float(coef)) : R(coef); };
    for (int i = 0; i < 4; ++i) {
        xn[i] = x[i] + (k1x[i] * cb(DP::b1) + k3x[i] * cb(DP::b3) + k4x[i] * cb(DP::b4) + k5x[i] * cb(DP::b5) +
                        k6x[i] * cb(DP::b6)) * h;
        pn[i] = p[i] + (k1p[i] * cb(DP::b1) + k3p[i] * cb(DP::b3) + k4p[i] * cb(DP::b4) + k5p[i] * cb(DP::b5) +
                        k6p[i] * cb(DP::b6)) * h;
    }
    rhs(m, xn, pn, k7x, k7p, compat);
    if (compat) {
        float en = 0.0f;
        for (int i = 0; i < 4; ++i) {
            const R e = (k1x[i] * cb(DP::e1) + k3x[i] * cb(DP::e3) + k4x[i] * cb(DP::e4) + k5x[i] * cb(DP::e5) +
                         k6x[i] * cb(DP::e6) + k7x[i] * cb(DP::e7)) * h;
            const float sc = float(double(float(c.abs_tolerance)) +
                                   double(float(c.rel_tolerance)) * std::abs(double(xn[i])));
            const float ei = float(std::abs(double(e)) / double(sc));
            en += ei * ei;
        }
        return R(std::sqrt(en / 4.0f));
    }
    R en = 0;
    for (int i = 0; i < 4; ++i) {
        const R e = h * (k1x[i] * R(DP::e1) + k3x[i] * R(DP::e3) + k4x[i] * R(DP::e4) + k5x[i] * R(DP::e5) +
                         k6x[i] * R(DP::e6) + k7x[i] * R(DP::e7));
        const R sc = R(c.abs_tolerance) + R(c.rel_tolerance) * std::abs(xn[i]);
        en += (e / sc) * (e / sc);
    }
    return std::sqrt(en / R(4));
}

// Geodesic::integrateStepRK45 as written (PHGD001A.cpp:530-641) on a Lightray
// (position x, contravariant velocity k, float step h): p from the stored
// velocity, stage 1 from it, the DP45 attempt with float roundings, reject ->
// false (terminated = 5 when h reaches min_step), NaN/Inf -> terminated = 3,
// and the null re-normalisation of k^0 when |g k k| > 1e-6 (:609-638).
template <class R>
bool compat_rk45_step(const sirius_metric& m, const sirius_trace_config& c, R x[4], R k[4], R& h, int& terminated) {
    R g0[4][4], dg0[4][4][4], p[4], k1x[4], k1p[4], xn[4], pn[4], k7x[4], k7p[4];
    metric_evaluate(m, x, g0, dg0);
    lower(g0, k, p);
    for (int mu = 0; mu < 4; ++mu) {
        R s = 0;
        for (int r = 0; r < 4; ++r)
            for (int q = 0; q < 4; ++q) s += dg0[mu][r][q] * k[r] * k[q];
        k1p[mu] = R(float(R(0.5) * s));
        k1x[mu] = k[mu];
    }
    const R err = dp45_attempt(m, c, x, p, h, k1x, k1p, xn, pn, k7x, k7p, true);
    if (float(err) > 1.0f) {
        h = optimal_step(h, err, c, true);
        if (h <= R(float(c.min_step))) terminated = 5;
        return false;
    }
    for (int i = 0; i < 4; ++i) { x[i] = xn[i]; k[i] = k7x[i]; }
    h = optimal_step(h, err, c, true);
    for (int i = 0; i < 4; ++i)
        if (!std::isfinite(double(x[i])) || !std::isfinite(double(k[i]))) { terminated = 3; return false; }
    R g1[4][4], dg1[4][4][4];
    metric_evaluate(m, x, g1, dg1);
    if (std::abs(double(inner(g1, k, k))) > 1e-6) {
        R kk[4] = {k[0], k[1], k[2], k[3]};
        normalize_null(g1, kk, true);
        bool ok = true;
        for (int i = 0; i < 4; ++i) ok &= std::isfinite(double(kk[i]));
        if (ok) for (int i = 0; i < 4; ++i) k[i] = kk[i];
    }
    return true;
}

// ---------------------------------------------------------------------------
// Symplectic integration (SymplecticIntegratorD, PHSI001A.h:43-80, 136-215,
// 430-455) on the Kerr-Schild Hamiltonian H = 1/2 g^{mu nu}(x) p_mu p_nu:
// a Yoshida composition (orders 4, 6, 8; Yoshida 1990) of the kick-drift-kick
// leapfrog  p += h/2 dp/dl(x, p);  x += h dx/dl(x, p);  p += h/2 dp/dl(x, p),
// with dx/dl = g^{-1} p and dp/dl = 1/2 d g k k (the reference's dHdp / dHdq).
// ---------------------------------------------------------------------------
inline void yoshida_weights(int order, int& n, const double*& w) {
    static const double w4[3] = {1.3512071919596576, -1.7024143839193153, 1.3512071919596576};
    static const double w6[7] = {0.78451361047756, 0.23557321335936, -1.17767998417887, 1.31518632068391,
                                 -1.17767998417887, 0.23557321335936, 0.78451361047756};
    static const double w8[15] = {0.74167036435061, -0.40910082580003, 0.19075471029623, -0.57386247111608,
                                  0.29906418130365, 0.33462491824529, 0.31529309239676, -0.79688793935291,
                                  0.31529309239676, 0.33462491824529, 0.29906418130365, -0.57386247111608,
                                  0.19075471029623, -0.40910082580003, 0.74167036435061};
    if (order >= 8) { n = 15; w = w8; }
    else if (order >= 6) { n = 7; w = w6; }
    else { n = 3; w = w4; }
}

template <class R>
void leapfrog(const sirius_metric& m, R x[4], R p[4], R h) {
    R k[4], f[4];
    rhs(m, x, p, k, f, false);
    for (int i = 0; i < 4; ++i) p[i] += R(0.5) * h * f[i];
    rhs(m, x, p, k, f, false);
    for (int i = 0; i < 4; ++i) x[i] += h * k[i];
    rhs(m, x, p, k, f, false);
    for (int i = 0; i < 4; ++i) p[i] += R(0.5) * h * f[i];
}

template <class R>
void symplectic_step(const sirius_metric& m, int order, R h, R x[4], R p[4]) {
    int n;
    const double* w;
    yoshida_weights(order, n, w);
    for (int s = 0; s < n; ++s) leapfrog(m, x, p, R(w[s]) * h);
}

// ---------------------------------------------------------------------------
// Radial coordinate of the family and its gradient (the covector dr used by the
// E/L_z-preserving re-projection — the Kerr-Schild form of the p_r
// renormalisation of SymplecticIntegratorD::renormalizeNull, PHSI001A.h:366-418).
// ---------------------------------------------------------------------------
template <class R>
R radial(const sirius_metric& m, const R x[4], R grad[4]) {
    grad[0] = R(0);
    if (m.family == SIRIUS_METRIC_MORRIS_THORNE) {
        grad[1] = R(1); grad[2] = R(0); grad[3] = R(0);
        return x[1];
    }
    const R X = x[1], Y = x[2], Z = x[3];
    const R R2 = X * X + Y * Y + Z * Z;
    if (m.family == SIRIUS_METRIC_ALCUBIERRE || std::abs(m.a) == 0) {
        const R Rr = std::sqrt(R2);
        grad[1] = X / Rr; grad[2] = Y / Rr; grad[3] = Z / Rr;
        return Rr;
    }
    const R a2 = R(m.a) * R(m.a), Rm2 = R2 - a2;
    const R sd = std::sqrt(Rm2 * Rm2 + R(4) * a2 * Z * Z);
    const R r = std::sqrt(std::max((Rm2 + sd) / R(2), R(1e-20)));
    grad[1] = r * X / sd;
    grad[2] = r * Y / sd;
    grad[3] = Z * (r * r + a2) / (r * sd);
    return r;
}

// Solve g^{mu nu}(p + alpha dr)_mu (p + alpha dr)_nu = 0 for the root alpha of
// smallest magnitude (the root "closest to the current p_r", PHSI001A.h:408-414).
// Returns the null value before the projection.
template <class R>
R project_null(const sirius_metric& m, const R x[4], R p[4]) {
    R g[4][4], dg[4][4][4], gi[4][4], d[4];
    metric_evaluate(m, x, g, dg);
    invert4x4(g, gi);
    radial(m, x, d);
    R A = 0, B = 0, C = 0;
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) {
            A += gi[i][j] * d[i] * d[j];
            B += R(2) * gi[i][j] * p[i] * d[j];
            C += gi[i][j] * p[i] * p[j];
        }
    const R disc = B * B - R(4) * A * C;
    if (disc < R(0) || std::abs(A) < R(1e-15)) return C;
    const R q = -R(0.5) * (B + (B >= R(0) ? std::sqrt(disc) : -std::sqrt(disc)));
    if (q == R(0)) return C;
    const R alpha = C / q;  // the small root of A a^2 + B a + C
    for (int i = 0; i < 4; ++i) p[i] += alpha * d[i];
    return C;
}

template <class R>
R null_value(const sirius_metric& m, const R x[4], const R p[4]) {
    R g[4][4], dg[4][4][4], gi[4][4];
    metric_evaluate(m, x, g, dg);
    invert4x4(g, gi);
    R C = 0;
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) C += gi[i][j] * p[i] * p[j];
    return C;
}

// ---------------------------------------------------------------------------
// Horizons, photon orbits, ISCO, Keplerian orbits
// ---------------------------------------------------------------------------
// KerrSchildFamily::outerHorizonRadius, PHMT100A.h:402-415 (-1: no horizon)
inline double r_plus(const sirius_metric& m) {
    const double d = m.M * m.M - m.a * m.a - m.Q * m.Q;
    return d < 0 ? -1.0 : m.M + std::sqrt(d);
}

// Equatorial circular photon orbit of Kerr (Bardeen, Press & Teukolsky 1972):
// r = 2M (1 + cos(2/3 acos(-+a/M))) — prograde (-) and retrograde (+); the
// reference uses the prograde one with the spin clamped to 0.998 (GTRC001A.cpp:173-184).
inline double r_photon(double M, double a, bool prograde) {
    double s = std::clamp(a / M, -1.0, 1.0);
    const double arg = prograde ? -s : s;
    return 2.0 * M * (1.0 + std::cos((2.0 / 3.0) * std::acos(std::clamp(arg, -1.0, 1.0))));
}

// AccretionDiskD::computeISCO, PHAD001A.h:88-105 (Bardeen, Press & Teukolsky 1972), in units of M.
inline double isco(double a_star) {
    double a = std::min(std::abs(a_star), 1.0);
    const double Z1 = 1 + std::cbrt(1 - a * a) * (std::cbrt(1 + a) + std::cbrt(1 - a));
    const double Z2 = std::sqrt(3 * a * a + Z1 * Z1);
    return a_star >= 0 ? 3 + Z2 - std::sqrt((3 - Z1) * (3 + Z1 + 2 * Z2))
                       : 3 + Z2 + std::sqrt((3 - Z1) * (3 + Z1 + 2 * Z2));
}

// Page & Thorne circular-orbit quantities, PHAD001A.h:112-223 (M = 1 units).
inline double pt_E(double r, double M, double a) {
    const double s = std::sqrt(M * r), d = r * std::sqrt(r * r - 3 * M * r + 2 * a * s);
    return std::abs(d) < 1e-15 ? 1.0 : (r * r - 2 * M * r + a * s) / d;
}
inline double pt_L(double r, double M, double a) {
    const double s = std::sqrt(M * r), d = r * std::sqrt(r * r - 3 * M * r + 2 * a * s);
    return std::abs(d) < 1e-15 ? 0.0 : std::sqrt(M) * (r * r - 2 * a * s + a * a) / d;
}
inline double pt_Omega(double r, double M, double a) { return std::sqrt(M) / (std::pow(r, 1.5) + a * std::sqrt(M)); }
inline double pt_dLdr(double r, double M, double a) {
    if (r <= 0 || M <= 0) return 0;
    const double sM = std::sqrt(M), sMr = std::sqrt(M * r), sr = std::sqrt(r);
    const double N = r * r - 2 * a * sMr + a * a, D = r * r - 3 * M * r + 2 * a * sMr;
    if (D <= 1e-15) return 0;
    const double sD = std::sqrt(D), q = a * sM / sr;
    const double dN = 2 * r - q, dD = 2 * r - 3 * M + q;
    const double drsD = (2 * D + r * dD) / (2 * sD), rsD = r * sD, den = rsD * rsD;
    if (std::abs(den) < 1e-30) return 0;
    return sM * (dN * rsD - N * drsD) / den;
}
inline double pt_dOmegadr(double r, double M, double a) {
    if (r <= 0 || M <= 0) return 0;
    const double den = std::pow(r, 1.5) + a * std::sqrt(M);
    if (std::abs(den) < 1e-30) return 0;
    return -3.0 * std::sqrt(M * r) / (2.0 * den * den);
}

// AccretionDiskD::flux (PHAD001A.h:321-361) with fullPageThorneFlux (:234-314),
// in geometric units (G = c = M = Mdot = 1): F = 3/(8 pi r^3) Q(r).
// Gauss-Legendre 16-point nodes/weights: Abramowitz & Stegun table 25.4.
inline double nt_flux(double r, double a_star, double r_in, double r_out) {
    static const double gx[8] = {0.0950125098376374, 0.2816035507792589, 0.4580167776572274,
                                 0.6178762444026438, 0.7554044083550030, 0.8656312023878318,
                                 0.9445750230732326, 0.9894009349916499};
    static const double gw[8] = {0.1894506104550685, 0.1826034150449236, 0.1691565193950025,
                                 0.1495959888165767, 0.1246289712555339, 0.0951585116824928,
                                 0.0622535239386479, 0.0271524594117541};
    const double ri = isco(a_star);
    if (r < r_in || r > r_out || r <= ri) return 0.0;
    const double a = a_star, M = 1.0;
    const double Fn = 3.0 / (8.0 * kPi * r * r * r);
    if (r > 1.5 * ri) {
        const double hw = 0.5 * (r - ri), mid = 0.5 * (r + ri);
        double I = 0;
        for (int s = -1; s <= 1; s += 2)
            for (int i = 0; i < 8; ++i) {
                const double rr = mid + hw * s * gx[i];
                I += gw[i] * (pt_E(rr, M, a) - pt_Omega(rr, M, a) * pt_L(rr, M, a)) * pt_dLdr(rr, M, a);
            }
        I *= hw;
        const double EmOL = pt_E(r, M, a) - pt_Omega(r, M, a) * pt_L(r, M, a);
        if (std::abs(EmOL) >= 1e-15) {
            const double F = Fn * (-pt_dOmegadr(r, M, a) / (EmOL * EmOL)) * I;
            if (std::isfinite(F) && F > 0) return F;
        }
    }
    const double it = 1 - std::sqrt(ri / r);
    if (it <= 0) return 0.0;
    const double y = std::sqrt(r), den = y * y * y * (y - 3.0 / y + 2 * a / (y * y));
    double Q = std::abs(den) > 1e-10 ? 1.0 / den : 1.0;
    if (!std::isfinite(Q) || Q <= 0) Q = 1.0;
    Q = std::clamp(Q, 0.1, 10.0);
    return Fn * it * Q;
}

// ---------------------------------------------------------------------------
// Camera: PinholeCamera::generateRay (CMBS001A.h:120-185) in float as written,
// and the 360x180 equirectangular sky camera the engine defines (the reference's
// Panoramic lens has no implementation, CMBS001A.h:68,351-362).
// ---------------------------------------------------------------------------
inline void camera_ray(const sirius_camera& cam, int px, int py, double origin[4], double dir[4], float u = 0.5f,
                       float v = 0.5f) {
    origin[0] = cam.t; origin[1] = cam.r; origin[2] = cam.theta; origin[3] = cam.phi;
    dir[0] = 0.0;
    if (cam.projection == SIRIUS_CAMERA_EQUIRECTANGULAR) {
        // longitude psi in [-pi, pi) across the width, latitude chi in (-pi/2, pi/2) down the height;
        // camera-local direction (right, up, forward) = (cos chi sin psi, sin chi, cos chi cos psi).
        const double psi = (2.0 * (px + double(u)) / cam.width - 1.0) * kPi;
        const double chi = (1.0 - 2.0 * (py + double(v)) / cam.height) * (0.5 * kPi);
        const double right = std::cos(chi) * std::sin(psi), up = std::sin(chi), fwd = std::cos(chi) * std::cos(psi);
        dir[1] = -fwd;  // forward is radially inward
        dir[2] = -up;   // up is -theta
        dir[3] = right; // right is +phi
        return;
    }
    const float aspect = float(cam.width) / float(cam.height);
    const float tanh = std::tan(cam.fov * float(kPi) / 360.0f);
    const float pxn = (2.0f * (px + u) / cam.width - 1.0f) * aspect;
    const float pyn = 1.0f - 2.0f * (py + v) / cam.height;
    const float dx = pxn * tanh, dy = pyn * tanh, dz = -1.0f;
    const float cY = std::cos(cam.yaw), sY = std::sin(cam.yaw);
    const float cP = std::cos(cam.pitch), sP = std::sin(cam.pitch);
    const float cR = std::cos(cam.roll), sR = std::sin(cam.roll);
    const float rx = dx * cR - dy * sR, ry = dx * sR + dy * cR;
    const float ry2 = ry * cP - dz * sP, rz = ry * sP + dz * cP;
    const float rx2 = rx * cY + rz * sY, rz2 = -rx * sY + rz * cY;
    const float len = std::sqrt(rx2 * rx2 + ry2 * ry2 + rz2 * rz2);
    dir[1] = rz2 / len;
    dir[2] = -ry2 / len;
    dir[3] = rx2 / len;
}

// The same pinhole and equirectangular mappings at a fractional pixel position
// (u, v) evaluated in FP64 after the camera's FP32 constants (aspect, tan of
// half the field of view, the rotation cosines and sines): smooth in (u, v),
// for derivatives of the image mapping (the beam checks).
inline void camera_ray_exact(const sirius_camera& cam, double u, double v, double origin[4], double dir[4]) {
    origin[0] = cam.t; origin[1] = cam.r; origin[2] = cam.theta; origin[3] = cam.phi;
    dir[0] = 0.0;
    if (cam.projection == SIRIUS_CAMERA_EQUIRECTANGULAR) {
        const double psi = (2.0 * u / cam.width - 1.0) * kPi;
        const double chi = (1.0 - 2.0 * v / cam.height) * (0.5 * kPi);
        dir[1] = -std::cos(chi) * std::cos(psi);
        dir[2] = -std::sin(chi);
        dir[3] = std::cos(chi) * std::sin(psi);
        return;
    }
    const float aspect = float(cam.width) / float(cam.height);
    const float tanh = std::tan(cam.fov * float(kPi) / 360.0f);
    const double pxn = (2.0 * u / cam.width - 1.0) * double(aspect), pyn = 1.0 - 2.0 * v / cam.height;
    const double dx = pxn * double(tanh), dy = pyn * double(tanh), dz = -1.0;
    const double cY = std::cos(cam.yaw), sY = std::sin(cam.yaw);
    const double cP = std::cos(cam.pitch), sP = std::sin(cam.pitch);
    const double cR = std::cos(cam.roll), sR = std::sin(cam.roll);
    const double rx = dx * cR - dy * sR, ry = dx * sR + dy * cR;
    const double ry2 = ry * cP - dz * sP, rz = ry * sP + dz * cP;
    const double rx2 = rx * cY + rz * sY, rz2 = -rx * sY + rz * cY;
    const double len = std::sqrt(rx2 * rx2 + ry2 * ry2 + rz2 * rz2);
    dir[1] = rz2 / len;
    dir[2] = -ry2 / len;
    dir[3] = rx2 / len;
}

// ---------------------------------------------------------------------------
// Ray tracing (GeodesicTracer::trace, GTRC001A.cpp:139-592)
// ---------------------------------------------------------------------------
struct TraceContext {
    sirius_metric metric;
    sirius_trace_config cfg;
    double disk_inner, disk_outer;
    double cam_pos[4];  // camera position in the integration chart (for the observer redshift)
};

struct Spectra {
    double I[SIRIUS_MAX_BINS];
    double tau[SIRIUS_MAX_BINS];
};

// Keplerian emitter in the equatorial plane at BL radius r: u = u^t (d_t + Omega d_phi).
// u^t from the Killing-vector norms of the metric at the point (coordinate invariant).
template <class R>
bool kepler_ut(const sirius_metric& m, const R pos[4], R r_bl, R& ut, R& Omega) {
    R g[4][4], dg[4][4][4];
    metric_evaluate(m, pos, g, dg);
    const R xi[4] = {R(0), -pos[2], pos[1], R(0)};
    R gtt = g[0][0], gtp = 0, gpp = 0;
    for (int i = 0; i < 4; ++i) {
        gtp += g[0][i] * xi[i];
        for (int j = 0; j < 4; ++j) gpp += g[i][j] * xi[i] * xi[j];
    }
    Omega = R(pt_Omega(double(r_bl), m.M, m.a));
    const R n = -(gtt + R(2) * Omega * gtp + Omega * Omega * gpp);
    if (!(n > R(0))) return false;
    ut = R(1) / std::sqrt(n);
    return true;
}

// Redshift factor g = (p.u_obs) / (p.u_em) on the traced geodesic: a static
// observer at the camera, u_obs = d_t / sqrt(-g_tt), and a Keplerian emitter,
// u_em = u^t (d_t + Omega d_phi):  g = 1 / (sqrt(-g_tt,cam) u^t (1 - Omega L_z / E)).
// The traced ray leaves the camera future-directed (the reference's convention,
// GTRC001A.cpp:82-106); the isometry (t, phi) -> (-t, -phi) maps it onto the
// physical photon that reaches the azimuth-mirrored camera, and leaves p.u
// unchanged, so this g is the physical redshift of that (left-right mirrored) image.
// E = -p_t and L_z = x p_y - y p_x are the ray's conserved quantities (taken
// from one consistent state), pos the emitter position.
template <class R>
R redshift_exact(const TraceContext& ctx, const R pos[4], R r_bl, R E, R Lz, R sqrt_m_gtt_cam) {
    R ut, Om;
    if (!kepler_ut(ctx.metric, pos, r_bl, ut, Om)) return R(0);
    const R den = sqrt_m_gtt_cam * ut * (R(1) - Om * Lz / E);
    return den > R(0) ? R(1) / den : R(0);
}

// computeGFactor / computeGFactorWithComponents, GTRC001A.cpp:645-828 (the
// reference's simplified g: grav / (gamma (1 - v.n)), clamped).
inline double redshift_compat(const sirius_metric& m, float r, float phi, const double vel[4]) {
    const double M = m.M, a = m.a;
    const float Om = float(std::sqrt(M) / (std::pow(double(r), 1.5) + a * std::sqrt(M)));
    const double vorb = double(r) * Om, rd = r;
    const double grav = std::sqrt(1.0 - 2.0 * M * rd / (rd * rd + a * a));
    double nx = vel[1], ny = vel[2], nz = vel[3];
    const double vm = std::sqrt(nx * nx + ny * ny + nz * nz);
    if (vm < 1e-10) return float(grav);
    nx /= vm; ny /= vm;
    const double gam = 1.0 / std::sqrt(std::max(1e-10, 1.0 - vorb * vorb));
    const double A = (-nx) * std::sin(double(phi)) - (-ny) * std::cos(double(phi));
    double dd = std::clamp(gam * (1.0 - vorb * A), 0.1, 10.0);
    return float(std::clamp(grav / dd, 0.1, 5.0));
}

// Carter constant of a Kerr-Schild state: theta from r(x,y,z), p_theta =
// cot(theta)(x p_x + y p_y) - r sin(theta) p_z, Q = p_th^2 + cos^2 (-a^2 E^2 + Lz^2 / sin^2)
// (GeodesicStateD::computeConservedQuantities, MTTP001A.h:123-132).
template <class R>
void invariants(const sirius_metric& m, const R x[4], const R p[4], R& E, R& Lz, R& Q) {
    E = -p[0];
    if (m.family == SIRIUS_METRIC_MORRIS_THORNE) {
        Lz = p[3];
        const R s = std::sin(x[2]), c = std::cos(x[2]);
        Q = p[2] * p[2] + c * c * Lz * Lz / (s * s);
        return;
    }
    Lz = x[1] * p[2] - x[2] * p[1];
    R d[4];
    const R r = radial(m, x, d);
    const R ct = std::clamp(x[3] / r, R(-1), R(1));
    const R st = std::sqrt(std::max(R(1) - ct * ct, R(1e-30)));
    const R pth = (ct / st) * (x[1] * p[1] + x[2] * p[2]) - r * st * p[3];
    const R a = m.a;
    Q = pth * pth + ct * ct * (-a * a * E * E + Lz * Lz / (st * st));
}

// Initial state from a camera ray: GeodesicTracer::initializeLightray
// (GTRC001A.cpp:15-134): theta clamp, spherical map, spherical->Cartesian
// velocity, normalizeNull for k^0, p = g k. compat rounds through float.
template <class R>
void init_state(const TraceContext& ctx, const double origin[4], const double dir[4], R x[4], R p[4], R k[4]) {
    const bool compat = ctx.cfg.compat != 0;
    const double t = origin[0], r = origin[1];
    const double th = std::clamp(origin[2], 0.01, kPi - 0.01), ph = origin[3];
    const double st = std::sin(th), ct = std::cos(th), sp = std::sin(ph), cp = std::cos(ph);
    const double vr = dir[1], vth = dir[2] / r;
    double vph = dir[3] / (r * st);
    if (std::abs(st) < 1e-10) vph = 0.0;
    R g[4][4], dg[4][4][4];
    if (ctx.metric.family == SIRIUS_METRIC_MORRIS_THORNE) {
        x[0] = t; x[1] = r; x[2] = th; x[3] = ph;
        metric_evaluate(ctx.metric, x, g, dg);
        // orthonormal spatial frame of the static observer: e_r = d_r/sqrt(g_rr), e_th = d_th/r, e_ph = d_ph/(r sin)
        k[0] = 0; k[1] = R(vr) / std::sqrt(g[1][1]); k[2] = R(vth); k[3] = R(vph);
        normalize_null(g, k, false);
        lower(g, k, p);
        return;
    }
    const double cart[4] = {t, r * st * cp, r * st * sp, r * ct};
    const double vel[4] = {0.0, vr * st * cp + r * vth * ct * cp - r * vph * st * sp,
                           vr * st * sp + r * vth * ct * sp + r * vph * st * cp, vr * ct - r * vth * st};
    for (int i = 0; i < 4; ++i) {
        x[i] = compat ? R(float(cart[i])) : R(cart[i]);
        k[i] = compat ? R(float(vel[i])) : R(vel[i]);
    }
    metric_evaluate(ctx.metric, x, g, dg);
    k[0] = 0;
    normalize_null(g, k, compat);
    if (compat)
        for (int i = 0; i < 4; ++i) k[i] = R(float(k[i]));
    lower(g, k, p);
}

// Gauss-Legendre points and weights on [0, 1] (n = 1..4; Abramowitz & Stegun 25.4),
// ordered along the step. The volumetric quadrature of one step.
inline void gauss_legendre(int n, int& m, const double*& x, const double*& w) {
    static const double x1[1] = {0.5}, w1[1] = {1.0};
    static const double x2[2] = {0.21132486540518713, 0.78867513459481287}, w2[2] = {0.5, 0.5};
    static const double x3[3] = {0.11270166537925831, 0.5, 0.88729833462074169},
                        w3[3] = {0.27777777777777778, 0.44444444444444444, 0.27777777777777778};
    static const double x4[4] = {0.069431844202973713, 0.33000947820757187, 0.66999052179242813,
                                 0.93056815579702629},
                        w4[4] = {0.17392742256872693, 0.32607257743127307, 0.32607257743127307,
                                 0.17392742256872693};
    switch (n <= 1 ? 1 : (n >= 4 ? 4 : n)) {
        case 1: m = 1; x = x1; w = w1; break;
        case 2: m = 2; x = x2; w = w2; break;
        case 3: m = 3; x = x3; w = w3; break;
        default: m = 4; x = x4; w = w4; break;
    }
}

// Cubic Hermite interpolation of the step (x0, k0) -> (x1, k1) over h: returns
// the fraction s in [0,1] where z(s) = 0 (bisection + Newton on the cubic).
template <class R>
R hermite_z_root(R z0, R z1, R dz0, R dz1, R h) {
    auto zf = [&](R s) {
        const R s2 = s * s, s3 = s2 * s;
        return (R(2) * s3 - R(3) * s2 + R(1)) * z0 + (s3 - R(2) * s2 + s) * h * dz0 + (R(-2) * s3 + R(3) * s2) * z1 +
               (s3 - s2) * h * dz1;
    };
    R lo = 0, hi = 1, flo = z0;
    for (int it = 0; it < 60; ++it) {
        const R mid = R(0.5) * (lo + hi);
        const R fm = zf(mid);
        if ((fm < R(0)) == (flo < R(0))) { lo = mid; flo = fm; } else { hi = mid; }
    }
    return R(0.5) * (lo + hi);
}

template <class R>
void hermite_point(const R x0[4], const R x1[4], const R k0[4], const R k1[4], R h, R s, R out[4]) {
    const R s2 = s * s, s3 = s2 * s;
    const R h00 = R(2) * s3 - R(3) * s2 + R(1), h10 = s3 - R(2) * s2 + s, h01 = R(-2) * s3 + R(3) * s2, h11 = s3 - s2;
    for (int i = 0; i < 4; ++i) out[i] = h00 * x0[i] + h10 * h * k0[i] + h01 * x1[i] + h11 * h * k1[i];
}

// Event location of the equatorial crossing inside an accepted step: DP45
// sub-steps from the step's start state (x0, p0, f(x0, p0)), the sub-step
// length corrected by Newton on z(l) (dz/dl = k^z), seeded by the cubic
// Hermite root; two sub-steps and a final first-order correction put z at
// rounding level, independent of the step sequence that bracketed it.
template <class R>
void locate_equator(const sirius_metric& m, const sirius_trace_config& c, const R x0[4], const R p0[4],
                    const R kx0[4], const R kp0[4], R hs, R xc[4]) {
    R xn[4], pn[4], k7x[4], k7p[4];
    for (int it = 0; it < 2; ++it) {
        dp45_attempt(m, c, x0, p0, hs, kx0, kp0, xn, pn, k7x, k7p, false);
        if (it == 0) hs -= xn[3] / k7x[3];
    }
    const R dl = -xn[3] / k7x[3];
    for (int i = 0; i < 4; ++i) xc[i] = xn[i] + dl * k7x[i];
    xc[3] = R(0);
}

// Volumetric emission of the engine: over one step segment x0 -> x1 of affine
// length h, Gauss-Legendre points (vol_substeps of them, 1..4) on the step's
// cubic Hermite interpolant (the reference marches the chord with midpoints,
// GTRC001A.cpp:943-958), restricted to the part of the step inside the
// emitting annulus r_in <= r <= r_out (the annulus edges are discontinuities of
// j, so the step is split there), camera-first accumulation per bin:
//   I_b += T_b S (1 - e^{-dtau}),  T_b *= e^{-dtau},
//   j = j0 r^-2 exp(-z^2 / (2 (h_z r)^2)) nu_em^-s  (|z| <= kVolCutoff h_z r),
//   alpha = c_a j,  dtau = alpha (nu_cam / g) dl,  S = g^3 / c_a
// (I_b stored as nu_b^3 I_inv).
constexpr double kVolCutoff = 6.0;  // emission beyond 6 scale heights (e^-18 of the peak) is dropped

// The Hermite parameter in [0, 1] at which r crosses `edge` between the step's
// ends, by bisection (r(0) and r(1) lie on opposite sides of `edge`).
template <class R>
R annulus_edge(const sirius_metric& m, const R x0[4], const R x1[4], const R k0[4], const R k1[4], R h, R r0,
               R edge) {
    R lo = R(0), hi = R(1);
    const bool inside_lo = r0 < edge;
    for (int it = 0; it < 30; ++it) {
        const R f = R(0.5) * (lo + hi);
        R xs[4], d[4];
        hermite_point(x0, x1, k0, k1, h, f, xs);
        if ((radial(m, xs, d) < edge) == inside_lo) lo = f;
        else hi = f;
    }
    return R(0.5) * (lo + hi);
}

template <class R>
void volumetric_segment(const TraceContext& ctx, const R x0[4], const R x1[4], const R k0[4], const R k1[4],
                        const R p[4], R h, R sqrt_m_gtt_cam, const R* nu, Spectra& sp) {
    const auto& c = ctx.cfg;
    int n;
    const double* gx;
    const double* gw;
    gauss_legendre(c.vol_substeps, n, gx, gw);
    const R E = -p[0], Lz = x1[1] * p[2] - x1[2] * p[1];  // p is the state at x1
    const R nu_cam = E / sqrt_m_gtt_cam;
    const R rin = R(ctx.disk_inner), rout = R(ctx.disk_outer);
    R d[4];
    const R r0 = radial(ctx.metric, x0, d), r1 = radial(ctx.metric, x1, d);
    const bool in0 = r0 >= rin && r0 <= rout, in1 = r1 >= rin && r1 <= rout;
    R fa = R(0), fb = R(1);
    if (in0 && !in1) fb = annulus_edge(ctx.metric, x0, x1, k0, k1, h, r0, r1 < rin ? rin : rout);
    if (!in0 && in1) fa = annulus_edge(ctx.metric, x0, x1, k0, k1, h, r0, r0 < rin ? rin : rout);
    const R span = fb - fa;
    for (int s = 0; s < n; ++s) {
        const R f = fa + span * R(gx[s]);
        R xs[4];
        hermite_point(x0, x1, k0, k1, h, f, xs);  // the step's cubic Hermite interpolant
        const R r = radial(ctx.metric, xs, d);
        if (r < rin || r > rout) continue;
        const R zr = xs[3] / (R(c.vol_height_ratio) * r);
        if (std::abs(zr) > R(kVolCutoff)) continue;
        const R jsp = R(c.vol_j0) / (r * r) * std::exp(R(-0.5) * zr * zr);
        const R g = redshift_exact(ctx, xs, r, E, Lz, sqrt_m_gtt_cam);
        if (!(g > R(0))) continue;
        const R dl = h * span * R(gw[s]);
        const R S = g * g * g / R(c.vol_alpha_over_j);
        for (int b = 0; b < c.n_bins; ++b) {
            const R nu_em = nu[b] / g;
            const R jnu = jsp * std::pow(nu_em, -R(c.vol_spectral_index));
            const R dtau = R(c.vol_alpha_over_j) * jnu * (nu_cam / g) * dl;
            const R T = std::exp(-sp.tau[b]);
            sp.I[b] += T * S * (R(1) - std::exp(-dtau));
            sp.tau[b] += dtau;
        }
    }
}

// Largest affine step near the emitting volume, so that the per-step
// quadrature, and hence the spectra, do not depend on the step sequence: half
// the local scale height h_z r over the spatial speed |dx/dl| inside the
// emitting region (r_in <= r <= r_out, |z| <= kVolCutoff h_z r), and outside it
// the distance to that region, so that no step jumps into its interior.
template <class R>
R volume_step_cap(const TraceContext& ctx, const R x[4], const R k[4]) {
    const auto& c = ctx.cfg;
    R d[4];
    const R r = radial(ctx.metric, x, d);
    const R rin = R(ctx.disk_inner), rout = R(ctx.disk_outer);
    const R H = R(c.vol_height_ratio) * std::min(std::max(r, rin), rout);
    const R dist = std::max(std::max(rin - r, r - rout), std::abs(x[3]) - R(kVolCutoff) * H);
    const R v = std::sqrt(k[1] * k[1] + k[2] * k[2] + k[3] * k[3]);
    return std::max(R(0.5) * H, dist) / std::max(v, R(1e-3));
}

// GeodesicTracer volumetric helpers (GTRC001A.cpp:834-912) — compat gray march.
struct CompatVol {
    const sirius_trace_config* c;
    float r_in, r_out;
    float H_over_r = 0.1f, H_power = 0.25f, tau_mid = 10.0f, tau_max = 10.0f;
    int samples = 32;
    float scale_height(float r) const {
        if (r <= 0) return 0;
        float h = H_over_r * std::pow(r / r_in, H_power);
        h = std::clamp(h, 0.01f, 0.5f);
        return h * r;
    }
    bool inside(float r, float z) const {
        if (r < r_in || r > r_out) return false;
        return std::abs(z) <= 3.0f * scale_height(r);
    }
    float opacity(float r, float z) const {
        if (!inside(r, z)) return 0;
        const float H = scale_height(r);
        if (H <= 0) return 0;
        const float zh = z / H, gs = std::exp(-0.5f * zh * zh);
        const float Hr = scale_height(r_in);
        const float k0 = tau_mid / (std::sqrt(2.0f * float(kPi)) * H) * std::pow(r / r_in, -1.5f) * (Hr / H);
        return k0 * gs;
    }
    float temperature(float r, float z) const {
        if (!inside(r, z)) return 0;
        const float Tm = float(c->disk_temperature_inner) * std::pow(r_in / r, 0.75f);
        if (Tm <= 0) return Tm;
        const float H = scale_height(r);
        if (H <= 0) return Tm;
        float zh2 = (std::abs(z) / H) * (std::abs(z) / H);
        zh2 = std::min(zh2, 9.0f);
        const float a4 = 0.8f * 0.8f * 0.8f * 0.8f;
        float f = 1.0f - zh2 * (1.0f - a4) / 9.0f;
        f = std::max(f, a4);
        return Tm * std::pow(f, 0.25f);
    }
};

// Trace one ray. Writes the result record and (engine mode, volumetric) the bins.
template <class R>
void trace_ray(const TraceContext& ctx, const double origin[4], const double dir[4], sirius_ray_result& res,
               double* bins_out) {
    const auto& c = ctx.cfg;
    const auto& m = ctx.metric;
    const bool compat = c.compat != 0;
    std::memset(&res, 0, sizeof(res));
    res.outcome = SIRIUS_MAX_STEPS;
    res.magnification = 1.0f;
    res.min_radius = 1e10f;
    for (int i = 0; i < SIRIUS_MAX_CROSSINGS; ++i) res.disk_g[i] = 1.0f;

    R x[4], p[4], k[4];
    init_state(ctx, origin, dir, x, p, k);
    R E0, L0, Q0;
    invariants(m, x, p, E0, L0, Q0);
    res.E0 = double(E0); res.Lz0 = double(L0); res.Carter0 = double(Q0);

    const bool ks = m.family == SIRIUS_METRIC_KERR_SCHILD;
    const bool mt = m.family == SIRIUS_METRIC_MORRIS_THORNE;
    // horizon radius: compat uses the spin-only r_+ of the "mass"/"spin" keys (GTRC001A.h:365-380)
    double r_hor = -1.0;
    if (compat) {
        const double M = m.M, a = m.a;
        const double hf = double(float(c.horizon_factor));  // TracerConfig stores floats
        r_hor = (a * a >= M * M) ? 2.0 * M * hf : (M + std::sqrt(M * M - a * a)) * hf;
        r_hor = float(r_hor);
    } else if (ks) {
        const double rp = r_plus(m);
        r_hor = rp > 0 ? rp * c.horizon_factor : -1.0;
    }
    const double a_over_M = std::clamp(m.M != 0 ? m.a / m.M : 0.0, -0.998, 0.998);
    const float r_ph = float(2.0 * m.M * (1.0 + std::cos((2.0 / 3.0) * std::acos(std::clamp(-a_over_M, -1.0, 1.0)))));

    // static observer at the camera: sqrt(-g_tt)
    R gcam[4][4], dgcam[4][4][4];
    metric_evaluate(m, x, gcam, dgcam);
    const R sqrt_m_gtt_cam = std::sqrt(std::max(-gcam[0][0], R(1e-30)));

    // impact parameter heuristic (GTRC001A.cpp:208-233)
    if (!mt) {
        const double R0 = std::sqrt(double(x[1] * x[1] + x[2] * x[2] + x[3] * x[3]));
        const double vx = k[1], vy = k[2], vz = k[3], vm = std::sqrt(vx * vx + vy * vy + vz * vz);
        const double vrad = (vx * x[1] + vy * x[2] + vz * x[3]) / R0;
        res.impact_parameter = float(R0 * std::sqrt(std::max(vm * vm - vrad * vrad, 0.0)) / std::max(vm, 1e-10));
    }

    // spectral bins
    R nu[SIRIUS_MAX_BINS];
    Spectra sp;
    const int nb = std::min(c.n_bins, SIRIUS_MAX_BINS);
    for (int b = 0; b < SIRIUS_MAX_BINS; ++b) { sp.I[b] = 0; sp.tau[b] = 0; nu[b] = 0; }
    for (int b = 0; b < nb; ++b)
        nu[b] = (nb == 1) ? R(c.nu_min) : R(c.nu_min) * std::pow(R(c.nu_max / c.nu_min), R(b) / R(nb - 1));
    CompatVol cv{&c, float(ctx.disk_inner), float(ctx.disk_outer)};
    double vol_acc = 0, vol_tau = 0;

    R h = compat ? R(float(c.initial_step)) : R(c.initial_step);
    R k1x[4], k1p[4];
    rhs(m, x, p, k1x, k1p, compat);
    if (compat) for (int i = 0; i < 4; ++i) k1x[i] = k[i];  // the reference's stage 1 uses the stored velocity

    float min_r = 1e10f;
    float prev_phi = float(std::atan2(double(x[2]), double(x[1])));
    float prev_z = float(x[3]);
    double prev_phi_d = std::atan2(double(x[2]), double(x[1]));
    double prev_z_d = double(x[3]);
    int eq = 0;
    float tphi = 0.0f;
    double tphi_d = 0.0;
    float null_max = 0.0f;
    int steps = 0, rejected = 0, attempts = 0;
    const int max_attempts = c.max_steps * 64 + 1024;
    double intensity = 0;

    while (steps < c.max_steps) {
        R xn[4], pn[4], k7x[4], k7p[4];
        if (compat) {
            // the reference recomputes p from the stored velocity each step (PHGD001A.cpp:537-541)
            R g0[4][4], dg0[4][4][4];
            metric_evaluate(m, x, g0, dg0);
            lower(g0, k, p);
            for (int mu = 0; mu < 4; ++mu) {
                R s = 0;
                for (int r = 0; r < 4; ++r)
                    for (int q = 0; q < 4; ++q) s += dg0[mu][r][q] * k[r] * k[q];
                k1p[mu] = R(float(R(0.5) * s));
                k1x[mu] = k[mu];
            }
        }
        const bool symp = !compat && c.integrator == SIRIUS_INTEGRATOR_SYMPLECTIC;
        R err;
        if (symp) {  // fixed d-lambda, always accepted
            for (int i = 0; i < 4; ++i) { xn[i] = x[i]; pn[i] = p[i]; }
            // d-lambda shrinks near the horizon as SymplecticIntegratorD::integrate does
            // (h0 min(1, ((r - r_+)/r_+)^2), PHSI001A.h:260-263)
            R hs = R(c.symplectic_step);
            if (r_hor > 0) {
                R dd[4];
                const R rp = R(r_plus(m));
                const R q = (radial(m, x, dd) - rp) / rp;
                hs = std::max(R(c.min_step), hs * std::min(R(1), q * q));
            }
            symplectic_step(m, c.symplectic_order, hs, xn, pn);
            rhs(m, xn, pn, k7x, k7p, false);
            err = R(0);
            h = hs;
        } else {
            err = dp45_attempt(m, c, x, p, h, k1x, k1p, xn, pn, k7x, k7p, compat);
        }
        ++attempts;
        if (!(err <= R(1))) {  // reject (NaN errors reject too)
            ++rejected;
            h = optimal_step(h, std::isfinite(double(err)) ? err : R(1e10), c, compat);
            if (!compat && c.enable_volumetric && c.enable_disk && m.family == SIRIUS_METRIC_KERR_SCHILD && r_hor > 0)
                h = std::max(R(c.min_step), std::min(h, volume_step_cap(ctx, x, k1x)));
            if (h <= (compat ? R(float(c.min_step)) : R(c.min_step))) {
                res.outcome = compat ? SIRIUS_MAX_STEPS : SIRIUS_STEP_UNDERFLOW;
                ++steps;
                break;
            }
            if (compat) {  // a rejected step ends the ray in the reference (GTRC001A.cpp:272-277)
                res.outcome = SIRIUS_MAX_STEPS;
                ++steps;
                break;
            }
            if (attempts > max_attempts) { res.outcome = SIRIUS_STEP_UNDERFLOW; break; }
            continue;
        }
        // accepted
        R x0[4], k0v[4], p0[4], k0p[4];
        for (int i = 0; i < 4; ++i) { x0[i] = x[i]; k0v[i] = compat ? k[i] : k1x[i]; p0[i] = p[i]; k0p[i] = k1p[i]; }
        const R hstep = h;
        if (!symp) h = optimal_step(h, err, c, compat);
        if (!symp && !compat && c.enable_volumetric && c.enable_disk && m.family == SIRIUS_METRIC_KERR_SCHILD && r_hor > 0)
            h = std::max(R(c.min_step), std::min(h, volume_step_cap(ctx, xn, k7x)));
        ++steps;
        bool bad = false;
        for (int i = 0; i < 4; ++i) bad |= !std::isfinite(double(xn[i])) || !std::isfinite(double(k7x[i]));
        if (compat) {
            for (int i = 0; i < 4; ++i) { x[i] = xn[i]; k[i] = k7x[i]; }
            if (bad) { res.outcome = SIRIUS_MAX_STEPS; res.flags |= SIRIUS_FLAG_NUMERICAL_FAILURE; break; }
            // periodic null re-normalisation (PHGD001A.cpp:609-638)
            R g1[4][4], dg1[4][4][4];
            metric_evaluate(m, x, g1, dg1);
            const R nv = inner(g1, k, k);
            if (std::abs(double(nv)) > 1e-6) {
                R kk[4] = {k[0], k[1], k[2], k[3]};
                normalize_null(g1, kk, true);
                bool ok = true;
                for (int i = 0; i < 4; ++i) ok &= std::isfinite(double(kk[i]));
                if (ok) for (int i = 0; i < 4; ++i) k[i] = kk[i];
            }
        } else {
            for (int i = 0; i < 4; ++i) { x[i] = xn[i]; p[i] = pn[i]; k1x[i] = k7x[i]; k1p[i] = k7p[i]; }
            bool badp = bad;
            for (int i = 0; i < 4; ++i) badp |= !std::isfinite(double(pn[i]));
            if (badp) { res.outcome = SIRIUS_NUMERICAL_FAILURE; break; }
            if (c.projection_period > 0 && (steps % c.projection_period) == 0) {
                R pb[4] = {p[0], p[1], p[2], p[3]};
                const R before = project_null(m, x, p);
                null_max = std::max(null_max, float(std::abs(double(before))));
                // a projection that moved p beyond 1e-10 (relative) makes f(x, p) stale: recompute it
                R dp = 0, pm = 0;
                for (int i = 0; i < 4; ++i) {
                    dp = std::max(dp, std::abs(p[i] - pb[i]));
                    pm = std::max(pm, std::abs(p[i]));
                }
                if (dp > R(1e-10) * pm) rhs(m, x, p, k1x, k1p, false);
            } else {
                null_max = std::max(null_max, float(std::abs(double(null_value(m, x, p)))));
            }
            for (int i = 0; i < 4; ++i) k[i] = k1x[i];
        }

        // radii
        R d[4];
        const double Reu = std::sqrt(double(x[1] * x[1] + x[2] * x[2] + x[3] * x[3]));
        const double rbl = mt ? double(x[1]) : double(radial(m, x, d));
        const double rr = compat ? Reu : rbl;
        if (float(rr) < min_r) min_r = float(rr);

        // winding (GTRC001A.cpp:294-309)
        if (!mt) {
            if (compat) {
                const float cphi = float(std::atan2(double(x[2]), double(x[1])));
                const float cz = float(x[3]);
                if (prev_z * cz < 0) ++eq;
                float dphi = cphi - prev_phi;
                if (dphi > kPi) dphi -= 2.0f * float(kPi);
                if (dphi < -kPi) dphi += 2.0f * float(kPi);
                tphi += std::abs(dphi);
                prev_phi = cphi; prev_z = cz;
            } else {
                const double cphi = std::atan2(double(x[2]), double(x[1]));
                const double cz = double(x[3]);
                if (prev_z_d * cz < 0) ++eq;
                double dphi = cphi - prev_phi_d;
                if (dphi > kPi) dphi -= 2.0 * kPi;
                if (dphi < -kPi) dphi += 2.0 * kPi;
                tphi_d += std::abs(dphi);
                prev_phi_d = cphi; prev_z_d = cz;
            }
        }

        // spiral early-out (GTRC001A.cpp:322-352), step index = steps - 1
        const int sidx = steps - 1;
        if (c.spiral_check && !mt && (sidx % 100 == 0) && sidx > 100) {
            const float ratio = min_r / r_ph;
            const float tot = compat ? tphi : float(tphi_d);
            if (ratio < 1.5f && ratio > 0.9f && tot > 2.0f * float(kPi)) {
                const double vx = double(k[1]), vy = double(k[2]), vz = double(k[3]);
                const double vrad = (double(x[1]) * vx + double(x[2]) * vy + double(x[3]) * vz) / Reu;
                const double vt = std::sqrt(vx * vx + vy * vy + vz * vz);
                if (std::abs(vrad) / std::max(vt, 1e-10) < 0.3) {
                    if (res.n_crossings == 0) res.outcome = SIRIUS_SPIRALING;
                    break;
                }
            }
        }

        // horizon (GTRC001A.cpp:358-367)
        if (r_hor > 0 && rr < r_hor) {
            res.outcome = SIRIUS_HORIZON;
            break;
        }
        // throat (Morris-Thorne: the metric clamps r >= 1.001 b0)
        if (mt && double(x[1]) <= 1.001 * m.b0 * 1.0001) {
            res.outcome = SIRIUS_THROAT;
            break;
        }
        // escape (GTRC001A.cpp:369-434)
        const double Resc = mt ? double(x[1]) : Reu;
        if (Resc > (compat ? double(float(c.escape_radius)) : c.escape_radius)) {
            const double vrad = mt ? double(k[1]) : (double(x[1] * k[1] + x[2] * k[2] + x[3] * k[3]));
            if (vrad > 0) {
                if (res.n_crossings == 0) res.outcome = SIRIUS_ESCAPED;
                const float ratio = min_r / r_ph;
                if (ratio < 1.5f) {
                    res.flags |= SIRIUS_FLAG_PHOTON_RING;
                    res.magnification = ratio > 1.0f ? std::min(1.0f + 2.0f / std::max(ratio - 1.0f, 0.1f), 20.0f) : 20.0f;
                }
                break;
            }
        }
        if (!ks || !c.enable_disk || (!compat && r_hor <= 0)) continue;  // the disk needs a horizon

        // volumetric
        if (c.enable_volumetric) {
            if (compat) {
                const float pr = float(std::sqrt(double(x0[1] * x0[1] + x0[2] * x0[2]))), pz = float(x0[3]);
                const float cr = float(std::sqrt(double(x[1] * x[1] + x[2] * x[2]))), cz = float(x[3]);
                if (cv.inside(pr, pz) || cv.inside(cr, cz)) {
                    const double dx = double(x[1] - x0[1]), dy = double(x[2] - x0[2]), dz = double(x[3] - x0[3]);
                    const double L = std::sqrt(dx * dx + dy * dy + dz * dz);
                    if (L >= 1e-10) {
                        const int N = cv.samples;
                        const double ds = L / N;
                        double acc = 0, tau = 0;
                        for (int i = 0; i < N; ++i) {
                            const double tt = (i + 0.5) * ds;
                            const double sx = double(x0[1]) + tt * dx / L, sy = double(x0[2]) + tt * dy / L,
                                         sz = double(x0[3]) + tt * dz / L;
                            const double rc = std::sqrt(sx * sx + sy * sy);
                            if (!cv.inside(float(rc), float(sz))) continue;
                            const float kr = cv.opacity(float(rc), float(sz)), T = cv.temperature(float(rc), float(sz));
                            if (kr <= 0 || T <= 0) continue;
                            const double dtau = kr * ds;
                            const double B = std::pow(T / float(c.disk_temperature_inner), 4.0);
                            const double tr = std::exp(-dtau);
                            acc = acc * tr + B * (1.0 - tr);
                            tau += dtau;
                            if (tau > cv.tau_max) break;
                        }
                        vol_acc = acc; vol_tau = tau;
                        if (tau > 0.01 && res.outcome != SIRIUS_DISK_HIT) {
                            res.outcome = SIRIUS_DISK_HIT;
                            res.disk_r[0] = cr;
                            res.disk_phi[0] = float(std::atan2(double(x[2]), double(x[1])));
                        }
                    }
                }
                continue;
            }
            volumetric_segment(ctx, x0, x, k0v, k, p, hstep, sqrt_m_gtt_cam, nu, sp);
        }

        // thin disk crossing (GTRC001A.h:404-431, GTRC001A.cpp:468-555)
        if (double(x0[3]) * double(x[3]) >= 0) continue;
        double rc, phc;
        R xc[4];
        if (compat) {
            const double al = -double(x0[3]) / (double(x[3]) - double(x0[3]));
            const double xcx = double(x0[1]) + al * double(x[1] - x0[1]), ycx = double(x0[2]) + al * double(x[2] - x0[2]);
            rc = std::sqrt(xcx * xcx + ycx * ycx);
            phc = std::atan2(ycx, xcx);
            xc[1] = R(xcx); xc[2] = R(ycx);
        } else {
            const R s = hermite_z_root(x0[3], x[3], k0v[3], k[3], hstep);
            locate_equator(m, c, x0, p0, k0v, k0p, s * hstep, xc);
            rc = double(radial(m, xc, d));
            phc = std::atan2(double(xc[2]), double(xc[1]));
        }
        const double din = compat ? double(float(ctx.disk_inner)) : ctx.disk_inner;
        const double dout = compat ? double(float(ctx.disk_outer)) : ctx.disk_outer;
        if (rc < din || rc > dout) continue;
        if (res.n_crossings < SIRIUS_MAX_CROSSINGS) {
            const int n = res.n_crossings;
            res.disk_r[n] = float(rc);
            res.disk_phi[n] = float(phc);
            if (compat) {
                const double vel[4] = {double(k[0]), double(k[1]), double(k[2]), double(k[3])};
                res.disk_g[n] = float(redshift_compat(m, float(rc), float(phc), vel));
            } else {
                res.disk_g[n] = float(redshift_exact(ctx, xc, R(rc), -p[0], x[1] * p[2] - x[2] * p[1], sqrt_m_gtt_cam));
            }
            const double F = nt_flux(rc, m.M != 0 ? m.a / m.M : 0.0, ctx.disk_inner, ctx.disk_outer);
            res.disk_flux[n] = float(F);
            const double gg = compat ? double(res.disk_g[n]) : double(redshift_exact(ctx, xc, R(rc), -p[0], x[1] * p[2] - x[2] * p[1], sqrt_m_gtt_cam));
            intensity += std::exp(-c.crossing_weight_decay * n) * gg * gg * gg * gg * F;
            if (n == 0) res.outcome = SIRIUS_DISK_HIT;
            res.n_crossings = n + 1;
            const float ratio = min_r / r_ph;
            if (ratio < 1.5f) {
                res.flags |= SIRIUS_FLAG_PHOTON_RING;
                res.magnification = ratio > 1.0f ? std::min(1.0f + 2.0f / std::max(ratio - 1.0f, 0.05f), 100.0f) : 100.0f;
            }
        }
        if (res.n_crossings >= SIRIUS_MAX_CROSSINGS) break;
    }

    res.steps = steps;
    res.rejected = rejected;
    res.min_radius = std::min(res.min_radius, min_r);
    res.equatorial_crossings = eq;
    res.total_phi_change = compat ? tphi : float(tphi_d);
    res.image_order = eq >= 1 ? (eq + 1) / 2 : 0;
    for (int i = 0; i < 4; ++i) {
        res.final_x[i] = double(x[i]);
        res.final_p[i] = double(p[i]);
        res.final_k[i] = float(k[i]);
    }
    if (compat) {  // p of the returned state
        R g1[4][4], dg1[4][4][4];
        metric_evaluate(m, x, g1, dg1);
        R pp[4];
        lower(g1, k, pp);
        for (int i = 0; i < 4; ++i) res.final_p[i] = double(pp[i]);
        R E, L, Q;
        invariants(m, x, pp, E, L, Q);
        res.E = double(E); res.Lz = double(L); res.Carter = double(Q);
        res.null_final = float(std::abs(double(inner(g1, k, k))));
        res.intensity = float(intensity + vol_acc);
        res.optical_depth = float(vol_tau);
    } else {
        R E, L, Q;
        invariants(m, x, p, E, L, Q);
        res.E = double(E); res.Lz = double(L); res.Carter = double(Q);
        res.null_final = float(std::abs(double(null_value(m, x, p))));
        res.intensity = float(intensity);
        double taumax = 0;
        for (int b = 0; b < nb; ++b) taumax = std::max(taumax, double(sp.tau[b]));
        res.optical_depth = float(taumax);
    }
    res.null_drift_max = null_max;
    if (bins_out)
        for (int b = 0; b < nb; ++b) bins_out[b] = double(sp.I[b]);
}

}  // namespace oracle

// spacetime.cuh — metric families on the device.
//
// Each family supplies, in any precision T:
//   rhs()          Hamilton's equations  dx^mu/dl = g^{mu nu} p_nu,
//                  dp_mu/dl = 1/2 d_mu g_{rs} k^r k^s  (PHGD001A.cpp:159-202),
//                  with d_mu g from register-resident dual numbers (dual.cuh);
//   ginv()         the inverse metric as a bilinear form (for the FP64
//                  constraint re-projection and the null value);
//   radial()       the radial coordinate of the family and its gradient dr;
//   metric_full()  g_{mu nu} and d_l g_{mu nu} (IMetric::evaluate, PHMT000A.h:38).
// The Kerr-Schild family never forms a 4x4 inverse: with the null covector
// l_mu = (1, (rx+ay)/(r^2+a^2), (ry-ax)/(r^2+a^2), z/r) (eta-null),
// g = eta + H l l  has  g^{-1} = eta - H l# l#  (l# = eta l), and the
// reference's "simplified" Lambda term -Lambda R^2/3 on g_tt
// (PHMT100A.h:362-369) is folded in exactly by a Sherman-Morrison update.
#pragma once

#include "dual.cuh"
#include "../../include/sirius_cuda.h"

namespace sirius {

struct MetricDev {
    int family;
    int shape;
    double M, a, Q, Lambda;
    double a2, Q2, lam3, sqrtM;   // a^2, Q^2, Lambda/3
    int has_lambda;        // |Lambda| > 1e-15 (PHMT100A.h:365)
    double b0, Phi0, gtt_mt;  // Morris-Thorne: g_tt = -exp(2 Phi0)
    double vs, sigma, Rb, inv_2tanhsR;  // Alcubierre
    // FP32 copies for the single-precision paths (rounded once on the host)
    float fa, fa2, fM2, fQ2, flam3, fsqrtM;
};

// A launch constant in precision T: the FP32 copy for float, else the double.
template <class T>
SIRIUS_HD __forceinline__ T cst(double d, float) { return T(d); }
template <>
SIRIUS_HD __forceinline__ float cst<float>(double, float f) { return f; }

// Host: the per-metric constants the device code reads.
inline MetricDev metric_dev(const sirius_metric& s) {
    MetricDev m{};
    m.family = s.family;
    m.shape = s.shape;
    m.M = s.M; m.a = s.a; m.Q = s.Q; m.Lambda = s.Lambda;
    m.a2 = s.a * s.a; m.Q2 = s.Q * s.Q; m.lam3 = s.Lambda / 3.0; m.sqrtM = std::sqrt(s.M > 0.0 ? s.M : 0.0);
    m.has_lambda = std::fabs(s.Lambda) > 1e-15;
    m.b0 = s.b0; m.Phi0 = s.Phi0; m.gtt_mt = -std::exp(2.0 * s.Phi0);
    m.vs = s.vs; m.sigma = s.sigma; m.Rb = s.R;
    m.inv_2tanhsR = (s.sigma * s.R != 0.0) ? 1.0 / (2.0 * std::tanh(s.sigma * s.R)) : 0.0;
    m.fa = float(m.a); m.fa2 = float(m.a2); m.fM2 = float(2.0 * m.M); m.fQ2 = float(m.Q2);
    m.flam3 = float(m.lam3); m.fsqrtM = float(m.sqrtM);
    return m;
}

template <class T>
SIRIUS_HD __forceinline__ T tmax(T a, T b) { return a > b ? a : b; }

// ---------------------------------------------------------------------------
// Kerr-Schild family (PHMT100A.h:198-396): H and l_i as dual numbers.
// r solves r^4 - (R^2 - a^2) r^2 - a^2 z^2 = 0; its gradient enters as the
// implicit-function seed  dr = (r x, r y, z (r^2 + a^2) / r) / sqrt(disc).
// ---------------------------------------------------------------------------
template <class T>
struct KSPieces {
    D3<T> H, l1, l2, l3;
    T r;
};

template <class T>
SIRIUS_HD __forceinline__ void ks_pieces(const MetricDev& m, T x, T y, T z, KSPieces<T>& o) {
    const T a = T(m.a), a2 = T(m.a2);
    const T R2 = x * x + y * y + z * z;
    const T Rm2 = R2 - a2;
    const T disc = tmax(Rm2 * Rm2 + T(4) * a2 * z * z, T(1e-20));
    const T sd = sqrtp_(disc);
    const T r2 = tmax((Rm2 + sd) * T(0.5), T(1e-10));
    const T r = sqrtp_(r2);
    const T isd = rcp_(sd);
    const T ir = rcp_(r);
    const D3<T> rd = dwith(r, r * x * isd, r * y * isd, z * (r2 + a2) * isd * ir);
    const D3<T> X = dvar(x, 0), Y = dvar(y, 1), Z = dvar(z, 2);
    const D3<T> rr2 = rd * rd;
    const D3<T> iden = inv(rr2 + a2);
    o.l1 = (rd * X + Y * a) * iden;
    o.l2 = (rd * Y - X * a) * iden;
    o.l3 = Z * dwith(ir, -ir * ir * rd.d[0], -ir * ir * rd.d[1], -ir * ir * rd.d[2]);
    const D3<T> num = (rd * T(2.0 * m.M) - T(m.Q2)) * rr2;
    const D3<T> fden = rr2 * rr2 + Z * Z * a2;
    o.H = num * inv(fden);
    o.r = r;
}

template <class T>
SIRIUS_HD __forceinline__ void ks_rhs(const MetricDev& m, const T x[4], const T p[4], T k[4], T f[4]) {
    KSPieces<T> P;
    ks_pieces(m, x[1], x[2], x[3], P);
    const T H = P.H.v, l1 = P.l1.v, l2 = P.l2.v, l3 = P.l3.v;
    // g^{-1} p = eta p - H l# (l# . p), l# = (-1, l1, l2, l3)
    const T lp = -p[0] + l1 * p[1] + l2 * p[2] + l3 * p[3];
    k[0] = -p[0] + H * lp;
    k[1] = p[1] - H * l1 * lp;
    k[2] = p[2] - H * l2 * lp;
    k[3] = p[3] - H * l3 * lp;
    if (m.has_lambda) {
        const T c = T(m.lam3) * (x[1] * x[1] + x[2] * x[2] + x[3] * x[3]);
        const T w0 = -T(1) - H, w1 = H * l1, w2 = H * l2, w3 = H * l3;
        const T s = c * (w0 * p[0] + w1 * p[1] + w2 * p[2] + w3 * p[3]) * rcp_(T(1) + c * (T(1) + H));
        k[0] += s * w0; k[1] += s * w1; k[2] += s * w2; k[3] += s * w3;
    }
    // dp_lambda = 1/2 dH (l.k)^2 + H (l.k)(dl.k) [- Lambda x_lambda (k^0)^2 / 3]
    const T lk = k[0] + l1 * k[1] + l2 * k[2] + l3 * k[3];
    f[0] = T(0);
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const T dlk = P.l1.d[i] * k[1] + P.l2.d[i] * k[2] + P.l3.d[i] * k[3];
        f[i + 1] = lk * (T(0.5) * P.H.d[i] * lk + H * dlk);
    }
    if (m.has_lambda) {
        const T q = T(m.lam3) * k[0] * k[0];
        f[1] -= q * x[1]; f[2] -= q * x[2]; f[3] -= q * x[3];
    }
}

// The same right-hand side with the forward-mode tangents of ks_pieces
// propagated term by term: the coordinate seeds dx = (1, 0, 0), ... have zero
// components, and an IEEE product with a zero cannot be dropped at compile time
// (inf * 0 is NaN), so the generic dual arithmetic pays for every one of them.
// Here only the non-zero terms are formed:
//   dr  = (r x, r y, z (r^2 + a^2) / r) / sqrt(disc)
//   d(1/(r^2 + a^2)) = -2 r / (r^2 + a^2)^2 dr
//   d l1 = (x dr + (r, a, 0)) / (r^2 + a^2) + (r x + a y) d(1/(r^2 + a^2)), l2 alike
//   d l3 = (0, 0, 1) / r - z / r^2 dr
//   d H  = ((2 M r^2 + 2 r (2 M r - Q^2) - H 4 r^3) dr - H (0, 0, 2 a^2 z)) / fden
// with num = (2 M r - Q^2) r^2, fden = r^4 + a^2 z^2, H = num / fden.
template <class T>
SIRIUS_HD __forceinline__ void ks_rhs_fast(const MetricDev& m, const T x[4], const T p[4], T k[4], T f[4]) {
    const T a = cst<T>(m.a, m.fa), a2 = cst<T>(m.a2, m.fa2);
    const T X = x[1], Y = x[2], Z = x[3];
    const T zz = Z * Z;
    const T R2 = X * X + Y * Y + zz;
    const T Rm2 = R2 - a2;
    const T a2zz = a2 * zz;
    const T disc = tmax(Rm2 * Rm2 + T(4) * a2zz, T(1e-20));
    const T sd = sqrtp_(disc);
    const T r2 = tmax((Rm2 + sd) * T(0.5), T(1e-10));
    const T r = sqrtp_(r2);
    const T isd = rcp_(sd), ir = rcp_(r);
    const T den = r2 + a2;
    const T risd = r * isd;
    const T rx = risd * X, ry = risd * Y, rz = Z * den * isd * ir;
    const T iden = rcp_(den);
    const T gi = -T(2) * r * iden * iden;
    const T n1 = r * X + a * Y, n2 = r * Y - a * X;
    const T l1 = n1 * iden, l2 = n2 * iden;
    const T n1g = n1 * gi, n2g = n2 * gi;
    const T l1d0 = (X * rx + r) * iden + n1g * rx, l1d1 = (X * ry + a) * iden + n1g * ry,
            l1d2 = X * rz * iden + n1g * rz;
    const T l2d0 = (Y * rx - a) * iden + n2g * rx, l2d1 = (Y * ry + r) * iden + n2g * ry,
            l2d2 = Y * rz * iden + n2g * rz;
    const T l3 = Z * ir;
    const T zi2 = -l3 * ir;
    const T l3d0 = zi2 * rx, l3d1 = zi2 * ry, l3d2 = zi2 * rz + ir;
    const T M2 = cst<T>(2.0 * m.M, m.fM2);
    const T q = M2 * r - cst<T>(m.Q2, m.fQ2);
    const T fden = r2 * r2 + a2zz;
    const T ifd = rcp_(fden);
    const T H = q * r2 * ifd;
    const T w = (M2 * r2 + T(2) * r * q - H * T(4) * r2 * r) * ifd;
    const T Hd0 = w * rx, Hd1 = w * ry, Hd2 = w * rz - H * ifd * T(2) * a2 * Z;
    // k = g^{-1} p = eta p - H l# (l# . p), l# = (-1, l1, l2, l3)
    const T lp = -p[0] + l1 * p[1] + l2 * p[2] + l3 * p[3];
    const T Hlp = H * lp;
    k[0] = -p[0] + Hlp;
    k[1] = p[1] - l1 * Hlp;
    k[2] = p[2] - l2 * Hlp;
    k[3] = p[3] - l3 * Hlp;
    if (m.has_lambda) {
        const T c = cst<T>(m.lam3, m.flam3) * R2;
        const T w0 = -T(1) - H, w1 = H * l1, w2 = H * l2, w3 = H * l3;
        const T s = c * (w0 * p[0] + w1 * p[1] + w2 * p[2] + w3 * p[3]) * rcp_(T(1) + c * (T(1) + H));
        k[0] += s * w0; k[1] += s * w1; k[2] += s * w2; k[3] += s * w3;
    }
    // dp_lambda = 1/2 dH (l.k)^2 + H (l.k)(dl.k) [- Lambda x_lambda (k^0)^2 / 3]
    const T lk = k[0] + l1 * k[1] + l2 * k[2] + l3 * k[3];
    const T hlk = T(0.5) * lk;
    f[0] = T(0);
    f[1] = lk * (Hd0 * hlk + H * (l1d0 * k[1] + l2d0 * k[2] + l3d0 * k[3]));
    f[2] = lk * (Hd1 * hlk + H * (l1d1 * k[1] + l2d1 * k[2] + l3d1 * k[3]));
    f[3] = lk * (Hd2 * hlk + H * (l1d2 * k[1] + l2d2 * k[2] + l3d2 * k[3]));
    if (m.has_lambda) {
        const T qq = cst<T>(m.lam3, m.flam3) * k[0] * k[0];
        f[1] -= qq * X; f[2] -= qq * Y; f[3] -= qq * Z;
    }
}

// ---------------------------------------------------------------------------
// Morris-Thorne (PHMT101A.h:195-345), chart (t, r, theta, phi); r clamped to
// >= 1.001 b0 as the reference does (:293); g diagonal.
// ---------------------------------------------------------------------------
template <class T>
SIRIUS_HD __forceinline__ D3<T> mt_grr(const MetricDev& m, T r) {
    const T b0 = T(m.b0);
    const D3<T> R = dvar(tmax(r, b0 * T(1.001)), 0);
    D3<T> b;
    if (m.shape == SIRIUS_WORMHOLE_ZERO_TIDAL) b = dconst(b0);
    else if (m.shape == SIRIUS_WORMHOLE_ABSURDLY_BENIGN) b = (dconst(T(2)) - inv(R) * b0) * b0;
    else b = inv(R) * (b0 * b0);  // Ellis
    D3<T> f = dconst(T(1)) - b * inv(R);
    if (f.v < T(1e-10)) f = dconst(T(1e-10));
    return inv(f);
}

template <class T>
SIRIUS_HD __forceinline__ void mt_rhs(const MetricDev& m, const T x[4], const T p[4], T k[4], T f[4]) {
    const T r = tmax(x[1], T(m.b0) * T(1.001));
    const T s = sin(x[2]), c = cos(x[2]);
    const T s2 = tmax(s * s, T(1e-24));
    const D3<T> grr = mt_grr(m, x[1]);
    const T r2 = r * r;
    k[0] = p[0] * rcp_(T(m.gtt_mt));
    k[1] = p[1] * rcp_(grr.v);
    k[2] = p[2] * rcp_(r2);
    k[3] = p[3] * rcp_(r2 * s2);
    f[0] = T(0);
    f[1] = T(0.5) * grr.d[0] * k[1] * k[1] + r * (k[2] * k[2] + s2 * k[3] * k[3]);
    f[2] = r2 * s * c * k[3] * k[3];
    f[3] = T(0);
}

// ---------------------------------------------------------------------------
// Alcubierre (PHMT102A.h:136-229), Cartesian, static bubble at the origin:
// g_tt = -(1 - v^2 f^2), g_tx = -v f;  g^{tt} = -1, g^{tx} = -v f, g^{xx} = 1 - v^2 f^2.
// ---------------------------------------------------------------------------
template <class T>
SIRIUS_HD __forceinline__ D3<T> alc_f(const MetricDev& m, T x, T y, T z) {
    const T rs = tmax(sqrt_(x * x + y * y + z * z), T(1e-10));
    const T irs = rcp_(rs);
    const D3<T> R = dwith(rs, x * irs, y * irs, z * irs);
    const T sg = T(m.sigma), Rb = T(m.Rb);
    return (dtanh((R + Rb) * sg) - dtanh((R - Rb) * sg)) * T(m.inv_2tanhsR);
}

template <class T>
SIRIUS_HD __forceinline__ void alc_rhs(const MetricDev& m, const T x[4], const T p[4], T k[4], T f[4]) {
    const D3<T> F = alc_f(m, x[1], x[2], x[3]);
    const T v = T(m.vs), vf = v * F.v;
    k[0] = -p[0] - vf * p[1];
    k[1] = -vf * p[0] + (T(1) - vf * vf) * p[1];
    k[2] = p[2];
    k[3] = p[3];
    // dp = v df (v f (k^t)^2 - k^t k^x)
    const T q = v * (vf * k[0] * k[0] - k[0] * k[1]);
    f[0] = T(0);
    f[1] = q * F.d[0];
    f[2] = q * F.d[1];
    f[3] = q * F.d[2];
}

// FAM selects the metric family at compile time (a kernel specialised for one
// family carries one right-hand side); kAnyFamily dispatches on m.family.
constexpr int kAnyFamily = -1;

template <class T, int FAM = kAnyFamily>
SIRIUS_HD __forceinline__ void rhs(const MetricDev& m, const T x[4], const T p[4], T k[4], T f[4]) {
    if constexpr (FAM == SIRIUS_METRIC_KERR_SCHILD) ks_rhs_fast(m, x, p, k, f);
    else if constexpr (FAM == SIRIUS_METRIC_MORRIS_THORNE) mt_rhs(m, x, p, k, f);
    else if constexpr (FAM == SIRIUS_METRIC_ALCUBIERRE) alc_rhs(m, x, p, k, f);
    else if (m.family == SIRIUS_METRIC_KERR_SCHILD) ks_rhs_fast(m, x, p, k, f);
    else if (m.family == SIRIUS_METRIC_MORRIS_THORNE) mt_rhs(m, x, p, k, f);
    else alc_rhs(m, x, p, k, f);
}

// Whether a ray of family FAM (or, for kAnyFamily, of m.family) is of family F.
template <int FAM>
SIRIUS_HD __forceinline__ bool is_family(const MetricDev& m, int F) {
    if constexpr (FAM == kAnyFamily) return m.family == F;
    else return FAM == F;
}

// ---------------------------------------------------------------------------
// Inverse metric as a bilinear form, evaluated once at x for up to three
// covectors: out = {g^{-1}(u,u), g^{-1}(u,v), g^{-1}(v,v)}. Also returns the
// family's radial coordinate r and its gradient d (the projection direction).
// ---------------------------------------------------------------------------
struct InvForm {
    double r;      // radial coordinate (KS: Boyer-Lindquist r; MT: r; Alcubierre: R)
    double d[4];   // dr
    double H, l[4], c, w[4], sm;  // KS pieces
    double diag[4];               // MT
    double vf;                    // Alcubierre
};

__device__ __forceinline__ void inv_form(const MetricDev& m, const double x[4], InvForm& F) {
    F.d[0] = 0.0;
    if (m.family == SIRIUS_METRIC_MORRIS_THORNE) {
        const double r = fmax(x[1], m.b0 * 1.001);
        const double s = sin(x[2]);
        const double s2 = fmax(s * s, 1e-24);
        const D3<double> grr = mt_grr<double>(m, x[1]);
        F.r = x[1];
        F.d[1] = 1.0; F.d[2] = 0.0; F.d[3] = 0.0;
        F.diag[0] = 1.0 / m.gtt_mt; F.diag[1] = 1.0 / grr.v; F.diag[2] = 1.0 / (r * r); F.diag[3] = 1.0 / (r * r * s2);
        return;
    }
    const double X = x[1], Y = x[2], Z = x[3];
    const double R2 = X * X + Y * Y + Z * Z;
    if (m.family == SIRIUS_METRIC_ALCUBIERRE) {
        const double Rr = sqrt(R2);
        F.r = Rr;
        F.d[1] = X / Rr; F.d[2] = Y / Rr; F.d[3] = Z / Rr;
        const D3<double> f = alc_f<double>(m, X, Y, Z);
        F.vf = m.vs * f.v;
        return;
    }
    const double a2 = m.a2, Rm2 = R2 - a2;
    const double sd = sqrt(fmax(Rm2 * Rm2 + 4.0 * a2 * Z * Z, 1e-20));
    const double r2 = fmax(0.5 * (Rm2 + sd), 1e-10);
    const double r = sqrt(r2);
    F.r = r;
    if (m.a == 0.0) {
        const double Rr = sqrt(R2);
        F.d[1] = X / Rr; F.d[2] = Y / Rr; F.d[3] = Z / Rr;
    } else {
        F.d[1] = r * X / sd; F.d[2] = r * Y / sd; F.d[3] = Z * (r2 + a2) / (r * sd);
    }
    const double den = r2 + a2;
    F.l[0] = -1.0;  // l# = eta l
    F.l[1] = (r * X + m.a * Y) / den;
    F.l[2] = (r * Y - m.a * X) / den;
    F.l[3] = Z / r;
    F.H = (2.0 * m.M * r - m.Q2) * r2 / (r2 * r2 + a2 * Z * Z);
    F.c = m.has_lambda ? m.lam3 * R2 : 0.0;
    F.w[0] = -1.0 - F.H; F.w[1] = F.H * F.l[1]; F.w[2] = F.H * F.l[2]; F.w[3] = F.H * F.l[3];
    F.sm = F.c / (1.0 + F.c * (1.0 + F.H));
}

__device__ __forceinline__ double inv_apply(const MetricDev& m, const InvForm& F, const double u[4], const double v[4]) {
    if (m.family == SIRIUS_METRIC_MORRIS_THORNE)
        return F.diag[0] * u[0] * v[0] + F.diag[1] * u[1] * v[1] + F.diag[2] * u[2] * v[2] + F.diag[3] * u[3] * v[3];
    if (m.family == SIRIUS_METRIC_ALCUBIERRE)
        return -u[0] * v[0] - F.vf * (u[0] * v[1] + u[1] * v[0]) + (1.0 - F.vf * F.vf) * u[1] * v[1] + u[2] * v[2] +
               u[3] * v[3];
    const double eta = -u[0] * v[0] + u[1] * v[1] + u[2] * v[2] + u[3] * v[3];
    const double lu = F.l[0] * u[0] + F.l[1] * u[1] + F.l[2] * u[2] + F.l[3] * u[3];
    const double lv = F.l[0] * v[0] + F.l[1] * v[1] + F.l[2] * v[2] + F.l[3] * v[3];
    double s = eta - F.H * lu * lv;
    if (m.has_lambda) {
        const double wu = F.w[0] * u[0] + F.w[1] * u[1] + F.w[2] * u[2] + F.w[3] * u[3];
        const double wv = F.w[0] * v[0] + F.w[1] * v[1] + F.w[2] * v[2] + F.w[3] * v[3];
        s += F.sm * wu * wv;
    }
    return s;
}

// E/L_z/Carter-preserving constraint re-projection: p <- p + alpha dr with the
// root alpha of g^{-1}(p + a dr, p + a dr) = 0 of smallest magnitude — the
// chart-independent form of SymplecticIntegratorD::renormalizeNull's p_r
// solve (PHSI001A.h:366-418). Returns the null value before projection.
__device__ __forceinline__ double project_null(const MetricDev& m, const InvForm& F, double p[4]) {
    const double A = inv_apply(m, F, F.d, F.d);
    const double B = 2.0 * inv_apply(m, F, p, F.d);
    const double C = inv_apply(m, F, p, p);
    const double disc = B * B - 4.0 * A * C;
    if (disc < 0.0 || fabs(A) < 1e-15) return C;
    const double q = -0.5 * (B + (B >= 0.0 ? sqrt(disc) : -sqrt(disc)));
    if (q == 0.0) return C;
    const double alpha = C / q;
#pragma unroll
    for (int i = 0; i < 4; ++i) p[i] += alpha * F.d[i];
    return C;
}

// The same re-projection for the mixed-precision path, Kerr-Schild family
// without Lambda. Only the null value C = g^{-1}(p, p) needs FP64: it is a
// difference of O(p^2) terms that must survive to ~1e-16 of them, so r, H and
// l are FP64 (their three reciprocals from one division). The direction dr and
// the coefficients A = g^{-1}(dr, dr), B = 2 g^{-1}(p, dr) only set alpha =
// C / q, which needs single-precision relative accuracy; they are FP32, and
// the constraint left after the update is ~1e-7 C. Returns C; r_out = r.
__device__ __forceinline__ double project_null_ks_mixed(const MetricDev& m, const double x[4], double p[4],
                                                        double& r_out) {
    const double X = x[1], Y = x[2], Z = x[3];
    const double a = m.a, a2 = m.a2;
    const double R2 = X * X + Y * Y + Z * Z, Rm2 = R2 - a2;
    const double sd = sqrt(fmax(Rm2 * Rm2 + 4.0 * a2 * Z * Z, 1e-20));
    const double r2 = fmax(0.5 * (Rm2 + sd), 1e-10);
    const double r = sqrt(r2);
    r_out = r;
    const double den = r2 + a2, hden = r2 * r2 + a2 * Z * Z;
    const double t = 1.0 / (den * r * hden);
    const double iden = t * r * hden, ir = t * den * hden, ihden = t * den * r;
    const double l1 = (r * X + a * Y) * iden, l2 = (r * Y - a * X) * iden, l3 = Z * ir;
    const double H = (2.0 * m.M * r - m.Q2) * r2 * ihden;
    const double lp = -p[0] + l1 * p[1] + l2 * p[2] + l3 * p[3];
    const double C = -p[0] * p[0] + p[1] * p[1] + p[2] * p[2] + p[3] * p[3] - H * lp * lp;
    const float rf = float(r), isd = 1.f / float(sd);
    const float d1 = rf * float(X) * isd, d2 = rf * float(Y) * isd, d3 = float(Z) * float(den) * isd / rf;
    const float Hf = float(H);
    const float ld = float(l1) * d1 + float(l2) * d2 + float(l3) * d3;
    const float A = d1 * d1 + d2 * d2 + d3 * d3 - Hf * ld * ld;
    const float pd = float(p[1]) * d1 + float(p[2]) * d2 + float(p[3]) * d3;
    const float B = 2.f * (pd - Hf * float(lp) * ld);
    const float Cf = float(C);
    const float disc = B * B - 4.f * A * Cf;
    if (!(disc >= 0.f) || fabsf(A) < 1e-15f) return C;
    const float q = -0.5f * (B + copysignf(sqrtf(disc), B));
    if (q == 0.f) return C;
    const double alpha = double(Cf / q);
    p[1] += alpha * double(d1);
    p[2] += alpha * double(d2);
    p[3] += alpha * double(d3);
    return C;
}

// ---------------------------------------------------------------------------
// The metric alone, FP64, closed form (no derivatives): g[16].
// ---------------------------------------------------------------------------
__device__ __forceinline__ void metric_g(const MetricDev& m, const double x[4], double g[16]) {
    for (int i = 0; i < 16; ++i) g[i] = 0.0;
    if (m.family == SIRIUS_METRIC_MORRIS_THORNE) {
        const double r = fmax(x[1], m.b0 * 1.001);
        const double s = sin(x[2]);
        g[0] = m.gtt_mt;
        g[5] = mt_grr<double>(m, x[1]).v;
        g[10] = r * r;
        g[15] = r * r * s * s;
        return;
    }
    if (m.family == SIRIUS_METRIC_ALCUBIERRE) {
        const double vf = m.vs * alc_f<double>(m, x[1], x[2], x[3]).v;
        g[0] = -(1.0 - vf * vf);
        g[1] = g[4] = -vf;
        g[5] = g[10] = g[15] = 1.0;
        return;
    }
    InvForm F;
    inv_form(m, x, F);
    const double l[4] = {1.0, F.l[1], F.l[2], F.l[3]};  // covariant l
    for (int a = 0; a < 4; ++a)
        for (int b = 0; b < 4; ++b) g[4 * a + b] = ((a == b) ? (a == 0 ? -1.0 : 1.0) : 0.0) + F.H * l[a] * l[b];
    if (m.has_lambda) g[0] -= m.lam3 * (x[1] * x[1] + x[2] * x[2] + x[3] * x[3]);
}

// ---------------------------------------------------------------------------
// Full metric and derivatives (IMetric::evaluate): g[16], dg[64], dg[l*16+m*4+n].
// ---------------------------------------------------------------------------
template <class T>
__device__ void metric_full(const MetricDev& m, const T x[4], T g[16], T dg[64]) {
    for (int i = 0; i < 16; ++i) g[i] = T(0);
    for (int i = 0; i < 64; ++i) dg[i] = T(0);
    if (m.family == SIRIUS_METRIC_KERR_SCHILD) {
        KSPieces<T> P;
        ks_pieces(m, x[1], x[2], x[3], P);
        const D3<T> one = dconst(T(1));
        const D3<T> l[4] = {one, P.l1, P.l2, P.l3};
        for (int a = 0; a < 4; ++a)
            for (int b = 0; b < 4; ++b) {
                const D3<T> h = P.H * l[a] * l[b];
                const T eta = (a == b) ? (a == 0 ? T(-1) : T(1)) : T(0);
                g[4 * a + b] = eta + h.v;
                for (int q = 0; q < 3; ++q) dg[16 * (q + 1) + 4 * a + b] = h.d[q];
            }
        if (m.has_lambda) {
            g[0] -= T(m.lam3) * (x[1] * x[1] + x[2] * x[2] + x[3] * x[3]);
            for (int q = 0; q < 3; ++q) dg[16 * (q + 1)] -= T(2) * T(m.lam3) * x[q + 1];
        }
    } else if (m.family == SIRIUS_METRIC_MORRIS_THORNE) {
        const T r = tmax(x[1], T(m.b0) * T(1.001));
        const T s = sin(x[2]), c = cos(x[2]);
        const D3<T> grr = mt_grr(m, x[1]);
        g[0] = T(m.gtt_mt);
        g[5] = grr.v;
        g[10] = r * r;
        g[15] = r * r * s * s;
        dg[16 + 5] = grr.d[0];
        dg[16 + 10] = T(2) * r;
        dg[16 + 15] = T(2) * r * s * s;
        dg[32 + 15] = T(2) * r * r * s * c;
    } else {
        const D3<T> F = alc_f(m, x[1], x[2], x[3]);
        const T v = T(m.vs), vf = v * F.v;
        g[0] = -(T(1) - vf * vf);
        g[1] = g[4] = -vf;
        g[5] = g[10] = g[15] = T(1);
        for (int q = 0; q < 3; ++q) {
            dg[16 * (q + 1)] = T(2) * v * v * F.v * F.d[q];
            dg[16 * (q + 1) + 1] = dg[16 * (q + 1) + 4] = -v * F.d[q];
        }
    }
}

}  // namespace sirius

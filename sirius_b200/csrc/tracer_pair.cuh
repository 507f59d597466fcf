// tracer_pair.cuh — the mixed-precision Kerr-Schild tracer with two rays per
// thread, their FP32 arithmetic in packed pairs (sm_100 f32x2 instructions).
//
// Each thread owns two rays (neighbouring pixels, so their geodesics take the
// same branches). The DP45 attempt of both rays runs as one instruction stream
// in which every FP32 operation is a packed pair: lane .x is the first ray,
// lane .y the second (fma.rn.f32x2 and friends, one instruction for two rays).
// That halves the FP32 instructions per ray of the attempt, which is the bulk
// of the kernel (six right-hand sides and the stage algebra per step), and
// halves the instruction fetches per ray. Each packed operation is the same
// IEEE operation on each lane, so a ray's arithmetic does not depend on the
// ray it is paired with: a ray gives the same bits in any pairing, in a full
// frame, a row window or a compacted list.
//
// Everything after the attempt (accept/reject, FP64 projection, terminations,
// volumetric segment, disk crossings) runs per ray through advance_post, the
// same code the one-ray kernel runs; rays on the FP64 island take their attempt
// from island_attempt as there.
#pragma once

#include "tracer.cuh"

namespace sirius {
namespace eng {

// The metric constants of the two lanes (the rays of a pair may belong to
// different frames of a batch).
struct MetricPair {
    float2 a, a2, M2, Q2, lam3;
    bool any_lambda;
};

__device__ __forceinline__ MetricPair metric_pair(const MetricDev& m0, const MetricDev& m1) {
    MetricPair q;
    q.a = make_float2(float(m0.a), float(m1.a));
    q.a2 = make_float2(float(m0.a2), float(m1.a2));
    q.M2 = make_float2(float(2.0 * m0.M), float(2.0 * m1.M));
    q.Q2 = make_float2(float(m0.Q2), float(m1.Q2));
    q.lam3 = make_float2(m0.has_lambda ? float(m0.lam3) : 0.f, m1.has_lambda ? float(m1.lam3) : 0.f);
    q.any_lambda = m0.has_lambda || m1.has_lambda;
    return q;
}

// Hamilton's equations of the Kerr-Schild family for two states at once:
// k = g^{-1} p, f = 1/2 d g(k, k) (PHGD001A.cpp:159-202), from
// g = eta + H l l with r(x, y, z) the Kerr-Schild radius and the null covector
// l = (1, (r x + a y)/(r^2 + a^2), (r y - a x)/(r^2 + a^2), z/r). The gradients
// of r, l and H are written out by the chain rule (the forward-mode dual
// numbers of ks_pieces, expanded): dr = (r x, r y, z (r^2 + a^2)/r)/sqrt(disc),
//   d l1 = (d(r x + a y) - 2 r l1 dr/(r^2 + a^2)) / (r^2 + a^2), l2 likewise,
//   d l3 = (0, 0, 1)/r - z dr/r^2,
//   d H = ((dnum/dr - H dfden/dr) dr - H (0, 0, 2 a^2 z)) / fden,
// num = (2 M r - Q^2) r^2, fden = r^4 + a^2 z^2. The reference's Lambda term
// (-Lambda R^2/3 on g_tt, PHMT100A.h:362-369) enters by Sherman-Morrison.
// xs[1..3], ps[0..3] in; k[0..3], f[1..3] out (f_0 = 0: the metric is static).
__device__ __forceinline__ void ks_rhs_pair(const MetricPair& m, const float2 xs[4], const float2 ps[4], float2 k[4],
                                            float2 f[4]) {
    const float2 x = xs[1], y = xs[2], z = xs[3];
    const float2 zz = mul2(z, z);
    const float2 R2 = fma2(x, x, fma2(y, y, zz));
    const float2 Rm2 = sub2(R2, m.a2);
    const float2 a2zz = mul2(m.a2, zz);
    const float2 disc = max2(fma2(Rm2, Rm2, mul2(p2(4.f), a2zz)), 1e-20f);
    const float2 sd = sqrt2(disc);
    const float2 r2 = max2(mul2(add2(Rm2, sd), p2(0.5f)), 1e-10f);
    const float2 r = sqrt2(r2);
    const float2 isd = rcp2(sd), ir = rcp2(r);
    // dr
    const float2 risd = mul2(r, isd);
    const float2 den = add2(r2, m.a2);
    const float2 rx = mul2(risd, x), ry = mul2(risd, y), rz = mul2(mul2(z, den), mul2(isd, ir));
    // l1, l2 and their gradients
    const float2 iden = rcp2(den);
    const float2 gi = mul2(neg2(mul2(iden, iden)), add2(r, r));  // d(1/den)/dr = -2 r / den^2
    const float2 n1 = fma2(r, x, mul2(m.a, y)), n2 = fma2(r, y, neg2(mul2(m.a, x)));
    const float2 l1 = mul2(n1, iden), l2 = mul2(n2, iden);
    const float2 n1g = mul2(n1, gi), n2g = mul2(n2, gi);
    const float2 l1d0 = fma2(fma2(x, rx, r), iden, mul2(n1g, rx));
    const float2 l1d1 = fma2(fma2(x, ry, m.a), iden, mul2(n1g, ry));
    const float2 l1d2 = fma2(mul2(x, rz), iden, mul2(n1g, rz));
    const float2 l2d0 = fma2(fma2(y, rx, neg2(m.a)), iden, mul2(n2g, rx));
    const float2 l2d1 = fma2(fma2(y, ry, r), iden, mul2(n2g, ry));
    const float2 l2d2 = fma2(mul2(y, rz), iden, mul2(n2g, rz));
    // l3 = z / r and its gradient
    const float2 l3 = mul2(z, ir);
    const float2 zi2 = neg2(mul2(l3, ir));
    const float2 l3d0 = mul2(zi2, rx), l3d1 = mul2(zi2, ry), l3d2 = fma2(zi2, rz, ir);
    // H and its gradient
    const float2 q = fma2(m.M2, r, neg2(m.Q2));  // 2 M r - Q^2
    const float2 fden = fma2(r2, r2, a2zz);
    const float2 ifd = rcp2(fden);
    const float2 H = mul2(mul2(q, r2), ifd);
    const float2 dnum = fma2(m.M2, r2, mul2(add2(r, r), q));  // d num / dr = 2 M r^2 + 2 r q
    const float2 dfden = mul2(p2(4.f), mul2(r2, r));          // d fden / dr (through r)
    const float2 w = mul2(fma2(neg2(H), dfden, dnum), ifd);
    const float2 Hd0 = mul2(w, rx), Hd1 = mul2(w, ry);
    const float2 Hd2 = fma2(w, rz, neg2(mul2(mul2(H, ifd), mul2(add2(m.a2, m.a2), z))));
    // k = g^{-1} p = eta p - H l# (l# . p), l# = (-1, l1, l2, l3)
    const float2 lp = fma2(l3, ps[3], fma2(l2, ps[2], fma2(l1, ps[1], neg2(ps[0]))));
    const float2 Hlp = mul2(H, lp), nHlp = neg2(Hlp);
    k[0] = sub2(Hlp, ps[0]);
    k[1] = fma2(l1, nHlp, ps[1]);
    k[2] = fma2(l2, nHlp, ps[2]);
    k[3] = fma2(l3, nHlp, ps[3]);
    if (m.any_lambda) {
        // Sherman-Morrison for g_tt -= Lambda R^2 / 3 (lanes without Lambda keep k)
        const float2 c = mul2(m.lam3, R2);
        const float2 w0 = sub2(p2(-1.f), H), w1 = mul2(H, l1), w2 = mul2(H, l2), w3 = mul2(H, l3);
        const float2 wp = fma2(w3, ps[3], fma2(w2, ps[2], fma2(w1, ps[1], mul2(w0, ps[0]))));
        const float2 sm = mul2(mul2(c, wp), rcp2(fma2(c, add2(p2(1.f), H), p2(1.f))));
        const float2 k0 = fma2(sm, w0, k[0]), k1 = fma2(sm, w1, k[1]), k2 = fma2(sm, w2, k[2]),
                     k3 = fma2(sm, w3, k[3]);
        const bool lx = m.lam3.x != 0.f, ly = m.lam3.y != 0.f;
        k[0] = make_float2(lx ? k0.x : k[0].x, ly ? k0.y : k[0].y);
        k[1] = make_float2(lx ? k1.x : k[1].x, ly ? k1.y : k[1].y);
        k[2] = make_float2(lx ? k2.x : k[2].x, ly ? k2.y : k[2].y);
        k[3] = make_float2(lx ? k3.x : k[3].x, ly ? k3.y : k[3].y);
    }
    // dp = 1/2 dH (l.k)^2 + H (l.k)(dl.k)
    const float2 lk = fma2(l3, k[3], fma2(l2, k[2], fma2(l1, k[1], k[0])));
    const float2 hlk = mul2(p2(0.5f), lk);
    const float2 dlk0 = fma2(l3d0, k[3], fma2(l2d0, k[2], mul2(l1d0, k[1])));
    const float2 dlk1 = fma2(l3d1, k[3], fma2(l2d1, k[2], mul2(l1d1, k[1])));
    const float2 dlk2 = fma2(l3d2, k[3], fma2(l2d2, k[2], mul2(l1d2, k[1])));
    f[0] = p2(0.f);
    f[1] = mul2(lk, fma2(Hd0, hlk, mul2(H, dlk0)));
    f[2] = mul2(lk, fma2(Hd1, hlk, mul2(H, dlk1)));
    f[3] = mul2(lk, fma2(Hd2, hlk, mul2(H, dlk2)));
    if (m.any_lambda) {
        const float2 lq = neg2(mul2(m.lam3, mul2(k[0], k[0])));  // zero on lanes without Lambda
        const float2 f1 = fma2(lq, x, f[1]), f2 = fma2(lq, y, f[2]), f3 = fma2(lq, z, f[3]);
        const bool lx = m.lam3.x != 0.f, ly = m.lam3.y != 0.f;
        f[1] = make_float2(lx ? f1.x : f[1].x, ly ? f1.y : f[1].y);
        f[2] = make_float2(lx ? f2.x : f[2].x, ly ? f2.y : f[2].y);
        f[3] = make_float2(lx ? f3.x : f[3].x, ly ? f3.y : f[3].y);
    }
}


// The two rays' DP45 attempts (dp45_attempt<float> for a pair): stage inputs
// x + h acc in packed FP32 with acc = sum_j a_sj k_j in a sliding window, the
// fifth-order solution accumulated in FP64 per ray. The p_0 component is not
// carried: f_0 = 0 for the static metrics, so p_0 (the conserved -E) is exact.
// On entry k holds f(x, p) of each ray; on exit xn, pn the fifth-order
// solutions, k7 = f(xn, pn), err the scaled RMS errors of the positions.
__device__ __forceinline__ void dp45_attempt_pair(const MetricPair& m, const CfgDev& c, const Ray<true>& s0,
                                                  const Ray<true>& s1, double xn[2][4], double pn[2][4],
                                                  float k7[2][8], double err[2]) {
    const DPTablePair& D = kDPpair;
    const float2 ht = make_float2(float(s0.h), float(s1.h));
    float2 X[8], kc[8];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        X[i] = make_float2(float(s0.x[i]), float(s1.x[i]));
        X[4 + i] = make_float2(float(s0.p[i]), float(s1.p[i]));
    }
#pragma unroll
    for (int i = 0; i < 8; ++i) kc[i] = make_float2(s0.k[i], s1.k[i]);
    float2 acc[6][8], eacc[4];
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int s = 0; s < 6; ++s) acc[s][i] = p2(0.f);
#pragma unroll
    for (int i = 0; i < 4; ++i) eacc[i] = p2(0.f);
#pragma unroll 1
    for (int j = 0; j < 6; ++j) {
#pragma unroll
        for (int s = 0; s < 6; ++s) {
            const float2 a = D.A[j][s];
#pragma unroll
            for (int i = 0; i < 8; ++i)
                if (i != 4) acc[s][i] = fma2(a, kc[i], acc[s][i]);
        }
        const float2 e = D.E[j];
#pragma unroll
        for (int i = 0; i < 4; ++i) eacc[i] = fma2(e, kc[i], eacc[i]);
        float2 xs[4], ps[4];
        if (j == 5) {  // stage 7 is the solution point
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                xn[0][i] = s0.x[i] + s0.h * double(acc[0][i].x);
                xn[1][i] = s1.x[i] + s1.h * double(acc[0][i].y);
                pn[0][i] = i == 0 ? s0.p[0] : s0.p[i] + s0.h * double(acc[0][4 + i].x);
                pn[1][i] = i == 0 ? s1.p[0] : s1.p[i] + s1.h * double(acc[0][4 + i].y);
                xs[i] = make_float2(float(xn[0][i]), float(xn[1][i]));
                ps[i] = make_float2(float(pn[0][i]), float(pn[1][i]));
            }
        } else {
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                xs[i] = fma2(ht, acc[0][i], X[i]);
                ps[i] = i == 0 ? X[4] : fma2(ht, acc[0][4 + i], X[4 + i]);
            }
        }
        ks_rhs_pair(m, xs, ps, kc, kc + 4);
#pragma unroll
        for (int s = 0; s < 5; ++s)
#pragma unroll
            for (int i = 0; i < 8; ++i)
                if (i != 4) acc[s][i] = acc[s + 1][i];
#pragma unroll
        for (int i = 0; i < 8; ++i) acc[5][i] = p2(0.f);
    }
    float2 en = p2(0.f);
    const float2 atol = p2(float(c.atol)), rtol = p2(float(c.rtol));
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const float2 ex = fma2(D.E[6], kc[i], eacc[i]);
        const float2 ax = make_float2(fabsf(float(xn[0][i])), fabsf(float(xn[1][i])));
        const float2 e = mul2(mul2(ht, ex), rcp2(fma2(rtol, ax, atol)));
        en = fma2(e, e, en);
    }
    const float2 es = mul2(p2(0.25f), en);
    err[0] = double(sqrtf(es.x));
    err[1] = double(sqrtf(es.y));
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        k7[0][i] = kc[i].x;
        k7[1][i] = kc[i].y;
    }
}

// Two rays per thread: rays 2 g and 2 g + 1 of the launch (g the thread's
// global index), neighbouring pixels of one row. A lane whose ray has ended
// keeps computing on its last state inside the packed attempt (lane-wise
// arithmetic: its values never reach the live lane) until both have ended. One-thread-per-ray launch
// shape otherwise (no queue); the dynamic shared memory holds the volumetric
// accumulators of both rays, [ray][bin pair: I, then T][thread].
template <bool UNI>
__device__ __forceinline__ void trace_pair_body(const Params& P) {
    constexpr int KS = SIRIUS_METRIC_KERR_SCHILD;
    extern __shared__ float smem[];
    const int np = (P.c.enable_vol && P.c.nbins > 0) ? P.c.npair : 0;
    float2* smem2 = reinterpret_cast<float2*>(smem);
    float2* volq[2] = {np ? smem2 + threadIdx.x : nullptr, np ? smem2 + 2 * np * blockDim.x + threadIdx.x : nullptr};
    const int lane = threadIdx.x & 31;
    Ray<true> s[2];
    bool alive[2] = {false, false};
    float mag[2] = {1.f, 1.f};
    int flags[2] = {0, 0};
    unsigned long long acc = 0, rej0 = 0, f64 = 0;
    unsigned long long t_start = 0;
    if (lane == 0) {
        const unsigned long long now = globaltimer();
        const unsigned long long first = atomicCAS(P.clock0, 0ull, now);
        t_start = first ? first : now;
    }
    t_start = __shfl_sync(kFull, t_start, 0);
    const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        const long long li = 2 * gid + q;
        // a lane without a ray computes on a benign state (result unused)
        s[q].frame = 0;
        s[q].h = 1.0;
        s[q].crit = 0;
#pragma unroll
        for (int i = 0; i < 4; ++i) { s[q].x[i] = i == 1 ? 10.0 : 0.0; s[q].p[i] = i == 0 ? -1.0 : (i == 1 ? 1.0 : 0.0); }
#pragma unroll
        for (int i = 0; i < 8; ++i) s[q].k[i] = 0.f;
        const unsigned entry = (P.list && li < P.total) ? P.list[li] : 0u;
        if (li < P.total && entry != kListSkip) {
            const long long idx = P.list ? (long long)entry : li;
            const int frame = P.n_frames > 1 ? find_frame(P.frames, P.n_frames, idx) : 0;
            if (P.family < 0 || P.frames[frame].m.family == P.family) {
                begin_ray<true, KS, UNI>(P, s[q], idx, frame, volq[q]);
                alive[q] = true;
            }
        }
    }
    for (unsigned iter = 0;; ++iter) {
        if ((iter & 255u) == 0) {
            int stop = 0;
            if (lane == 0) {
                if (globaltimer() - t_start > P.watchdog_ns) atomicOr(P.status, 1);
                stop = *((volatile int*)P.status) & 1;
            }
            stop = __shfl_sync(kFull, stop, 0);
            if (stop) {
#pragma unroll
                for (int q = 0; q < 2; ++q)
                    if (alive[q]) {
                        end_ray<true, UNI>(P, s[q], SIRIUS_MAX_STEPS, mag[q], flags[q], volq[q]);
                        alive[q] = false;
                    }
            }
        }
        if (__ballot_sync(kFull, alive[0] || alive[1]) == 0) break;
        if (!(alive[0] || alive[1])) continue;
        const FrameDev& F0 = frame_of<UNI>(P, s[0].frame);
        const FrameDev& F1 = frame_of<UNI>(P, s[1].frame);
        bool island[2];
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            const FrameDev& F = q ? F1 : F0;
            const double R2 = s[q].x[1] * s[q].x[1] + s[q].x[2] * s[q].x[2] + s[q].x[3] * s[q].x[3];
            island[q] = alive[q] && (s[q].crit || R2 < F.island_r * F.island_r);
        }
        double xn[2][4], pn[2][4], err[2];
        float k7[2][8];
        if ((alive[0] && !island[0]) || (alive[1] && !island[1])) {
            const MetricPair mp = UNI ? metric_pair(P.f0.m, P.f0.m) : metric_pair(F0.m, F1.m);
            dp45_attempt_pair(mp, P.c, s[0], s[1], xn, pn, k7, err);
        }
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            if (!alive[q]) continue;
            Ray<true>& r = s[q];
            if (island[q]) {
                const FrameDev& F = frame_of<UNI>(P, r.frame);
                const IslandStep o = island_attempt<KS>(F.m, P.c, vec4v(r.x), vec4v(r.p), r.h);
#pragma unroll
                for (int i = 0; i < 4; ++i) { xn[q][i] = o.xn[i]; pn[q][i] = o.pn[i]; }
#pragma unroll
                for (int i = 0; i < 8; ++i) k7[q][i] = o.k7[i];
                err[q] = o.err;
            }
            const int out = advance_post<true, KS, UNI, SIRIUS_INTEGRATOR_DP45>(P, r, island[q], xn[q], pn[q], k7[q], err[q], mag[q], flags[q],
                                                        volq[q]);
            if (out >= 0) {
                end_ray<true, UNI>(P, r, out, mag[q], flags[q], volq[q]);
                acc += r.steps;
                rej0 += r.rejected;
                f64 += r.fp64_steps;
                alive[q] = false;
            }
        }
    }
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

template <int MINB, bool UNI>
__global__ void __launch_bounds__(128, MINB) trace_pair_kernel(const __grid_constant__ Params P) {
    trace_pair_body<UNI>(P);
}

}  // namespace eng
}  // namespace sirius

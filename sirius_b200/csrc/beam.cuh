// beam.cuh — the beam of neighbouring rays around a pixel ray (geodesic
// deviation), and the magnification it gives.
//
// The reference's BeamIntegratorD (INBI001A.h:178-363) carries a Jacobian J of
// Boyer-Lindquist coordinates along a leapfrog ray with a Jacobi equation in
// the Riemann tensor, and reports 1 / |det| of J's (theta, phi) block. Here the
// same idea is restated on the engine's Hamiltonian form: the ray y = (x^mu,
// p_mu) carries two tangent vectors V_u = dy/du, V_v = dy/dv (u, v: the pixel
// coordinates of its start), which obey the linearised equation
//   dV/dlambda = (df/dy) V,   f = (dx/dlambda, dp/dlambda)
// (the geodesic deviation equation in first-order form). df/dy V is a central
// difference of the right-hand side along V; the ray and its tangents advance
// together by Dormand-Prince 5(4) steps controlled on the ray. When the ray
// escapes, its unit direction n and the tangents' dn/du, dn/dv give the solid
// angle the pixel maps to on the sky, |dn/du x dn/dv| du dv; the pixel's own
// solid angle is |dd/du x dd/dv| du dv with d the start direction in the
// camera frame; the magnification is their ratio (1 in flat space) and the
// parity is the sign of the map (negative for a mirror-reversed image).
//
// This file is a fragment of engine.cu's kernel section (it uses the engine's
// find_frame and globaltimer) and is included there.
#pragma once

// start direction of pixel position (u, v) (pixel units, the centre of pixel
// (px, py) is (px + 0.5, py + 0.5)) in FP64 without the camera's FP32
// roundings, so that its derivatives are smooth
__device__ __forceinline__ void camera_dir_exact(const FrameDev& F, double u, double v, double dir[4]) {
    dir[0] = 0.0;
    if (F.projection == SIRIUS_CAMERA_EQUIRECTANGULAR) {
        const double psi = (2.0 * u / F.width - 1.0) * kPi;
        const double chi = (1.0 - 2.0 * v / F.height) * (0.5 * kPi);
        double sc, cc, sps, cps;
        sincos(chi, &sc, &cc);
        sincos(psi, &sps, &cps);
        dir[1] = -cc * cps;
        dir[2] = -sc;
        dir[3] = cc * sps;
        return;
    }
    const double pxn = (2.0 * u / F.width - 1.0) * double(F.aspect), pyn = 1.0 - 2.0 * v / F.height;
    const double T = F.tan_half_fov;
    const double dx = pxn * T, dy = pyn * T, dz = -1.0;
    const double cR = F.cR, sR = F.sR, cP = F.cP, sP = F.sP, cY = F.cY, sY = F.sY;
    const double rx = dx * cR - dy * sR, ry = dx * sR + dy * cR;
    const double ry2 = ry * cP - dz * sP, rz = ry * sP + dz * cP;
    const double rx2 = rx * cY + rz * sY, rz2 = -rx * sY + rz * cY;
    const double len = sqrt(rx2 * rx2 + ry2 * ry2 + rz2 * rz2);
    dir[1] = rz2 / len;
    dir[2] = -ry2 / len;
    dir[3] = rx2 / len;
}

__device__ __forceinline__ void beam_start(const FrameDev& F, double u, double v, double y[8]) {
    double dir[4];
    camera_dir_exact(F, u, v, dir);
    init_state(F, dir, y, y + 4);
}

__device__ __forceinline__ void beam_f(const MetricDev& m, const double y[8], double f[8]) {
    rhs<double, kAnyFamily>(m, y, y + 4, f, f + 4);
}

// f(y) and (df/dy) V for both tangents
__device__ __forceinline__ void beam_rhs(const MetricDev& m, const double Y[24], double FY[24]) {
    beam_f(m, Y, FY);
    double ysc = 1.0;
    for (int i = 0; i < 8; ++i) ysc = fmax(ysc, fabs(Y[i]));
#pragma unroll 1
    for (int t = 0; t < 2; ++t) {
        const double* V = Y + 8 + 8 * t;
        double vn = 0.0;
        for (int i = 0; i < 8; ++i) vn = fmax(vn, fabs(V[i]));
        double* out = FY + 8 + 8 * t;
        if (!(vn > 0.0)) {
            for (int i = 0; i < 8; ++i) out[i] = 0.0;
            continue;
        }
        const double eps = 1e-6 * ysc / vn;
        double yp[8], ym[8], fp[8], fm[8];
        for (int i = 0; i < 8; ++i) {
            yp[i] = Y[i] + eps * V[i];
            ym[i] = Y[i] - eps * V[i];
        }
        beam_f(m, yp, fp);
        beam_f(m, ym, fm);
        for (int i = 0; i < 8; ++i) out[i] = (fp[i] - fm[i]) / (2.0 * eps);
    }
}

__device__ __forceinline__ void cross3(const double a[3], const double b[3], double c[3]) {
    c[0] = a[1] * b[2] - a[2] * b[1];
    c[1] = a[2] * b[0] - a[0] * b[2];
    c[2] = a[0] * b[1] - a[1] * b[0];
}

struct BeamParams {
    const FrameDev* frames;
    int n_frames;
    long long total;
    CfgDev c;
    sirius_beam_result* out;
    unsigned long long watchdog_ns;
    int* status;
};

__global__ void __launch_bounds__(64) beam_kernel(const __grid_constant__ BeamParams B) {
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= B.total) return;
    const int fi = B.n_frames > 1 ? find_frame(B.frames, B.n_frames, idx) : 0;
    const FrameDev& F = B.frames[fi];
    const CfgDev& c = B.c;
    const MetricDev& m = F.m;
    const long long pix = idx - F.ray_offset;
    const double u0 = double(pix % F.width) + 0.5, v0 = double(F.row0 + pix / F.width) + 0.5;
    // start: the ray, its tangents along u and v, and the pixel's solid angle
    double Y[24];
    beam_start(F, u0, v0, Y);
    const double hpx = 1e-3;
    double dd[2][3];
    for (int t = 0; t < 2; ++t) {
        double yp[8], ym[8], dp[4], dm[4];
        const double du = t == 0 ? hpx : 0.0, dv = t == 0 ? 0.0 : hpx;
        beam_start(F, u0 + du, v0 + dv, yp);
        beam_start(F, u0 - du, v0 - dv, ym);
        for (int i = 0; i < 8; ++i) Y[8 + 8 * t + i] = (yp[i] - ym[i]) / (2.0 * hpx);
        camera_dir_exact(F, u0 + du, v0 + dv, dp);
        camera_dir_exact(F, u0 - du, v0 - dv, dm);
        for (int i = 0; i < 3; ++i) dd[t][i] = (dp[1 + i] - dm[1 + i]) / (2.0 * hpx);
    }
    double d0[4], cimg[3];
    camera_dir_exact(F, u0, v0, d0);
    cross3(dd[0], dd[1], cimg);
    const double omega_img = sqrt(cimg[0] * cimg[0] + cimg[1] * cimg[1] + cimg[2] * cimg[2]);
    const double sgn_img = cimg[0] * d0[1] + cimg[1] * d0[2] + cimg[2] * d0[3] >= 0.0 ? 1.0 : -1.0;

    const DPTable<double>& D = dp_table<double>();
    double h = c.h0;
    double K[7][24];
    beam_rhs(m, Y, K[0]);
    int outcome = SIRIUS_MAX_STEPS, steps = 0;
    const unsigned long long t0 = globaltimer();
    double r_prev = ks_radius(m, Y);
    for (int it = 0; it < 4 * c.max_steps && steps < c.max_steps; ++it) {
        if ((it & 63) == 0 && globaltimer() - t0 > B.watchdog_ns) {
            atomicOr(B.status, 1);
            break;
        }
        // Dormand-Prince 5(4) on the 24 components (the stages' weights from the shared table)
        double Ys[24];
        for (int s = 1; s <= 6; ++s) {
            for (int i = 0; i < 24; ++i) {
                double acc = 0.0;
                for (int j = 0; j < s; ++j) acc += D.A[j][s - 1 - j] * K[j][i];
                Ys[i] = Y[i] + h * acc;
            }
            beam_rhs(m, Ys, K[s]);
        }
        // Ys is the fifth-order solution (stage 7 = b weights); error on the position components
        double err2 = 0.0;
        for (int i = 0; i < 4; ++i) {
            double e = 0.0;
            for (int j = 0; j < 7; ++j) e += D.E[j] * K[j][i];
            e *= h;
            const double sc = c.atol + c.rtol * fmax(fabs(Y[i]), fabs(Ys[i]));
            err2 += (e / sc) * (e / sc);
        }
        const double err = sqrt(err2 / 4.0);
        if (!(err == err)) {
            outcome = SIRIUS_NUMERICAL_FAILURE;
            break;
        }
        if (err > 1.0 && h > c.hmin) {
            h = fmax(c.hmin, optimal_step(h, err, c));
            continue;
        }
        const double z0 = Y[3];
        for (int i = 0; i < 24; ++i) Y[i] = Ys[i];
        for (int i = 0; i < 24; ++i) K[0][i] = K[6][i];
        ++steps;
        h = optimal_step(h, err, c);
        const double r = ks_radius(m, Y);
        if (F.has_horizon && r < F.r_hor) {
            outcome = SIRIUS_HORIZON;
            break;
        }
        if (c.enable_disk && z0 * Y[3] < 0.0) {
            const double rc = 0.5 * (r + r_prev);
            if (rc >= F.disk_in && rc <= F.disk_out) {
                outcome = SIRIUS_DISK_HIT;
                break;
            }
        }
        r_prev = r;
        const double R2 = Y[1] * Y[1] + Y[2] * Y[2] + Y[3] * Y[3];
        const double out = Y[1] * K[0][1] + Y[2] * K[0][2] + Y[3] * K[0][3];
        if (R2 > c.escape_r * c.escape_r && out > 0.0) {
            outcome = SIRIUS_ESCAPED;
            break;
        }
    }
    sirius_beam_result res{};
    res.outcome = outcome;
    res.steps = steps;
    if (outcome == SIRIUS_ESCAPED) {
        // n = k / |k| (spatial, contravariant), dn = (dk - n (n . dk)) / |k| along each tangent
        double k[8];
        beam_f(m, Y, k);
        const double kn = sqrt(k[1] * k[1] + k[2] * k[2] + k[3] * k[3]);
        double n[3] = {k[1] / kn, k[2] / kn, k[3] / kn}, dn[2][3];
        double ysc = 1.0;
        for (int i = 0; i < 8; ++i) ysc = fmax(ysc, fabs(Y[i]));
        for (int t = 0; t < 2; ++t) {
            const double* V = Y + 8 + 8 * t;
            double vn = 0.0;
            for (int i = 0; i < 8; ++i) vn = fmax(vn, fabs(V[i]));
            const double eps = vn > 0.0 ? 1e-6 * ysc / vn : 0.0;
            double yp[8], ym[8], fp[8], fm[8];
            for (int i = 0; i < 8; ++i) {
                yp[i] = Y[i] + eps * V[i];
                ym[i] = Y[i] - eps * V[i];
            }
            beam_f(m, yp, fp);
            beam_f(m, ym, fm);
            double dk[3];
            for (int i = 0; i < 3; ++i) dk[i] = eps > 0.0 ? (fp[1 + i] - fm[1 + i]) / (2.0 * eps) : 0.0;
            const double nd = n[0] * dk[0] + n[1] * dk[1] + n[2] * dk[2];
            for (int i = 0; i < 3; ++i) dn[t][i] = (dk[i] - n[i] * nd) / kn;
        }
        double cs[3];
        cross3(dn[0], dn[1], cs);
        const double omega_src = sqrt(cs[0] * cs[0] + cs[1] * cs[1] + cs[2] * cs[2]);
        const double sgn_src = cs[0] * n[0] + cs[1] * n[1] + cs[2] * n[2] >= 0.0 ? 1.0 : -1.0;
        res.magnification = omega_src > 0.0 ? float(omega_img / omega_src) : 1e30f;
        res.parity = float(sgn_img * sgn_src);
        for (int i = 0; i < 3; ++i) res.final_dir[i] = float(n[i]);
    }
    B.out[idx] = res;
}

// sirius_b200.hpp — C++17 host layer over the C ABI (sirius_cuda.h).
//
// Mirrors the reference's own host interfaces for the geodesic path so that
// C++ callers keep their types and call patterns:
//   KerrSchildFamily   parameters / getParameters / setParameter / getName
//                      (src/Sirius.Core/Metric/PHMT100A.h:149-196)
//   IntegratorConfig   (src/Sirius.Core/Geodesic/PHGD001A.h:48-58)
//   TracerConfig       (src/Sirius.Render/Integration/GTRC001A.h:162-196)
//   CameraRay          (src/Sirius.Core/Camera/CMBS001A.h:26-32)
//   TraceResult        (src/Sirius.Render/Integration/GTRC001A.h:44-157)
//   CudaGeodesicTracer the GeodesicTracer contract: trace(CameraRay) ->
//                      TraceResult, trace(ray, M, a), plus a batch overload
//                      (GTRC001A.h:201-350)
//   IAccelerator, LaunchConfig, BackendType, createAccelerator
//                      (src/Sirius.Render/Acceleration/Backend/ACIB001A.h:24-200,
//                      ACBF001A.cpp:16-53): CudaAccelerator fills the reserved
//                      BackendType::CUDA slot.
// Header-only; link libsirius_b200.so. Errors are reported as the reference
// reports them: bool returns and getLastError(); no exception crosses the C ABI.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "sirius_cuda.h"

namespace sirius_b200 {

// ---------------------------------------------------------------- metric ---
struct MetricParameter {
    double value, min, max;
};
using Config = std::map<std::string, MetricParameter>;

struct KerrSchildParams {
    double M = 1.0, a = 0.0, Q = 0.0, Lambda = 0.0;
};

/// Parameter holder with the reference's keys, ranges and clamping
/// ("mass", "spin" = a/M, "charge" = Q/M, "lambda"); produces the C metric.
class KerrSchildFamily {
public:
    KerrSchildFamily() {
        m_Config["mass"] = {1.0, 0.0, 100.0};
        m_Config["spin"] = {0.0, -0.998, 0.998};
        m_Config["charge"] = {0.0, -1.0, 1.0};
        m_Config["lambda"] = {0.0, -0.1, 0.1};
    }
    explicit KerrSchildFamily(const KerrSchildParams& p) : KerrSchildFamily() { setParams(p); }
    void setParams(const KerrSchildParams& p) {
        m_Params = p;
        m_Config["mass"].value = p.M;
        m_Config["spin"].value = p.a / std::max(p.M, 1e-10);
        m_Config["charge"].value = p.Q / std::max(p.M, 1e-10);
        m_Config["lambda"].value = p.Lambda;
    }
    KerrSchildParams getParams() const { return m_Params; }
    const Config& getParameters() const { return m_Config; }
    void setParameter(const std::string& key, double value) {
        auto it = m_Config.find(key);
        if (it != m_Config.end()) it->second.value = std::clamp(value, it->second.min, it->second.max);
        m_Params.M = m_Config["mass"].value;
        m_Params.a = m_Config["spin"].value * m_Params.M;
        m_Params.Q = m_Config["charge"].value * m_Params.M;
        m_Params.Lambda = m_Config["lambda"].value;
    }
    const char* getName() const {
        const auto& p = m_Params;
        if (p.M == 0 && p.Lambda == 0) return "Minkowski";
        if (p.a == 0 && p.Q == 0 && p.Lambda == 0) return "Schwarzschild";
        if (p.Q == 0 && p.Lambda == 0) return "Kerr";
        if (p.a == 0 && p.Lambda == 0) return "Reissner-Nordstr\xc3\xb6m";
        if (p.Lambda == 0) return "Kerr-Newman";
        if (p.M == 0) return "de Sitter";
        if (p.a == 0 && p.Q == 0) return "Schwarzschild-de Sitter";
        if (p.Q == 0) return "Kerr-de Sitter";
        return "Kerr-Newman-de Sitter";
    }
    sirius_metric toMetric() const {
        sirius_metric m{};
        m.family = SIRIUS_METRIC_KERR_SCHILD;
        m.M = m_Params.M; m.a = m_Params.a; m.Q = m_Params.Q; m.Lambda = m_Params.Lambda;
        m.b0 = 1.0; m.sigma = 8.0; m.R = 1.0;
        return m;
    }

private:
    Config m_Config;
    KerrSchildParams m_Params{1.0, 0.0, 0.0, 0.0};
};

// --------------------------------------------------------- tracer types ---
struct Vec4 {
    double v[4] = {0, 0, 0, 0};
    double& operator()(int i) { return v[i]; }
    double operator()(int i) const { return v[i]; }
};

struct CameraRay {
    Vec4 origin;     ///< (t, r, theta, phi) Boyer-Lindquist
    Vec4 direction;  ///< (0, v_r, r v_theta, r sin(theta) v_phi)
    float weight = 1.0f;
};

struct IntegratorConfig {
    float abs_tolerance = 1e-6f, rel_tolerance = 1e-6f, min_step = 1e-6f, max_step = 0.1f, initial_step = 0.01f;
    float safety_factor = 0.9f, step_grow_max = 2.0f, step_shrink_min = 0.1f;
    bool use_rk45 = true;
};

struct TracerConfig {
    float escape_radius = 100.0f;
    float horizon_factor = 1.05f;
    int max_steps = 5000;
    bool enable_disk = true;
    float disk_inner = 6.0f, disk_outer = 20.0f, disk_thickness = 0.01f, disk_temperature_inner = 1.0f;
    bool enable_volumetric = false;
    IntegratorConfig integrator;
    // engine knobs (not in the reference): precision and the FP64 projection period
    int precision = SIRIUS_PRECISION_FP64;
    int projection_period = 1;
};

struct TraceResult {
    enum class Outcome { ESCAPED, HORIZON, DISK_HIT, MAX_STEPS, SPIRALING };
    Outcome outcome = Outcome::MAX_STEPS;
    Vec4 final_position, final_direction;
    float disk_radius = 0.0f, disk_temperature = 0.0f, disk_phi = 0.0f;
    int steps_taken = 0;
    float redshift = 1.0f;
    bool numerical_failure = false;
    float magnification = 1.0f, min_radius = 1e10f;
    bool photon_ring = false;
    int equatorial_crossings = 0;
    float total_phi_change = 0.0f;
    int image_order = 0;
    float impact_parameter = 0.0f;
    static constexpr int MAX_DISK_CROSSINGS = 4;
    struct DiskCrossing {
        float r = 0.0f, phi = 0.0f, temperature = 0.0f, redshift = 1.0f;
        int crossing_index = 0;
        bool valid = false;
    };
    DiskCrossing disk_crossings[MAX_DISK_CROSSINGS] = {};
    int num_disk_crossings = 0;
    float optical_depth = 0.0f;
    // engine extras
    int engine_outcome = SIRIUS_MAX_STEPS;  ///< enum sirius_outcome (splits MAX_STEPS by cause)
    float intensity = 0.0f;                 ///< bolometric intensity sum_n e^{-pi n} g_n^4 F(r_n)
    float null_final = 0.0f;                ///< |g^{mu nu} p_mu p_nu| of the returned state
};

inline sirius_trace_config toEngineConfig(const TracerConfig& t) {
    sirius_trace_config c{};
    sirius_cuda_default_config(&c);
    c.abs_tolerance = t.integrator.abs_tolerance;
    c.rel_tolerance = t.integrator.rel_tolerance;
    c.min_step = t.integrator.min_step;
    c.max_step = t.integrator.max_step;
    c.initial_step = t.integrator.initial_step;
    c.safety_factor = t.integrator.safety_factor;
    c.step_grow_max = t.integrator.step_grow_max;
    c.step_shrink_min = t.integrator.step_shrink_min;
    c.escape_radius = t.escape_radius;
    c.horizon_factor = t.horizon_factor;
    c.max_steps = t.max_steps;
    c.enable_disk = t.enable_disk ? 1 : 0;
    c.disk_temperature_inner = t.disk_temperature_inner;
    c.enable_volumetric = t.enable_volumetric ? 1 : 0;
    c.n_bins = t.enable_volumetric ? 1 : 0;
    c.precision = t.precision;
    c.projection_period = t.projection_period;
    return c;
}

/// sirius_ray_result -> TraceResult (GTRC001A.h:44-157 field meanings).
inline TraceResult toTraceResult(const sirius_ray_result& r, const TracerConfig& cfg) {
    TraceResult o;
    o.engine_outcome = r.outcome;
    switch (r.outcome) {
        case SIRIUS_ESCAPED: o.outcome = TraceResult::Outcome::ESCAPED; break;
        case SIRIUS_HORIZON: o.outcome = TraceResult::Outcome::HORIZON; break;
        case SIRIUS_DISK_HIT: o.outcome = TraceResult::Outcome::DISK_HIT; break;
        case SIRIUS_SPIRALING: o.outcome = TraceResult::Outcome::SPIRALING; break;
        default: o.outcome = TraceResult::Outcome::MAX_STEPS; break;
    }
    for (int i = 0; i < 4; ++i) {
        o.final_position.v[i] = r.final_x[i];
        o.final_direction.v[i] = r.final_k[i];
    }
    o.numerical_failure = (r.flags & SIRIUS_FLAG_NUMERICAL_FAILURE) != 0;
    o.photon_ring = (r.flags & SIRIUS_FLAG_PHOTON_RING) != 0;
    o.steps_taken = r.steps;
    o.magnification = r.magnification;
    o.min_radius = r.min_radius;
    o.equatorial_crossings = r.equatorial_crossings;
    o.total_phi_change = r.total_phi_change;
    o.image_order = r.image_order;
    o.impact_parameter = r.impact_parameter;
    o.num_disk_crossings = r.n_crossings;
    auto temperature = [&](float rad) {  // computeDiskTemperature, GTRC001A.h:382-394
        return rad > 0 ? cfg.disk_temperature_inner * std::pow(cfg.disk_inner / rad, 0.75f) : 0.0f;
    };
    for (int i = 0; i < r.n_crossings && i < TraceResult::MAX_DISK_CROSSINGS; ++i) {
        auto& c = o.disk_crossings[i];
        c.r = r.disk_r[i];
        c.phi = r.disk_phi[i];
        c.redshift = r.disk_g[i];
        c.temperature = temperature(c.r);
        c.crossing_index = i;
        c.valid = true;
    }
    if (r.n_crossings > 0) {
        o.disk_radius = r.disk_r[0];
        o.disk_phi = r.disk_phi[0];
        o.redshift = r.disk_g[0];
        o.disk_temperature = temperature(o.disk_radius);
    }
    o.optical_depth = r.optical_depth;
    o.intensity = r.intensity;
    o.null_final = r.null_final;
    return o;
}

/// The GeodesicTracer contract on the GPU. One tracer per host thread; the
/// metric is borrowed and must outlive the tracer (GTRC001A.h:203-206).
class CudaGeodesicTracer {
public:
    CudaGeodesicTracer(KerrSchildFamily* metric, const TracerConfig& config, int device = 0)
        : m_Metric(metric), m_Config(config) {
        m_Status = sirius_cuda_create(device, &m_Handle);
    }
    ~CudaGeodesicTracer() {
        if (m_Handle) sirius_cuda_destroy(m_Handle);
    }
    CudaGeodesicTracer(const CudaGeodesicTracer&) = delete;
    CudaGeodesicTracer& operator=(const CudaGeodesicTracer&) = delete;

    bool ok() const { return m_Status == SIRIUS_OK && m_Handle != nullptr; }
    std::string getLastError() const {
        if (!m_Handle) return "no CUDA device available (status " + std::to_string(m_Status) + ")";
        return sirius_cuda_get_last_error(m_Handle);
    }

    TraceResult trace(const CameraRay& ray) {
        std::vector<TraceResult> out = traceBatch(std::vector<CameraRay>{ray});
        return out.empty() ? TraceResult{} : out[0];
    }
    /// trace(ray, M, a): updates the metric's mass and spin and the disk inner
    /// edge to the prograde ISCO (GTRC001A.cpp:597-640).
    TraceResult trace(const CameraRay& ray, double mass, double spin) {
        m_Metric->setParameter("mass", mass);
        m_Metric->setParameter("spin", spin / mass);
        const double a = std::clamp(spin / mass, -1.0, 1.0), aa = std::fabs(a);
        const double Z1 = 1 + std::cbrt(1 - a * a) * (std::cbrt(1 + aa) + std::cbrt(1 - aa));
        const double Z2 = std::sqrt(3 * a * a + Z1 * Z1);
        const double risco = std::fabs(spin) < 1e-10 ? 6.0 : (a >= 0 ? 3 + Z2 - std::sqrt((3 - Z1) * (3 + Z1 + 2 * Z2))
                                                                    : 3 + Z2 + std::sqrt((3 - Z1) * (3 + Z1 + 2 * Z2)));
        m_Config.disk_inner = static_cast<float>(risco * mass);
        return trace(ray);
    }
    /// Batch form: all rays share the camera origin of the first (one frame).
    std::vector<TraceResult> traceBatch(const std::vector<CameraRay>& rays) {
        std::vector<TraceResult> out;
        if (!ok() || rays.empty()) return out;
        sirius_trace_config c = toEngineConfig(m_Config);
        if (sirius_cuda_configure(m_Handle, &c) != SIRIUS_OK) return out;
        std::vector<sirius_camera_ray> in(rays.size());
        for (size_t i = 0; i < rays.size(); ++i)
            for (int j = 0; j < 4; ++j) {
                in[i].origin[j] = rays[i].origin(j);
                in[i].direction[j] = rays[i].direction(j);
            }
        std::vector<sirius_ray_result> res(rays.size());
        const sirius_metric m = m_Metric->toMetric();
        if (sirius_cuda_trace_rays(m_Handle, &m, m_Config.disk_inner, m_Config.disk_outer, in.data(),
                                   static_cast<int64_t>(in.size()), res.data()) != SIRIUS_OK)
            return out;
        out.reserve(res.size());
        for (const auto& r : res) out.push_back(toTraceResult(r, m_Config));
        return out;
    }
    void setConfig(const TracerConfig& c) { m_Config = c; }
    const TracerConfig& getConfig() const { return m_Config; }
    void setMetric(KerrSchildFamily* m) { m_Metric = m; }

private:
    KerrSchildFamily* m_Metric;
    TracerConfig m_Config;
    sirius_cuda_handle m_Handle = nullptr;
    int m_Status = SIRIUS_ERR_NO_DEVICE;
};

// ------------------------------------------------------------ accelerator --
enum class BackendType : uint8_t { None, OptiX, CUDA, HIP, OneAPI, Metal, CPU };

struct DeviceCapabilities {
    std::string deviceName;
    size_t totalMemory = 0, freeMemory = 0;
    int computeCapability = 0;
    bool supportsRTCores = false, supportsFP64 = false;
    int multiprocessorCount = 0, maxThreadsPerBlock = 0;
};

/// The LaunchConfig fields the geodesic path reads (ACIB001A.h:64-143).
struct LaunchConfig {
    int width = 1920, height = 1080, samplesPerPixel = 64, tileSize = 64;
    float blackHoleMass = 1.0f, blackHoleSpin = 0.0f, observerDistance = 100.0f, observerInclination = 1.5708f,
          observerAzimuth = 0.0f, cameraFOV = 45.0f;
    float diskInnerRadius = 6.0f, diskOuterRadius = 30.0f, diskTemperature = 50000.0f, diskEmission = 2.5f;
    int temperatureModel = 1;
    float maxStepSize = 0.5f;
    int maxSteps = 10000;
    int metricType = 2, metricFamily = 0;
    float throatRadius = 1.0f, warpVelocity = 0.5f, bubbleRadius = 1.0f, bubbleSigma = 0.5f;
    float exposure = 0.5f;
};

class IAccelerator {
public:
    virtual ~IAccelerator() = default;
    virtual BackendType getType() const = 0;
    virtual DeviceCapabilities getCapabilities() const = 0;
    virtual bool initialise(int width, int height) = 0;
    virtual bool isInitialised() const = 0;
    virtual void launch(const LaunchConfig& config) = 0;
    virtual float* getFrameBuffer() = 0;  ///< RGBA float; the caller does NOT own it
    virtual size_t getFrameBufferSize() const = 0;
    virtual bool uploadBackground(const uint8_t* data, int width, int height) = 0;
    virtual void synchronise() = 0;
    virtual void cleanup() = 0;
    virtual std::string getLastError() const = 0;
    virtual void resetAccumulation() {}
};

/// BackendType::CUDA. The framebuffer holds the bolometric intensity times the
/// exposure in R, G and B (linear, no tone map) and 1 in A.
class CudaAccelerator : public IAccelerator {
public:
    explicit CudaAccelerator(int device = 0) : m_Device(device) {}
    ~CudaAccelerator() override { cleanup(); }
    BackendType getType() const override { return BackendType::CUDA; }
    DeviceCapabilities getCapabilities() const override {
        DeviceCapabilities d;
        d.deviceName = "NVIDIA B200 (sm_100a)";
        d.computeCapability = 100;
        d.supportsFP64 = true;
        return d;
    }
    bool initialise(int width, int height) override {
        if (width <= 0 || height <= 0) { m_LastError = "invalid framebuffer size"; return false; }
        if (!m_Handle) {
            const int rc = sirius_cuda_create(m_Device, &m_Handle);
            if (rc != SIRIUS_OK) { m_LastError = "sirius_cuda_create failed: " + std::to_string(rc); return false; }
        }
        m_Width = width;
        m_Height = height;
        m_Frame.assign(size_t(width) * height * 4, 0.0f);
        m_Image.assign(size_t(width) * height, 0.0f);
        return true;
    }
    bool isInitialised() const override { return m_Handle != nullptr; }
    void launch(const LaunchConfig& lc) override {
        if (!m_Handle) { m_LastError = "not initialised"; return; }
        sirius_trace_config c{};
        sirius_cuda_default_config(&c);
        c.max_steps = lc.maxSteps;
        c.max_step = lc.maxStepSize;
        c.precision = SIRIUS_PRECISION_MIXED;
        c.samples_per_pixel = std::max(1, std::min(lc.samplesPerPixel, 4096));
        if (sirius_cuda_configure(m_Handle, &c) != SIRIUS_OK) { m_LastError = sirius_cuda_get_last_error(m_Handle); return; }
        sirius_frame f{};
        f.metric.family = lc.metricFamily;
        f.metric.M = lc.blackHoleMass;
        f.metric.a = double(lc.blackHoleSpin) * lc.blackHoleMass;
        f.metric.b0 = lc.throatRadius;
        f.metric.vs = lc.warpVelocity;
        f.metric.R = lc.bubbleRadius;
        f.metric.sigma = lc.bubbleSigma;
        f.camera.r = lc.observerDistance;
        f.camera.theta = lc.observerInclination;
        f.camera.phi = lc.observerAzimuth;
        f.camera.fov = lc.cameraFOV;
        f.camera.width = m_Width;
        f.camera.height = m_Height;
        f.camera.projection = SIRIUS_CAMERA_PINHOLE;
        f.disk_inner = lc.diskInnerRadius;
        f.disk_outer = lc.diskOuterRadius;
        f.ray_offset = 0;
        if (sirius_cuda_trace_frames(m_Handle, &f, 1, nullptr, m_Image.data(), nullptr) != SIRIUS_OK) {
            m_LastError = sirius_cuda_get_last_error(m_Handle);
            return;
        }
        for (size_t i = 0; i < m_Image.size(); ++i) {
            const float v = m_Image[i] * lc.exposure;
            m_Frame[4 * i + 0] = v;
            m_Frame[4 * i + 1] = v;
            m_Frame[4 * i + 2] = v;
            m_Frame[4 * i + 3] = 1.0f;
        }
    }
    float* getFrameBuffer() override { return m_Frame.empty() ? nullptr : m_Frame.data(); }
    size_t getFrameBufferSize() const override { return size_t(m_Width) * m_Height * 4 * sizeof(float); }
    bool uploadBackground(const uint8_t*, int, int) override {
        m_LastError = "background textures are not used by the geodesic engine";
        return false;
    }
    void synchronise() override {}  // every launch is synchronous
    void cleanup() override {
        if (m_Handle) sirius_cuda_destroy(m_Handle);
        m_Handle = nullptr;
    }
    std::string getLastError() const override { return m_LastError; }
    const float* intensity() const { return m_Image.data(); }

private:
    int m_Device;
    sirius_cuda_handle m_Handle = nullptr;
    int m_Width = 0, m_Height = 0;
    std::vector<float> m_Frame, m_Image;
    std::string m_LastError;
};

/// The backend factory with the CUDA slot filled (ACBF001A.cpp:16-53).
inline std::unique_ptr<IAccelerator> createAccelerator(BackendType type) {
    if (type == BackendType::CUDA) return std::make_unique<CudaAccelerator>();
    return nullptr;
}

}  // namespace sirius_b200

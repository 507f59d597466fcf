// CUDAAccelerator: the reference-side adapter for the reserved BackendType::CUDA
// slot (src/Sirius.Render/Acceleration/Backend/ACIB001A.h:27,148-189, factory slot
// ACBF001A.cpp:12,26,38,50), modelled on OptiXAccelerator (RDOX001A.h).
//
// A maintainer copies this file into the reference tree as
// src/Sirius.Render/Acceleration/CUDA/RDCA001A.h, adds this repository's include/
// to the include path and links libsirius_b200.so. It forwards IAccelerator to the
// C ABI of include/sirius_cuda.h: launch() maps LaunchConfig (ACIB001A.h:64-143)
// onto a sirius_frame and a sirius_trace_config and traces the frame in mixed
// precision; the frame buffer is RGBA float, the bolometric intensity times the
// exposure in the three colour channels.
#pragma once
#include "../Backend/ACIB001A.h"
#include "sirius_cuda.h"  // this repository's include/
#include <string>
#include <vector>

namespace Sirius::Acceleration::CUDA {

class CUDAAccelerator : public IAccelerator {
public:
    ~CUDAAccelerator() override { cleanup(); }

    BackendType getType() const override { return BackendType::CUDA; }

    DeviceCapabilities getCapabilities() const override {
        DeviceCapabilities d;
        d.supportsFP64 = true;
        return d;
    }

    bool initialise(int w, int h) override {
        if (!m_H && sirius_cuda_create(0, &m_H) != SIRIUS_OK) {
            m_H = nullptr;
            m_Err = "no CUDA device";
            return false;
        }
        m_W = w;
        m_Hgt = h;
        m_I.assign(size_t(w) * h, 0.f);
        m_FB.assign(size_t(w) * h * 4, 0.f);
        return true;
    }

    bool isInitialised() const override { return m_H != nullptr; }

    void launch(const LaunchConfig& lc) override {
        m_Err.clear();
        sirius_trace_config c;
        sirius_cuda_default_config(&c);
        c.max_steps = lc.maxSteps;
        c.max_step = lc.maxStepSize;
        c.samples_per_pixel = lc.samplesPerPixel > 0 ? lc.samplesPerPixel : 1;
        c.precision = SIRIUS_PRECISION_MIXED;
        if (sirius_cuda_configure(m_H, &c) != SIRIUS_OK) {
            m_Err = sirius_cuda_get_last_error(m_H);
            return;
        }
        sirius_frame f{};
        f.metric.family = lc.metricFamily;
        f.metric.M = lc.blackHoleMass;
        f.metric.a = lc.blackHoleSpin * lc.blackHoleMass;
        f.metric.b0 = lc.throatRadius;
        f.metric.vs = lc.warpVelocity;
        f.metric.R = lc.bubbleRadius;
        f.metric.sigma = lc.bubbleSigma;
        f.camera.r = lc.observerDistance;
        f.camera.theta = lc.observerInclination;
        f.camera.phi = lc.observerAzimuth;
        f.camera.fov = lc.cameraFOV;
        f.camera.width = m_W;
        f.camera.height = m_Hgt;
        f.disk_inner = lc.diskInnerRadius;
        f.disk_outer = lc.diskOuterRadius;
        if (sirius_cuda_trace_frames(m_H, &f, 1, nullptr, m_I.data(), nullptr) != SIRIUS_OK) {
            m_Err = sirius_cuda_get_last_error(m_H);
            return;
        }
        for (size_t i = 0; i < m_I.size(); ++i) {
            const float v = m_I[i] * lc.exposure;
            m_FB[4 * i] = m_FB[4 * i + 1] = m_FB[4 * i + 2] = v;
            m_FB[4 * i + 3] = 1.f;
        }
    }

    float* getFrameBuffer() override { return m_FB.data(); }
    size_t getFrameBufferSize() const override { return m_FB.size() * sizeof(float); }
    bool uploadBackground(const uint8_t*, int, int) override { return false; }
    void synchronise() override {}

    void cleanup() override {
        if (m_H) sirius_cuda_destroy(m_H);
        m_H = nullptr;
    }

    std::string getLastError() const override { return m_Err; }

private:
    sirius_cuda_handle m_H = nullptr;
    int m_W = 0, m_Hgt = 0;
    std::vector<float> m_I, m_FB;
    std::string m_Err;
};

}  // namespace Sirius::Acceleration::CUDA

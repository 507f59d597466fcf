/*
 * sirius_cuda.h — C ABI of the B200 geodesic engine.
 *
 * This is the drop-in boundary for Sirius's per-pixel null-geodesic hot path.
 * It replaces, for the CUDA backend slot the reference reserves:
 *   - the OptiX C entry points  sirius_optix_*      (src/Sirius.Render/Acceleration/OptiX/RDOP006A.h:10-39)
 *   - the per-ray CPU tracer    GeodesicTracer::trace (src/Sirius.Render/Integration/GTRC001A.h:220, GTRC001A.cpp:139-592)
 *   - the integrator step       Geodesic::integrateStepRK45 (src/Sirius.Core/Geodesic/PHGD001A.h:120)
 *   - the metric evaluation     IMetric::evaluate (src/Sirius.Core/Metric/PHMT000A.h:38)
 *
 * Conventions (all entry points):
 *   - plain C types only; every struct below is POD with a fixed layout (static
 *     asserts in the implementation pin the sizes);
 *   - every call returns an int status (SIRIUS_OK == 0); no C++ exception ever
 *     crosses this boundary; the last error message of a handle is available
 *     from sirius_cuda_get_last_error();
 *   - "host" entry points take caller-owned HOST buffers, copy in, run, copy out
 *     and synchronise before returning (like sirius_optix_launch, RDOP001A.cu:1044);
 *   - "_device" entry points take caller-owned DEVICE buffers and a CUDA stream
 *     (cudaStream_t passed as void*), and are stream-ordered and asynchronous;
 *   - one handle per host thread; a handle owns its device scratch memory;
 *   - there is no CPU fallback: if the CUDA kernels cannot run the call fails
 *     with SIRIUS_ERR_CUDA / SIRIUS_ERR_NO_DEVICE.
 */
#ifndef SIRIUS_CUDA_H
#define SIRIUS_CUDA_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SIRIUS_CUDA_ABI_VERSION 2

/* ---- status codes --------------------------------------------------------- */
enum sirius_status {
    SIRIUS_OK = 0,
    SIRIUS_ERR_INVALID_ARGUMENT = 1,
    SIRIUS_ERR_CUDA = 2,
    SIRIUS_ERR_NO_DEVICE = 3,
    SIRIUS_ERR_NOT_CONFIGURED = 4,
    SIRIUS_ERR_TIMEOUT = 5,
    SIRIUS_ERR_OUT_OF_MEMORY = 6,
    SIRIUS_ERR_UNSUPPORTED = 7
};

/* ---- metric families (IMetric implementations) ---------------------------- */
enum sirius_metric_family {
    SIRIUS_METRIC_KERR_SCHILD = 0,   /* KerrSchildFamily (M,a,Q,Lambda), PHMT100A.h:72   */
    SIRIUS_METRIC_MORRIS_THORNE = 1, /* MorrisThorneFamily, PHMT101A.h:111               */
    SIRIUS_METRIC_ALCUBIERRE = 2     /* WarpDriveFamily, PHMT102A.h:71                   */
};

/* Morris-Thorne shape functions (WormholeShapeType, PHMT101A.h) */
enum sirius_wormhole_shape {
    SIRIUS_WORMHOLE_ELLIS = 0,
    SIRIUS_WORMHOLE_ZERO_TIDAL = 1,
    SIRIUS_WORMHOLE_ABSURDLY_BENIGN = 2
};

/* ---- ray outcomes ---------------------------------------------------------
 * The first five keep the order of TraceResult::Outcome (GTRC001A.h:46-52);
 * the rest split the reference's catch-all MAX_STEPS into explicit causes. */
enum sirius_outcome {
    SIRIUS_ESCAPED = 0,
    SIRIUS_HORIZON = 1,
    SIRIUS_DISK_HIT = 2,
    SIRIUS_MAX_STEPS = 3,
    SIRIUS_SPIRALING = 4,
    SIRIUS_NUMERICAL_FAILURE = 5, /* NaN/Inf in the state (reference terminated = 3) */
    SIRIUS_STEP_UNDERFLOW = 6,    /* h <= min_step after a reject (reference terminated = 5) */
    SIRIUS_THROAT = 7,            /* reached the Morris-Thorne throat clamp */
    SIRIUS_REJECTED = 8           /* reference-compatible mode only: a rejected step ends the ray
                                     (GTRC001A.cpp:272-277 reports it as MAX_STEPS) */
};

/* ---- precision modes ------------------------------------------------------ */
enum sirius_precision {
    SIRIUS_PRECISION_FP64 = 0,  /* every operation in FP64 (the plain FP64 GPU integrator) */
    SIRIUS_PRECISION_MIXED = 1  /* FP32 dual-number RHS, FP64 state accumulation, FP64
                                   constraint re-projection, FP64 RHS and error control inside
                                   the photon region and near the horizon */
};

enum sirius_integrator {
    SIRIUS_INTEGRATOR_DP45 = 0,       /* Dormand-Prince RK45, PHGD001A.cpp:530-641 */
    SIRIUS_INTEGRATOR_SYMPLECTIC = 1  /* Yoshida-composed kick-drift-kick, PHSI001A.h:136-215 */
};

enum sirius_projection {
    SIRIUS_CAMERA_PINHOLE = 0,        /* PinholeCamera, CMBS001A.h:113-205 */
    SIRIUS_CAMERA_EQUIRECTANGULAR = 1 /* 360x180 sky map (LensType::Panoramic has no
                                         implementation in the reference, CMBS001A.h:68,351-362) */
};

/* Whose frame the pixel directions are given in. */
enum sirius_observer {
    SIRIUS_OBSERVER_STATIC = 0, /* the reference's convention (GTRC001A.cpp:15-134): the camera at
                                   the spherical map (r sin(theta) cos(phi), ...) of its (r, theta,
                                   phi), pixel directions as coordinate velocities there, k^0 from the
                                   null condition; redshifts relative to a static observer */
    SIRIUS_OBSERVER_ZAMO = 1    /* Kerr-Schild family with Lambda = 0 only: the camera at the
                                   Kerr-Schild point whose Boyer-Lindquist coordinates are exactly (r,
                                   theta, phi) (the oblate map, PHCT002A.h:149-169), pixel directions
                                   as unit vectors in the orthonormal frame of the zero-angular-momentum
                                   observer there (Bardeen 1972 tetrad; FIDO, RDOP002A.cu:2528-2604),
                                   photon energy 1 in that frame; redshifts relative to that observer */
};

/* ---- metric parameters ---------------------------------------------------- */
typedef struct sirius_metric {
    int32_t family;   /* enum sirius_metric_family */
    int32_t shape;    /* enum sirius_wormhole_shape (Morris-Thorne only) */
    double M, a, Q, Lambda;      /* Kerr-Schild family; a is the spin length a = a_* M */
    double b0, Phi0;             /* Morris-Thorne throat radius and constant redshift */
    double vs, sigma, R;         /* Alcubierre bubble velocity, wall steepness, radius */
} sirius_metric;

/* ---- camera (CameraConfig, CMBS001A.h:37-58) -------------------------------- */
typedef struct sirius_camera {
    double t, r, theta, phi;     /* observer position (Boyer-Lindquist / spherical) */
    float yaw, pitch, roll;      /* radians */
    float fov;                   /* degrees (pinhole) */
    int32_t width, height;
    int32_t projection;          /* enum sirius_projection */
    int32_t observer;            /* enum sirius_observer (one sample per pixel, at the pixel centre) */
} sirius_camera;

/* ---- one frame of a (possibly heterogeneous) batch ------------------------ */
typedef struct sirius_frame {
    sirius_metric metric;
    sirius_camera camera;
    double disk_inner;           /* <= 0: use the prograde ISCO of the frame's (M,a) */
    double disk_outer;
    int64_t ray_offset;          /* first ray/pixel index of this frame in the batch outputs */
    /* Row window: trace only camera rows [row_begin, row_begin + row_count) of the
     * width x height image (row_count 0: every row, row_begin 0). Each ray is the
     * one the full frame traces through that pixel, so a frame split into row
     * blocks across devices reassembles the full frame bit for bit (the tile
     * distribution of ACMG001A.h:256). The frame then holds width * row_count
     * rays, output (y - row_begin) * width + x. */
    int32_t row_begin;
    int32_t row_count;
} sirius_frame;

/* ---- a host-generated camera ray (CameraRay, CMBS001A.h:26-32) -------------- */
typedef struct sirius_camera_ray {
    double origin[4];            /* (t, r, theta, phi) Boyer-Lindquist */
    double direction[4];         /* (0, v_r, r v_theta, r sin(theta) v_phi) */
} sirius_camera_ray;

/* ---- tracer + integrator configuration -------------------------------------
 * Mirrors IntegratorConfig (PHGD001A.h:48-58), TracerConfig (GTRC001A.h:162-196)
 * and the precision / batching knobs of the B200 engine. */
typedef struct sirius_trace_config {
    /* IntegratorConfig */
    double abs_tolerance;
    double rel_tolerance;
    double min_step;
    double max_step;
    double initial_step;
    double safety_factor;
    double step_grow_max;
    double step_shrink_min;
    /* TracerConfig */
    double escape_radius;        /* coordinate radius sqrt(x^2+y^2+z^2) beyond which an outgoing ray escapes */
    double horizon_factor;       /* terminate at r_BL < horizon_factor * r_+ */
    int32_t max_steps;           /* accepted steps per ray */
    int32_t enable_disk;         /* thin Novikov-Thorne disk crossings */
    double disk_temperature_inner;
    double crossing_weight_decay;/* image intensity weight exp(-decay * n) for crossing n */
    /* volumetric radiative transfer */
    int32_t enable_volumetric;
    int32_t n_bins;              /* frequency bins, <= SIRIUS_MAX_BINS */
    double nu_min, nu_max;       /* log-spaced bin centres, in units of the reference frequency */
    double vol_j0;               /* emissivity normalisation: j = vol_j0 r^-2 exp(-z^2/(2 (h r)^2)) (nu_em)^-s */
    double vol_alpha_over_j;     /* absorption alpha_nu = vol_alpha_over_j * j_nu */
    double vol_height_ratio;     /* h in the Gaussian scale height h*r */
    double vol_spectral_index;   /* s */
    int32_t vol_substeps;        /* midpoint samples per step segment inside the emitting volume */
    /* engine knobs */
    int32_t integrator;          /* enum sirius_integrator */
    int32_t precision;           /* enum sirius_precision */
    int32_t compat;              /* 1: reference-compatible semantics (float roundings, stop on reject,
                                    E-changing normalizeNull, Euclidean horizon/disk radii) */
    int32_t projection_period;   /* FP64 constraint re-projection every N accepted steps (0 = never) */
    int32_t spiral_check;        /* 1: the reference's spiral early-out (GTRC001A.cpp:322-352) */
    double island_factor;        /* FP64 island: r_BL < island_factor * r_ph(retrograde) or r_BL < 2 r_+ */
    double critical_band;        /* mixed precision, Kerr-Newman frames: a ray whose radial potential
                                    R(r) = ((r^2+a^2)E - a L)^2 - Delta (Q + (L - a E)^2) has
                                    |min R / (E^2 r^4)| < critical_band (it skims the photon region)
                                    runs every step in FP64 */
    double symplectic_step;      /* fixed d-lambda of the symplectic integrator */
    int32_t symplectic_order;    /* 4, 6 or 8 (Yoshida) */
    int32_t block_size;          /* threads per block of the trace kernel: 32, 64 or 128 (0 = 128) */
    int32_t refill_threshold;    /* persistent mode: refill a warp when fewer than this many lanes are
                                    live (1..32; 0 = 1, i.e. only once the whole warp is done, which keeps
                                    the 32 rays of a warp on neighbouring pixels and so coherent) */
    int32_t blocks_per_sm;       /* 0 = one thread per ray, a block per 128 consecutive rays (default);
                                    1..4 = persistent grid of SMs * blocks_per_sm blocks that pull rays
                                    from a queue; < 0 = persistent, occupancy-sized grid */
    int32_t watchdog_ms;         /* bound on any spin-wait inside the kernels */
    int32_t samples_per_pixel;   /* 0 or 1: one ray through each pixel centre. n > 1: the image and
                                    spectra average a g x g stratified grid, g = floor(sqrt(n)), of
                                    sub-pixel rays at ((sx + 0.5) / g, (sy + 0.5) / g) as
                                    RenderSession::shadePixel does (SNRS001A.cpp:480-530), one
                                    progressive pass per sub-pixel offset, summed in a fixed order;
                                    per-ray results are then not available (NULL), and the launch
                                    statistics count the last pass. At most 4096. */
    int32_t max_registers;       /* one-thread-per-ray launch: the register cap of the trace kernel,
                                    255 (8 warps per SM), 168 (12) or 128 (16; these two spill).
                                    0 = measured default: 128 for mixed DP45, 168 for FP64 DP45,
                                    255 for the symplectic integrator. The budgets' FP32
                                    roundings differ, so mixed
                                    images at different caps agree to ~1e-5 of the peak, not
                                    bit for bit. The persistent launch takes its budget from
                                    blocks_per_sm. */
    int32_t rays_per_thread;     /* one-thread-per-ray launch of mixed-precision DP45 over Kerr-Schild
                                    frames: 2 = each thread carries two neighbouring rays whose FP32
                                    arithmetic runs as packed pairs (f32x2); 1 = one ray per thread;
                                    0 = the measured default. Other configurations trace one ray
                                    per thread. The two forms round differently (FP32 contraction
                                    order), so their images agree to ~1e-5 of the peak, not bit
                                    for bit; within one form a ray's result does not depend on its
                                    pairing. */
    int32_t reserved[2];
} sirius_trace_config;

#define SIRIUS_MAX_BINS 32
#define SIRIUS_FLAG_NUMERICAL_FAILURE 1  /* TraceResult::numerical_failure */
#define SIRIUS_FLAG_PHOTON_RING 2        /* TraceResult::photon_ring */
#define SIRIUS_MAX_CROSSINGS 4

/* ---- per-ray result (TraceResult, GTRC001A.h:44-157) ------------------------ */
typedef struct sirius_ray_result {
    int32_t outcome;             /* enum sirius_outcome */
    int32_t steps;               /* accepted steps */
    int32_t rejected;            /* rejected step attempts */
    int32_t n_crossings;         /* valid disk crossings (<= 4) */
    double final_x[4];           /* KS Cartesian (t,x,y,z) (spherical for Morris-Thorne) */
    double final_p[4];           /* covariant momentum p_mu at termination */
    float final_k[4];            /* contravariant k^mu = g^{mu nu} p_nu at termination */
    float disk_r[SIRIUS_MAX_CROSSINGS];      /* radius at crossing (BL r; Euclidean cylindrical in compat) */
    float disk_phi[SIRIUS_MAX_CROSSINGS];
    float disk_g[SIRIUS_MAX_CROSSINGS];      /* redshift factor g at crossing */
    float disk_flux[SIRIUS_MAX_CROSSINGS];   /* Novikov-Thorne/Page-Thorne flux F(r) */
    int32_t equatorial_crossings;
    int32_t image_order;
    float total_phi_change;
    float min_radius;
    float intensity;             /* bolometric: sum_n exp(-decay n) g_n^4 F(r_n) (+ volumetric) */
    int32_t fp64_steps;          /* accepted steps taken on the FP64 island path (mixed precision) */
    /* conserved quantities (computeConservedQuantities, MTTP001A.h:114-132), evaluated in
     * FP64 from the FP64 state: E = -p_t, L_z = x p_y - y p_x (the Kerr-Schild azimuthal
     * momentum), Carter Q = p_theta^2 + cos^2(theta) (-a^2 E^2 + L_z^2 / sin^2(theta)) */
    double E, Lz, Carter;        /* at termination */
    double E0, Lz0, Carter0;     /* at initialisation */
    float null_drift_max;        /* max over accepted steps of |g^{mu nu} p_mu p_nu| before re-projection */
    float null_final;            /* |g^{mu nu} p_mu p_nu| of the returned state */
    float impact_parameter;
    float magnification;
    float optical_depth;
    int32_t flags;               /* SIRIUS_FLAG_* bits */
} sirius_ray_result;

/* ---- launch statistics ------------------------------------------------------ */
typedef struct sirius_launch_stats {
    double kernel_ms;            /* device time of the trace kernel(s), CUDA events on the launch stream */
    double total_ms;             /* device time of the whole call including copies */
    int64_t rays;
    int64_t accepted_steps;
    int64_t rejected_steps;
    int64_t fp64_steps;
    int32_t kernel_launches;     /* kernels this engine launched for the call */
    int32_t grid_blocks;
    int32_t block_size;
    int32_t status_flags;        /* bit 0: watchdog expired in a spin-wait */
} sirius_launch_stats;

typedef void* sirius_cuda_handle;

/* ---- lifecycle (sirius_optix_create/destroy/initialize, RDOP006A.h:14-19) ---- */
int sirius_cuda_create(int device, sirius_cuda_handle* out_handle);
int sirius_cuda_destroy(sirius_cuda_handle handle);
const char* sirius_cuda_get_last_error(sirius_cuda_handle handle);
int sirius_cuda_abi_version(void);

/* The defaults of TracerConfig/IntegratorConfig as set by RenderSession
 * (SNRS001A.cpp:103-129) with the engine knobs at their defaults. */
int sirius_cuda_default_config(sirius_trace_config* out_config);
int sirius_cuda_configure(sirius_cuda_handle handle, const sirius_trace_config* config);

/* ---- frame rendering (IAccelerator::launch + getFrameBuffer, ACIB001A.h:166-170;
 *      sirius_optix_launch + sirius_optix_get_frame_buffer, RDOP006A.h:22,28) ---------
 * Camera rays are generated on the device. Outputs are indexed by
 * frame.ray_offset + y * width + x. Any output pointer may be NULL.
 *   image:   one float per pixel (bolometric intensity)
 *   spectra: n_bins floats per pixel (volumetric transfer), pixel-major
 * Host variant: host buffers, synchronous. When every output given is
 * page-locked (cudaHostAlloc / cudaHostRegister) and one frame of at least
 * 2048 pixel tiles (16 x 8) is traced with samples_per_pixel <= 1, the trace
 * runs as up to 8 launches of consecutive tile rows on their own streams, and
 * each piece's outputs are copied to the host while the later pieces trace;
 * the outputs are bit for bit those of one launch. */
int sirius_cuda_trace_frames(sirius_cuda_handle handle,
                             const sirius_frame* frames, int32_t n_frames,
                             sirius_ray_result* results, float* image, float* spectra);

/* Device variant: frames/results/image/spectra are device pointers; stream-ordered
 * on `stream` (a cudaStream_t; NULL = the legacy default stream). Timing and
 * counters of the launch are read by the next sirius_cuda_last_stats call. */
int sirius_cuda_trace_frames_device(sirius_cuda_handle handle,
                                    const sirius_frame* d_frames, int32_t n_frames,
                                    int64_t total_rays,
                                    sirius_ray_result* d_results, float* d_image, float* d_spectra,
                                    void* stream);

/* Allocation-free form of sirius_cuda_trace_frames_device (no counterpart in the
 * reference): same arguments, same results, but the launch scratch (frame
 * descriptors, ray-queue and step counters, status word, per-frame disk flux
 * tables; 160 KB in all) lives in a static device array of the library, held
 * by every GPU that loads it, so the call makes no device allocation. For
 * callers that cannot let a library allocate: a host whose own allocator
 * already holds the device memory it is given, or a frame loop that cannot
 * afford the implicit device-wide synchronisation of cudaMalloc/cudaFree.
 * Limits: at most SIRIUS_STATIC_MAX_FRAMES frames per call (more is rejected
 * with SIRIUS_ERR_INVALID_ARGUMENT). Each call copies the frame descriptors to
 * the host and synchronises `stream` before it launches; it returns while its
 * kernels still run. The counters and status word must start a launch at zero;
 * the call zeroes them on `stream` itself. The scratch is one per device, and
 * every call rewrites it: calls whose kernels overlap on one device race on
 * it. A host-side lock is not enough, because a call returns before its kernels
 * end: order successive calls on the device, on one stream, or with an event
 * recorded after call N that call N+1's stream waits on. The scratch address
 * is resolved on the first call per device; make that first call before any
 * stream capture. sirius_cuda_last_stats does not describe these launches: the
 * handle's statistics keep describing its last traced call. */
#define SIRIUS_STATIC_MAX_FRAMES 64
int sirius_cuda_trace_frames_static(sirius_cuda_handle handle,
                                    const sirius_frame* d_frames, int32_t n_frames,
                                    int64_t total_rays,
                                    sirius_ray_result* d_results, float* d_image, float* d_spectra,
                                    void* stream);

/* ---- surrogate MLP (no counterpart in the reference) ---------------------------
 * 5 -> 256 -> 256 -> 256 -> 256 -> 4, SiLU after the hidden layers, BF16
 * weights and activations with FP32 accumulation on the tensor cores.
 * params: host array of SIRIUS_SURROGATE_PARAMS floats in torch nn.Linear
 *   order (out x in): W1[256][5] b1[256] W2[256][256] b2 W3 b3 W4 b4 W5[4][256] b5[4].
 * infer: d_features = n x 5 floats, d_out = n x 4 floats (device), stream-ordered
 *   on `stream` and synchronous on return. */
#define SIRIUS_SURROGATE_PARAMS 199940
int sirius_cuda_surrogate_load(sirius_cuda_handle handle, const float* params, int64_t n_params);
int sirius_cuda_surrogate_infer(sirius_cuda_handle handle, const float* d_features, int64_t n, float* d_out,
                                void* stream);

/* Surrogate-gated rendering of Kerr frames (thin Novikov-Thorne disk).
 * Per pixel: features f = (2 a* - 1, (theta_o[deg] - 47)/42, alpha/20, beta/20,
 * (r_obs - 110)/90) with the celestial coordinates of the camera ray's own
 * constants of motion, alpha = -L_z / (E sin theta_o), beta = p_theta / E; the MLP
 * predicts (disk-hit logit, r_1 = 15 (1 + o_1), g_1, higher-order intensity / 1e-3)
 * and the pixel takes g_1^4 F(r_1) + higher orders. Rays within gate_band (M) of
 * the critical curve (Bardeen's spherical photon orbits at the camera's
 * inclination), an audit_fraction of the others (runs of 32 consecutive pixels
 * chosen by a hash seeded with audit_seed), and
 * every ray of a frame that is not charge- and Lambda-free Kerr are integrated
 * instead (the configured integrator, compacted into one launch) and overwrite
 * their pixels. gate (optional): per pixel 0 = MLP, 1 = gated, 2 = audit, 3 = empty
 * (no disk crossing predicted around it: intensity 0, no MLP; see empty_skip). A ray
 * that never crosses the disk plane inside the disk carries no light (thin disk only),
 * so the coarse pass's confident no-hit cells need no per-pixel network.
 * The inner-disk gate: the MLP first runs on a coarse grid (every
 * coarse_stride-th pixel in each direction, the cell centres); every pixel whose
 * coarse cell or a neighbouring one predicts a disk hit at r_1 < inner_gate *
 * r_in is integrated too. There the flux rises steeply from zero at the inner
 * edge, so a small error of the network's r_1 is a large error of the pixel.
 * audit_budget > 0: when the audit finds max |I_mlp - I| / max I above it, the
 * frame is rendered once more with the critical-curve band and inner_gate 1.5
 * times wider (sirius_surrogate_stats.rerendered). */
typedef struct {
    double gate_band;          /* half width of the gate around the critical curve, M (0.3) */
    double audit_fraction;     /* fraction of ungated rays also integrated (0.01) */
    uint32_t audit_seed;
    float inner_gate;          /* r_1 bound of the inner-disk gate in units of r_in: 0 = 2.75, < 0 = off */
    int32_t coarse_stride;     /* pixels per coarse cell side of the inner-disk gate: 0 = 8 */
    float audit_budget;        /* 0: the audit only reports */
    int32_t empty_skip;        /* 0 = on, < 0 = off: pixels whose coarse cell and its eight
                                  neighbours all predict no disk crossing (hit logit below -4)
                                  take intensity 0 without the per-pixel MLP (gate 3); the MLP
                                  runs only on the pixels it shades and the audit pixels. Off
                                  when d_image_mlp is requested (it needs every pixel). */
    int32_t reserved;
} sirius_surrogate_config;

typedef struct {
    int64_t rays, integrated;
    float ms_features, ms_mlp, ms_shade, ms_trace, ms_total;  /* CUDA-event times of the stages */
    /* the audit's judgement of the surrogate: over the audit pixels (gate 2), where
     * both the MLP's and the integrator's intensity exist, sum |I_mlp - I| / sum I
     * and max |I_mlp - I| / max I */
    int32_t audit_count;
    float audit_rel_l1, audit_rel_max;
    int32_t rerendered;        /* 1: the audit exceeded audit_budget and the frame was rendered again */
    int32_t coarse_rays;       /* MLP rows of the inner-disk gate's coarse pass */
} sirius_surrogate_stats;

/* features (n x 5 floats, device) and gate (n bytes, device, may be NULL) of the frames' pixels; the
 * gate's inner-disk part needs loaded weights (its coarse MLP pass) and is left out without them */
int sirius_cuda_surrogate_features(sirius_cuda_handle handle, const sirius_frame* frames, int32_t n_frames,
                                   const sirius_surrogate_config* config, float* d_features, uint8_t* d_gate,
                                   void* stream);
/* host frame descriptors, device outputs; synchronous on return */
int sirius_cuda_render_surrogate_device(sirius_cuda_handle handle, const sirius_frame* frames, int32_t n_frames,
                                        const sirius_surrogate_config* config, float* d_image, float* d_image_mlp,
                                        uint8_t* d_gate, void* stream, sirius_surrogate_stats* stats);
/* host buffers (image_mlp: the MLP's own image before the integrated rays overwrite it; may be NULL) */
int sirius_cuda_render_surrogate(sirius_cuda_handle handle, const sirius_frame* frames, int32_t n_frames,
                                 const sirius_surrogate_config* config, float* image, float* image_mlp,
                                 uint8_t* gate, sirius_surrogate_stats* stats);

/* ---- surrogate training on the tensor cores (no counterpart in the reference) ----
 * The network above, trained by the library's own tcgen05 forward and backward
 * GEMMs and an Adam kernel; one optimiser step is captured as a CUDA graph and
 * replayed. Training rows live on the device: d_features n x 5 floats (as
 * sirius_cuda_surrogate_features writes them), d_targets n x 4 floats
 * (disk hit 0/1, r_1 / 15 - 1, g_1, higher-order intensity * 1e3), d_weights n
 * floats (the squared errors' brightness weights).
 * Loss per batch of B rows: BCE(o_0, hit) + 100 (l_r + l_g) + 10 l_h with
 * l_r = sum hit w (o_1 - t_1)^2 / sum hit w, l_g likewise on o_2, and
 * l_h = sum w (o_3 - t_3)^2 / sum w. loss_parts = (BCE, l_r, l_g, l_h). */
typedef struct {
    int32_t batch;             /* rows per optimiser step, a multiple of 128 (16384) */
    int32_t reserved0;
    int64_t total_steps;       /* length of the learning-rate schedule */
    float max_lr;              /* peak learning rate (2e-3): linear warm-up from max/25, cosine to max * 4e-6 */
    float warmup_fraction;     /* 0.05 */
    float beta1, beta2, eps;   /* Adam: 0.9, 0.999, 1e-8 */
    float weight_decay;        /* decoupled (AdamW), 0 */
    uint32_t seed;             /* key of the per-epoch row permutation */
    int32_t reserved[5];
} sirius_train_config;

void sirius_cuda_default_train_config(sirius_train_config* config);
/* FP32 master weights from params (host, SIRIUS_SURROGATE_PARAMS floats, nn.Linear
 * order); Adam moments and the step counter reset to zero. */
int sirius_cuda_train_init(sirius_cuda_handle handle, const float* params, const sirius_train_config* config);
/* n_steps optimiser steps over rows [0, n_rows): each epoch visits the rows of
 * n_rows / batch full batches in a fresh keyed permutation; synchronous on return.
 * device_ms (may be NULL): CUDA-event time of the steps on the library's stream. */
int sirius_cuda_train_steps(sirius_cuda_handle handle, const float* d_features, const float* d_targets,
                            const float* d_weights, int64_t n_rows, int64_t n_steps, float* device_ms);
/* loss parts of the current weights over rows [0, n_rows), in batches of the configured size
 * (averaged, each batch weighted by its rows) */
int sirius_cuda_train_evaluate(sirius_cuda_handle handle, const float* d_features, const float* d_targets,
                               const float* d_weights, int64_t n_rows, float* loss_parts);
/* loss parts and gradient (host, SIRIUS_SURROGATE_PARAMS floats, parameter order) of
 * one batch of rows [0, n_rows), n_rows a multiple of 128 and at most the batch; no update */
int sirius_cuda_train_gradient(sirius_cuda_handle handle, const float* d_features, const float* d_targets,
                               const float* d_weights, int64_t n_rows, float* loss_parts, float* grad);
/* the FP32 master weights (host) and the optimiser steps taken */
int sirius_cuda_train_params(sirius_cuda_handle handle, float* params, int64_t* steps);

/* ---- prepared frames: a launch sequence for CUDA graph capture ------------------
 * (no counterpart in the reference) prepare_frames does the host work of a
 * frame batch once: it validates the frames and uploads their descriptors into
 * scratch that belongs to the prepared batch (descriptors, queue and counter
 * words, status word, flux tables); synchronous. launch_prepared then issues
 * the trace of those frames on `stream` as device work only (memsets and
 * kernels: no allocation, no host synchronisation, no statistics), so a caller
 * can capture it in a CUDA graph and replay the graph. The prepared scratch
 * lives until the next prepare_frames or destroy; a graph captured before
 * either of those must not be replayed after it. A captured graph renders the
 * configuration in force when it was captured. One sample per pixel
 * (samples_per_pixel > 1 is refused). Outputs as sirius_cuda_trace_frames_device. */
int sirius_cuda_prepare_frames(sirius_cuda_handle handle, const sirius_frame* frames, int32_t n_frames,
                               int64_t* total_rays);
int sirius_cuda_launch_prepared(sirius_cuda_handle handle, sirius_ray_result* d_results, float* d_image,
                                float* d_spectra, void* stream);

/* ---- beams: geodesic deviation around each pixel ray -------------------------
 * The counterpart of BeamIntegratorD (INBI001A.h:178-363), on the engine's
 * Hamiltonian form: each pixel's ray (FP64, Dormand-Prince 5(4) with the
 * configured tolerances, whatever the precision setting) carries the two
 * tangent vectors dy/du, dy/dv of its state with respect to its start in pixel
 * coordinates (the linearised geodesic equation). For an escaped ray,
 * magnification = |dd/du x dd/dv| / |dn/du x dn/dv|: the solid angle of the
 * pixel in the camera frame over the solid angle it covers on the sky (d the
 * start direction, n the escape direction); 1 in flat space. Kerr-Schild
 * family only; host frames and results (one per pixel); synchronous. */
typedef struct {
    int32_t outcome;             /* SIRIUS_ESCAPED, HORIZON, DISK_HIT, MAX_STEPS or NUMERICAL_FAILURE */
    int32_t steps;               /* accepted steps */
    float magnification;         /* escaped rays; 0 otherwise */
    float parity;                /* escaped rays: +1 direct image, -1 mirror-reversed; 0 otherwise */
    float final_dir[3];          /* escaped rays: unit escape direction (Kerr-Schild Cartesian) */
    int32_t reserved;
} sirius_beam_result;

int sirius_cuda_trace_beams(sirius_cuda_handle handle, const sirius_frame* frames, int32_t n_frames,
                            sirius_beam_result* results);

/* ---- image output of a headless frame buffer ---------------------------------
 * Host functions (no handle, no device): row-major float pixels, top row first.
 * Pixel conversions as the reference's output drivers:
 *   write_png  PNGWriter::writeRGB / writeRGBA (OUPN001A.cpp:45-97): colour channels
 *              through the sRGB curve to 8 bits (toSRGB8, OUPN001A.h:154-163), alpha
 *              linear; channels 3 (RGB) or 4 (RGBA)
 *   write_exr  EXRWriter::writeEXR (OUEW001A.cpp:17-195): OpenEXR scanline file, HALF
 *              channels B, G, R (A, B, G, R), ZIP compression; channels 3 or 4
 *   write_pfm  EXRWriter::writePFM (OUEW001A.h:108-124): RGB floats, bottom row first
 *   write_ppm  EXRWriter::writePPM (OUEW001A.h:94-105): RGB through the sRGB curve
 * SIRIUS_ERR_INVALID_ARGUMENT for bad sizes or a file that cannot be written. */
int sirius_cuda_write_png(const char* path, int32_t width, int32_t height, int32_t channels, const float* pixels);
int sirius_cuda_write_exr(const char* path, int32_t width, int32_t height, int32_t channels, const float* pixels);
int sirius_cuda_write_pfm(const char* path, int32_t width, int32_t height, const float* rgb);
int sirius_cuda_write_ppm(const char* path, int32_t width, int32_t height, const float* rgb);

/* ---- batch form of GeodesicTracer::trace(const CameraRay&) (GTRC001A.h:220) ----
 * Host-generated rays through one metric; disk_inner <= 0 selects the ISCO. */
int sirius_cuda_trace_rays(sirius_cuda_handle handle, const sirius_metric* metric,
                           double disk_inner, double disk_outer,
                           const sirius_camera_ray* rays, int64_t n_rays,
                           sirius_ray_result* results);

/* ---- IMetric::evaluate on the device for a batch of points (PHMT000A.h:38) -------
 * positions: n x 4; g: n x 16; dg: n x 64 with dg[l*16 + m*4 + n] = d_l g_mn.
 * precision selects the FP64 or FP32 dual-number path. Host buffers. */
int sirius_cuda_metric_evaluate(sirius_cuda_handle handle, const sirius_metric* metric,
                                const double* positions, int64_t n, int32_t precision,
                                double* g, double* dg);

/* ---- one Dormand-Prince step for a batch of states (Geodesic::integrateStepRK45,
 *      PHGD001A.cpp:530-641, without termination logic) ---------------------------
 * state: n x 8 (x^mu, p_mu), h: n step sizes. On return state holds the accepted
 * state (or the input if rejected), h the next step size, accepted[i] 0/1 and
 * err[i] the scaled error norm. Host buffers. */
int sirius_cuda_dp45_step(sirius_cuda_handle handle, const sirius_metric* metric,
                          double* state, double* h, int32_t* accepted, double* err,
                          int64_t n);

/* ---- statistics of the last trace call ---------------------------------------- */
int sirius_cuda_last_stats(sirius_cuda_handle handle, sirius_launch_stats* out_stats);

/* ---- autotuner: times the one-thread-per-ray launch (register caps; one ray or
 * two packed rays per thread) and the persistent launch (blocks/SM x refill
 * threshold) on the given frames and stores the best setting in the handle's
 * configuration.
 * The chosen values are written to *out_config (may be NULL). ---------------- */
int sirius_cuda_autotune(sirius_cuda_handle handle, const sirius_frame* frames, int32_t n_frames,
                         sirius_trace_config* out_config);

/* ---- SIMT peak microbenchmark: FMA-chain throughput of the device in FLOP/s
 * (one FMA = 2 FLOP); precision 0 = FP64, 1 = FP32. ------------------------- */
int sirius_cuda_measure_fma_peak(sirius_cuda_handle handle, int32_t precision, double* flops_per_s);

/* ---- algorithmic operation count (host only, no device needed): one
 * right-hand-side evaluation of the metric family as the kernels compute it,
 * one DP45 attempt (6 evaluations + stage algebra) and one accepted step
 * (attempt + FP64 re-projection). The roofline numerator of the benchmark. */
int sirius_cuda_flop_count(const sirius_metric* metric, double* rhs_flops, double* attempt_flops,
                           double* accepted_step_flops);

#ifdef __cplusplus
}
#endif

#endif /* SIRIUS_CUDA_H */

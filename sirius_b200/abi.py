"""ctypes mirror of include/sirius_cuda.h (struct layouts, enums, defaults).

The C header is the source of truth; tests/test_abi.py checks every size and
field offset here against the compiled library.
"""
import ctypes as C

ABI_VERSION = 2
MAX_BINS = 32
MAX_CROSSINGS = 4
STATIC_MAX_FRAMES = 64  # SIRIUS_STATIC_MAX_FRAMES
SURROGATE_PARAMS = 199940  # SIRIUS_SURROGATE_PARAMS

# status
OK = 0
ERR_INVALID_ARGUMENT = 1
ERR_CUDA = 2
ERR_NO_DEVICE = 3
ERR_NOT_CONFIGURED = 4
ERR_TIMEOUT = 5
ERR_OUT_OF_MEMORY = 6
ERR_UNSUPPORTED = 7

# metric families
KERR_SCHILD = 0
MORRIS_THORNE = 1
ALCUBIERRE = 2

# outcomes (first five: TraceResult::Outcome order)
ESCAPED = 0
HORIZON = 1
DISK_HIT = 2
MAX_STEPS = 3
SPIRALING = 4
NUMERICAL_FAILURE = 5
STEP_UNDERFLOW = 6
THROAT = 7
REJECTED = 8
OUTCOME_NAMES = ["escaped", "horizon", "disk_hit", "max_steps", "spiraling", "numerical_failure",
                 "step_underflow", "throat", "rejected"]

PRECISION_FP64 = 0
PRECISION_MIXED = 1
INTEGRATOR_DP45 = 0
INTEGRATOR_SYMPLECTIC = 1
CAMERA_PINHOLE = 0
CAMERA_EQUIRECTANGULAR = 1
OBSERVER_STATIC = 0  # enum sirius_observer
OBSERVER_ZAMO = 1

FLAG_NUMERICAL_FAILURE = 1
FLAG_PHOTON_RING = 2


class Metric(C.Structure):
    _fields_ = [("family", C.c_int32), ("shape", C.c_int32),
                ("M", C.c_double), ("a", C.c_double), ("Q", C.c_double), ("Lambda", C.c_double),
                ("b0", C.c_double), ("Phi0", C.c_double),
                ("vs", C.c_double), ("sigma", C.c_double), ("R", C.c_double)]


class Camera(C.Structure):
    _fields_ = [("t", C.c_double), ("r", C.c_double), ("theta", C.c_double), ("phi", C.c_double),
                ("yaw", C.c_float), ("pitch", C.c_float), ("roll", C.c_float), ("fov", C.c_float),
                ("width", C.c_int32), ("height", C.c_int32), ("projection", C.c_int32),
                ("observer", C.c_int32)]


class Frame(C.Structure):
    _fields_ = [("metric", Metric), ("camera", Camera), ("disk_inner", C.c_double),
                ("disk_outer", C.c_double), ("ray_offset", C.c_int64),
                ("row_begin", C.c_int32), ("row_count", C.c_int32)]


class CameraRay(C.Structure):
    _fields_ = [("origin", C.c_double * 4), ("direction", C.c_double * 4)]


class TraceConfig(C.Structure):
    _fields_ = [("abs_tolerance", C.c_double), ("rel_tolerance", C.c_double), ("min_step", C.c_double),
                ("max_step", C.c_double), ("initial_step", C.c_double), ("safety_factor", C.c_double),
                ("step_grow_max", C.c_double), ("step_shrink_min", C.c_double),
                ("escape_radius", C.c_double), ("horizon_factor", C.c_double),
                ("max_steps", C.c_int32), ("enable_disk", C.c_int32),
                ("disk_temperature_inner", C.c_double), ("crossing_weight_decay", C.c_double),
                ("enable_volumetric", C.c_int32), ("n_bins", C.c_int32),
                ("nu_min", C.c_double), ("nu_max", C.c_double), ("vol_j0", C.c_double),
                ("vol_alpha_over_j", C.c_double), ("vol_height_ratio", C.c_double),
                ("vol_spectral_index", C.c_double), ("vol_substeps", C.c_int32),
                ("integrator", C.c_int32), ("precision", C.c_int32), ("compat", C.c_int32),
                ("projection_period", C.c_int32), ("spiral_check", C.c_int32),
                ("island_factor", C.c_double), ("critical_band", C.c_double), ("symplectic_step", C.c_double),
                ("symplectic_order", C.c_int32), ("block_size", C.c_int32),
                ("refill_threshold", C.c_int32), ("blocks_per_sm", C.c_int32),
                ("watchdog_ms", C.c_int32), ("samples_per_pixel", C.c_int32), ("max_registers", C.c_int32),
                ("rays_per_thread", C.c_int32), ("reserved", C.c_int32 * 2)]


class RayResult(C.Structure):
    _fields_ = [("outcome", C.c_int32), ("steps", C.c_int32), ("rejected", C.c_int32),
                ("n_crossings", C.c_int32),
                ("final_x", C.c_double * 4), ("final_p", C.c_double * 4), ("final_k", C.c_float * 4),
                ("disk_r", C.c_float * 4), ("disk_phi", C.c_float * 4), ("disk_g", C.c_float * 4),
                ("disk_flux", C.c_float * 4),
                ("equatorial_crossings", C.c_int32), ("image_order", C.c_int32),
                ("total_phi_change", C.c_float), ("min_radius", C.c_float), ("intensity", C.c_float),
                ("fp64_steps", C.c_int32),
                ("E", C.c_double), ("Lz", C.c_double), ("Carter", C.c_double),
                ("E0", C.c_double), ("Lz0", C.c_double), ("Carter0", C.c_double),
                ("null_drift_max", C.c_float), ("null_final", C.c_float),
                ("impact_parameter", C.c_float), ("magnification", C.c_float), ("optical_depth", C.c_float),
                ("flags", C.c_int32)]


class LaunchStats(C.Structure):
    _fields_ = [("kernel_ms", C.c_double), ("total_ms", C.c_double), ("rays", C.c_int64),
                ("accepted_steps", C.c_int64), ("rejected_steps", C.c_int64), ("fp64_steps", C.c_int64),
                ("kernel_launches", C.c_int32), ("grid_blocks", C.c_int32), ("block_size", C.c_int32),
                ("status_flags", C.c_int32)]


class SurrogateConfig(C.Structure):
    _fields_ = [("gate_band", C.c_double), ("audit_fraction", C.c_double), ("audit_seed", C.c_uint32),
                ("inner_gate", C.c_float), ("coarse_stride", C.c_int32), ("audit_budget", C.c_float),
                ("empty_skip", C.c_int32), ("reserved", C.c_int32)]


class SurrogateStats(C.Structure):
    _fields_ = [("rays", C.c_int64), ("integrated", C.c_int64), ("ms_features", C.c_float), ("ms_mlp", C.c_float),
                ("ms_shade", C.c_float), ("ms_trace", C.c_float), ("ms_total", C.c_float),
                ("audit_count", C.c_int32), ("audit_rel_l1", C.c_float), ("audit_rel_max", C.c_float),
                ("rerendered", C.c_int32), ("coarse_rays", C.c_int32)]


def surrogate_config(gate_band=0.3, audit_fraction=0.01, audit_seed=0, inner_gate=0.0, coarse_stride=0,
                     audit_budget=0.0, empty_skip=0):
    """sirius_surrogate_config (inner_gate 0: 2.75 r_in, < 0: off; coarse_stride 0: 8; audit_budget 0: report
    only; empty_skip 0: on, < 0: off)."""
    return SurrogateConfig(gate_band, audit_fraction, audit_seed, inner_gate, coarse_stride, audit_budget, empty_skip)


class BeamResult(C.Structure):
    _fields_ = [("outcome", C.c_int32), ("steps", C.c_int32), ("magnification", C.c_float), ("parity", C.c_float),
                ("final_dir", C.c_float * 3), ("reserved", C.c_int32)]


class TrainConfig(C.Structure):
    _fields_ = [("batch", C.c_int32), ("reserved0", C.c_int32), ("total_steps", C.c_int64), ("max_lr", C.c_float),
                ("warmup_fraction", C.c_float), ("beta1", C.c_float), ("beta2", C.c_float), ("eps", C.c_float),
                ("weight_decay", C.c_float), ("seed", C.c_uint32), ("reserved", C.c_int32 * 5)]


def train_config(batch=16384, total_steps=1, max_lr=2e-3, warmup_fraction=0.05, beta1=0.9, beta2=0.999, eps=1e-8,
                 weight_decay=0.0, seed=0):
    """sirius_train_config (the library's defaults unless given)."""
    return TrainConfig(batch, 0, total_steps, max_lr, warmup_fraction, beta1, beta2, eps, weight_decay, seed)


# numpy structured dtype of RayResult (for zero-copy views of result arrays)
def result_dtype():
    import numpy as np
    fields = []
    for name, ctype in RayResult._fields_:
        n = getattr(ctype, "_length_", None)
        base = ctype._type_ if n else ctype
        np_t = {C.c_int32: np.int32, C.c_float: np.float32, C.c_double: np.float64}[base]
        fields.append((name, np_t, (n,)) if n else (name, np_t))
    dt = np.dtype(fields, align=True)
    assert dt.itemsize == C.sizeof(RayResult), (dt.itemsize, C.sizeof(RayResult))
    return dt


def default_config(**overrides):
    """RenderSession's tracer settings (SNRS001A.cpp:103-129) and the engine defaults."""
    c = TraceConfig()
    c.abs_tolerance = 5e-6
    c.rel_tolerance = 5e-6
    c.min_step = 1e-5
    c.max_step = 2.0
    c.initial_step = 0.1
    c.safety_factor = 0.9
    c.step_grow_max = 2.0
    c.step_shrink_min = 0.1
    c.escape_radius = 200.0
    c.horizon_factor = 1.05
    c.max_steps = 20000
    c.enable_disk = 1
    c.disk_temperature_inner = 1.0
    c.crossing_weight_decay = 3.141592653589793
    c.enable_volumetric = 0
    c.n_bins = 0
    c.nu_min = 1e-2
    c.nu_max = 1e2
    c.vol_j0 = 1.0
    c.vol_alpha_over_j = 0.1
    c.vol_height_ratio = 0.1
    c.vol_spectral_index = 0.7
    c.vol_substeps = 4
    c.integrator = INTEGRATOR_DP45
    c.precision = PRECISION_FP64
    c.compat = 0
    c.projection_period = 1
    c.spiral_check = 0
    c.island_factor = 1.5
    c.critical_band = 0.05
    c.symplectic_step = 0.01
    c.symplectic_order = 4
    c.block_size = 0
    c.refill_threshold = 0
    c.blocks_per_sm = 0
    c.watchdog_ms = 30000
    for k, v in overrides.items():
        setattr(c, k, v)
    return c


def make_metric(family=KERR_SCHILD, M=1.0, a=0.0, Q=0.0, Lambda=0.0, b0=1.0, Phi0=0.0, vs=0.5, sigma=8.0,
                R=1.0, shape=0):
    return Metric(family, shape, M, a, Q, Lambda, b0, Phi0, vs, sigma, R)


def make_camera(r=50.0, theta_deg=85.0, phi=0.0, fov=30.0, width=256, height=256, projection=CAMERA_PINHOLE,
                yaw=0.0, pitch=0.0, roll=0.0, observer=0):
    import math
    return Camera(0.0, r, math.radians(theta_deg), phi, yaw, pitch, roll, fov, width, height, projection, observer)


def make_frame(metric, camera, disk_inner=0.0, disk_outer=20.0, ray_offset=0, row_begin=0, row_count=0):
    return Frame(metric, camera, disk_inner, disk_outer, ray_offset, row_begin, row_count)


def frame_rays(frame):
    """Rays of a frame: width x its row window (row_count 0: every row)."""
    rows = frame.camera.height if frame.row_count <= 0 else frame.row_count
    return frame.camera.width * rows

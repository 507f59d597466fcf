"""Python loader for the CPU checker libraries.

TEST INFRASTRUCTURE ONLY — imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, as the checker; never by the product package.

  Oracle     liboracle.so: the CPU restatement of the path (oracle.hpp)
  Reference  _ref/libsirius_ref.so: the reference's own CPU tracer, compiled
             from its sources by oracle/Makefile (absent if never built)
"""
import ctypes as C
import os

import numpy as np

from sirius_b200 import abi

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libsirius_ref.so")

_P = C.POINTER


class Oracle:
    def __init__(self, path=ORACLE_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle`")
        L = self.lib = C.CDLL(path)
        L.oracle_trace_frame.argtypes = [_P(abi.Frame), _P(abi.TraceConfig), C.c_int64, C.c_int64,
                                         C.c_void_p, C.c_void_p, C.c_int, C.c_int]
        L.oracle_trace_rays.argtypes = [_P(abi.Metric), C.c_double, C.c_double, _P(abi.TraceConfig),
                                        C.c_void_p, C.c_int64, C.c_void_p, C.c_int]
        L.oracle_camera_ray.argtypes = [_P(abi.Camera), C.c_int, C.c_int, C.c_void_p, C.c_void_p]
        L.oracle_camera_ray_uv.argtypes = [_P(abi.Camera), C.c_int, C.c_int, C.c_float, C.c_float, C.c_void_p,
                                           C.c_void_p]
        L.oracle_camera_ray_exact.argtypes = [_P(abi.Camera), C.c_double, C.c_double, C.c_void_p, C.c_void_p]
        L.oracle_metric_evaluate.argtypes = [_P(abi.Metric), C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p]
        L.oracle_invert4x4.argtypes = [C.c_void_p, C.c_void_p]
        L.oracle_rhs.argtypes = [_P(abi.Metric), C.c_void_p, C.c_int64, C.c_void_p, C.c_int]
        L.oracle_dp45_step.argtypes = [_P(abi.Metric), _P(abi.TraceConfig), C.c_void_p, C.c_void_p,
                                       C.c_void_p, C.c_void_p, C.c_int64]
        L.oracle_project_null.argtypes = [_P(abi.Metric), C.c_void_p, C.c_void_p]
        L.oracle_project_null.restype = C.c_double
        L.oracle_null_value.argtypes = [_P(abi.Metric), C.c_void_p, C.c_void_p]
        L.oracle_null_value.restype = C.c_double
        L.oracle_invariants.argtypes = [_P(abi.Metric), C.c_void_p, C.c_void_p, C.c_void_p]
        L.oracle_radial.argtypes = [_P(abi.Metric), C.c_void_p, C.c_void_p]
        L.oracle_radial.restype = C.c_double
        for fn in ("oracle_isco",):
            getattr(L, fn).argtypes = [C.c_double]
            getattr(L, fn).restype = C.c_double
        L.oracle_r_photon.argtypes = [C.c_double, C.c_double, C.c_int]
        L.oracle_r_photon.restype = C.c_double
        L.oracle_r_plus.argtypes = [_P(abi.Metric)]
        L.oracle_r_plus.restype = C.c_double
        L.oracle_nt_flux.argtypes = [C.c_double] * 4
        L.oracle_nt_flux.restype = C.c_double
        L.oracle_init_state.argtypes = [_P(abi.Metric), _P(abi.TraceConfig), C.c_void_p, C.c_void_p,
                                        C.c_void_p, C.c_void_p, C.c_void_p]
        L.oracle_rk45_step_compat.argtypes = [_P(abi.Metric), _P(abi.TraceConfig), C.c_void_p, C.c_void_p,
                                              C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64]
        assert L.oracle_sizeof_result() == C.sizeof(abi.RayResult)
        assert L.oracle_sizeof_config() == C.sizeof(abi.TraceConfig)
        assert L.oracle_sizeof_frame() == C.sizeof(abi.Frame)

    def trace_frame(self, frame, cfg, first=0, count=None, threads=1, long_double=False):
        if count is None:
            count = abi.frame_rays(frame) - first
        out = np.zeros(count, dtype=abi.result_dtype())
        nb = max(cfg.n_bins, 0)
        bins = np.zeros((count, max(nb, 1)), dtype=np.float64)
        rc = self.lib.oracle_trace_frame(C.byref(frame), C.byref(cfg), first, count, out.ctypes.data,
                                         bins.ctypes.data if nb else None, threads, 1 if long_double else 0)
        assert rc == 0
        return out, bins[:, :nb]

    def trace_rays(self, metric, rays, cfg, disk_inner=0.0, disk_outer=20.0, threads=1):
        n = len(rays)
        arr = (abi.CameraRay * n)(*rays)
        out = np.zeros(n, dtype=abi.result_dtype())
        rc = self.lib.oracle_trace_rays(C.byref(metric), disk_inner, disk_outer, C.byref(cfg),
                                        C.addressof(arr), n, out.ctypes.data, threads)
        assert rc == 0
        return out

    def camera_ray(self, cam, px, py, u=0.5, v=0.5):
        o = np.zeros(4)
        d = np.zeros(4)
        self.lib.oracle_camera_ray_uv(C.byref(cam), px, py, C.c_float(u), C.c_float(v), o.ctypes.data,
                                      d.ctypes.data)
        return o, d

    def camera_ray_exact(self, cam, u, v):
        """The camera mapping in FP64 at fractional pixel position (u, v)."""
        o = np.zeros(4)
        d = np.zeros(4)
        self.lib.oracle_camera_ray_exact(C.byref(cam), u, v, o.ctypes.data, d.ctypes.data)
        return o, d

    def metric_evaluate(self, metric, pos):
        pos = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1, 4)
        n = len(pos)
        g = np.zeros((n, 4, 4))
        dg = np.zeros((n, 4, 4, 4))
        self.lib.oracle_metric_evaluate(C.byref(metric), pos.ctypes.data, n, g.ctypes.data, dg.ctypes.data)
        return g, dg

    def invert(self, m):
        m = np.ascontiguousarray(m, dtype=np.float64)
        out = np.zeros((4, 4))
        self.lib.oracle_invert4x4(m.ctypes.data, out.ctypes.data)
        return out

    def rhs(self, metric, state, compat=False):
        s = np.ascontiguousarray(state, dtype=np.float64).reshape(-1, 8)
        out = np.zeros_like(s)
        self.lib.oracle_rhs(C.byref(metric), s.ctypes.data, len(s), out.ctypes.data, 1 if compat else 0)
        return out

    def dp45_step(self, metric, cfg, state, h):
        s = np.array(state, dtype=np.float64).reshape(-1, 8).copy()
        hh = np.array(h, dtype=np.float64).reshape(-1).copy()
        acc = np.zeros(len(s), dtype=np.int32)
        err = np.zeros(len(s))
        self.lib.oracle_dp45_step(C.byref(metric), C.byref(cfg), s.ctypes.data, hh.ctypes.data,
                                  acc.ctypes.data, err.ctypes.data, len(s))
        return s, hh, acc, err

    def rk45_step_compat(self, metric, cfg, pos, vel, h):
        pos = np.array(pos, dtype=np.float64).reshape(-1, 4).copy()
        vel = np.array(vel, dtype=np.float64).reshape(-1, 4).copy()
        hh = np.array(h, dtype=np.float32).reshape(-1).copy()
        n = len(pos)
        ok = np.zeros(n, dtype=np.int32)
        term = np.zeros(n, dtype=np.int32)
        self.lib.oracle_rk45_step_compat(C.byref(metric), C.byref(cfg), pos.ctypes.data, vel.ctypes.data,
                                         hh.ctypes.data, ok.ctypes.data, term.ctypes.data, n)
        return pos, vel, hh, ok, term

    def project_null(self, metric, x, p):
        x = np.ascontiguousarray(x, dtype=np.float64)
        p = np.array(p, dtype=np.float64).copy()
        before = self.lib.oracle_project_null(C.byref(metric), x.ctypes.data, p.ctypes.data)
        return before, p

    def null_value(self, metric, x, p):
        x = np.ascontiguousarray(x, dtype=np.float64)
        p = np.ascontiguousarray(p, dtype=np.float64)
        return self.lib.oracle_null_value(C.byref(metric), x.ctypes.data, p.ctypes.data)

    def invariants(self, metric, x, p):
        x = np.ascontiguousarray(x, dtype=np.float64)
        p = np.ascontiguousarray(p, dtype=np.float64)
        out = np.zeros(3)
        self.lib.oracle_invariants(C.byref(metric), x.ctypes.data, p.ctypes.data, out.ctypes.data)
        return out

    def radial(self, metric, x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        g = np.zeros(4)
        r = self.lib.oracle_radial(C.byref(metric), x.ctypes.data, g.ctypes.data)
        return r, g

    def init_state(self, metric, cfg, origin, direction):
        o = np.ascontiguousarray(origin, dtype=np.float64)
        d = np.ascontiguousarray(direction, dtype=np.float64)
        x, p, k = np.zeros(4), np.zeros(4), np.zeros(4)
        self.lib.oracle_init_state(C.byref(metric), C.byref(cfg), o.ctypes.data, d.ctypes.data,
                                   x.ctypes.data, p.ctypes.data, k.ctypes.data)
        return x, p, k

    def isco(self, a_star):
        return self.lib.oracle_isco(a_star)

    def r_photon(self, M, a, prograde=True):
        return self.lib.oracle_r_photon(M, a, 1 if prograde else 0)

    def r_plus(self, metric):
        return self.lib.oracle_r_plus(C.byref(metric))

    def nt_flux(self, r, a_star, r_in, r_out):
        return self.lib.oracle_nt_flux(r, a_star, r_in, r_out)


# ---------------------------------------------------------------------------
class RefTracerConfig(C.Structure):
    _fields_ = [("escape_radius", C.c_float), ("horizon_factor", C.c_float), ("max_steps", C.c_int32),
                ("enable_disk", C.c_int32), ("disk_inner", C.c_float), ("disk_outer", C.c_float),
                ("disk_temperature_inner", C.c_float), ("enable_volumetric", C.c_int32),
                ("abs_tolerance", C.c_float), ("rel_tolerance", C.c_float), ("min_step", C.c_float),
                ("max_step", C.c_float), ("initial_step", C.c_float), ("safety_factor", C.c_float),
                ("step_grow_max", C.c_float), ("step_shrink_min", C.c_float)]


REF_RECORD = np.dtype([("outcome", np.int32), ("steps_taken", np.int32), ("numerical_failure", np.int32),
                       ("num_disk_crossings", np.int32), ("final_position", np.float64, (4,)),
                       ("final_direction", np.float64, (4,)), ("disk_r", np.float32, (4,)),
                       ("disk_phi", np.float32, (4,)), ("disk_redshift", np.float32, (4,)),
                       ("disk_temperature", np.float32, (4,)), ("equatorial_crossings", np.int32),
                       ("image_order", np.int32), ("total_phi_change", np.float32),
                       ("min_radius", np.float32), ("redshift", np.float32), ("magnification", np.float32),
                       ("impact_parameter", np.float32), ("optical_depth", np.float32),
                       ("volumetric_emission", np.float32), ("photon_ring", np.int32)], align=True)


def ref_config_from(cfg, disk_inner, disk_outer):
    """The reference TracerConfig equivalent of an engine TraceConfig."""
    return RefTracerConfig(cfg.escape_radius, cfg.horizon_factor, cfg.max_steps, cfg.enable_disk, disk_inner,
                           disk_outer, cfg.disk_temperature_inner, cfg.enable_volumetric, cfg.abs_tolerance,
                           cfg.rel_tolerance, cfg.min_step, cfg.max_step, cfg.initial_step, cfg.safety_factor,
                           cfg.step_grow_max, cfg.step_shrink_min)


def ref_available(path=REF_SO):
    return os.path.exists(path)


class Reference:
    def __init__(self, path=REF_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle ref` where the reference sources exist")
        L = self.lib = C.CDLL(path)
        assert L.ref_sizeof_record() == REF_RECORD.itemsize, (L.ref_sizeof_record(), REF_RECORD.itemsize)
        L.ref_ks_evaluate.argtypes = [C.c_double] * 4 + [C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p]
        L.ref_camera_rays.argtypes = [C.c_double, C.c_double, C.c_double, C.c_float, C.c_int, C.c_int,
                                      C.c_float, C.c_float, C.c_float, C.c_void_p, C.c_void_p, C.c_int64,
                                      C.c_void_p, C.c_void_p]
        L.ref_camera_rays_uv.argtypes = [C.c_double, C.c_double, C.c_double, C.c_float, C.c_int, C.c_int,
                                         C.c_float, C.c_float, C.c_float, C.c_void_p, C.c_void_p, C.c_void_p,
                                         C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p]
        L.ref_rk45_step.argtypes = [C.c_double, C.c_double, _P(RefTracerConfig), C.c_void_p, C.c_void_p,
                                    C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64]
        L.ref_trace_rays.argtypes = [C.c_double, C.c_double, _P(RefTracerConfig), C.c_void_p, C.c_void_p,
                                     C.c_int64, C.c_void_p, C.c_int]
        L.ref_trace_frame.argtypes = [C.c_double, C.c_double, _P(RefTracerConfig), C.c_double, C.c_double,
                                      C.c_double, C.c_float, C.c_int, C.c_int, C.c_int64, C.c_int64,
                                      C.c_void_p, C.c_int]
        L.ref_isco.argtypes = [C.c_double]
        L.ref_isco.restype = C.c_double
        L.ref_nt_flux_q.argtypes = [C.c_double, C.c_double]
        L.ref_nt_flux_q.restype = C.c_double

    def ks_evaluate(self, M, a, Q, Lam, pos):
        pos = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1, 4)
        n = len(pos)
        g = np.zeros((n, 4, 4))
        dg = np.zeros((n, 4, 4, 4))
        self.lib.ref_ks_evaluate(M, a, Q, Lam, pos.ctypes.data, n, g.ctypes.data, dg.ctypes.data)
        return g, dg

    def camera_rays(self, cam, px, py):
        px = np.ascontiguousarray(px, dtype=np.int32)
        py = np.ascontiguousarray(py, dtype=np.int32)
        n = len(px)
        o = np.zeros((n, 4))
        d = np.zeros((n, 4))
        self.lib.ref_camera_rays(cam.r, cam.theta, cam.phi, cam.fov, cam.width, cam.height, cam.yaw, cam.pitch,
                                 cam.roll, px.ctypes.data, py.ctypes.data, n, o.ctypes.data, d.ctypes.data)
        return o, d

    def camera_rays_uv(self, cam, px, py, u, v):
        px = np.ascontiguousarray(px, dtype=np.int32)
        py = np.ascontiguousarray(py, dtype=np.int32)
        u = np.ascontiguousarray(u, dtype=np.float32)
        v = np.ascontiguousarray(v, dtype=np.float32)
        n = len(px)
        o = np.zeros((n, 4))
        d = np.zeros((n, 4))
        self.lib.ref_camera_rays_uv(cam.r, cam.theta, cam.phi, cam.fov, cam.width, cam.height, cam.yaw, cam.pitch,
                                    cam.roll, px.ctypes.data, py.ctypes.data, u.ctypes.data, v.ctypes.data, n,
                                    o.ctypes.data, d.ctypes.data)
        return o, d

    def rk45_step(self, M, a, rcfg, pos, vel, h):
        pos = np.array(pos, dtype=np.float64).reshape(-1, 4).copy()
        vel = np.array(vel, dtype=np.float64).reshape(-1, 4).copy()
        hh = np.array(h, dtype=np.float32).reshape(-1).copy()
        n = len(pos)
        ok = np.zeros(n, dtype=np.int32)
        term = np.zeros(n, dtype=np.int32)
        self.lib.ref_rk45_step(M, a, C.byref(rcfg), pos.ctypes.data, vel.ctypes.data, hh.ctypes.data,
                               ok.ctypes.data, term.ctypes.data, n)
        return pos, vel, hh, ok, term

    def trace_rays(self, M, a, rcfg, origins, dirs, threads=1):
        o = np.ascontiguousarray(origins, dtype=np.float64).reshape(-1, 4)
        d = np.ascontiguousarray(dirs, dtype=np.float64).reshape(-1, 4)
        out = np.zeros(len(o), dtype=REF_RECORD)
        self.lib.ref_trace_rays(M, a, C.byref(rcfg), o.ctypes.data, d.ctypes.data, len(o), out.ctypes.data,
                                threads)
        return out

    def trace_frame(self, M, a, rcfg, cam, first=0, count=None, threads=1, keep=True):
        if count is None:
            count = cam.width * cam.height - first
        out = np.zeros(count, dtype=REF_RECORD) if keep else None
        self.lib.ref_trace_frame(M, a, C.byref(rcfg), cam.r, cam.theta, cam.phi, cam.fov, cam.width, cam.height,
                                 first, count, out.ctypes.data if keep else None, threads)
        return out

    def isco(self, a_star):
        return self.lib.ref_isco(a_star)

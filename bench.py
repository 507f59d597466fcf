"""Benchmark: Mrays/s of the geodesic engine on the Kerr a = 0.9, 1024^2 workload.

Workload (one "step" = one full frame traced):
  Kerr a = 0.9, M = 1, 1024 x 1024 pinhole camera at r_obs = 100 M, FOV 30 deg,
  inclination drawn from U[10, 89] deg with a recorded seed; mixed precision
  (FP32 dual-number RHS, FP64 state, FP64 constraint re-projection every step,
  FP64 RHS + error control inside 1.5 r_ph(retrograde) and 2 r_+); DP45 at
  rtol = atol = 1e-8, h in [1e-9, 2], escape at R > 200 M (RenderSession's),
  horizon at r < 1.01 r_+; Novikov-Thorne disk r_in = r_ISCO, r_out = 30 M plus
  volumetric transfer over 16 log-spaced frequency bins.
The reference arm (--impl reference) runs the reference's own CPU tracer
(oracle/_ref, GeodesicTracer) on a bounded pixel sample of the same frame with
all host threads.

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
Under torchrun the frame is split into contiguous row blocks, one per rank (each
rank traces its block's row window); every step ends with the gather of the image
rows to rank 0, the one exchange of a split frame (strong scaling: value = the
frame's rays over the slowest rank's device time).
"""
import argparse
import ctypes as C
import json
import math
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WIDTH = HEIGHT = 1024
SEED = 0
N_BINS = 16
MEASURED_PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")
# DRAM bytes (read + write) per ray of the trace kernel, from one ncu capture of
# the 512^2 case of this workload (profiles/trace_kernel_mixed_kerr512_full.md):
# (4.01 + 1.49) MB / 262,144 rays; traffic grows with the ray count.
TRAFFIC_BYTES_PER_RAY = 21.0


def inclination_deg(seed=SEED):
    import numpy as np
    return float(np.random.default_rng(seed).uniform(10.0, 89.0))


def workload_config(abi, precision):
    return abi.default_config(abs_tolerance=1e-8, rel_tolerance=1e-8, min_step=1e-9, max_step=2.0, initial_step=0.1,
                              escape_radius=200.0, horizon_factor=1.01, max_steps=10000, precision=precision,
                              enable_volumetric=1, n_bins=N_BINS, nu_min=1e-2, nu_max=1e2, vol_spectral_index=0.7,
                              vol_substeps=4, projection_period=1, island_factor=1.5)


def workload_frame(abi, width=WIDTH, height=HEIGHT):
    cam = abi.make_camera(r=100.0, theta_deg=inclination_deg(), fov=30.0, width=width, height=height)
    return abi.make_frame(abi.make_metric(M=1.0, a=0.9), cam, 0.0, 30.0)


def workload_desc(size=WIDTH):
    return {"workload": f"kerr_a0.9_{size}x{size}_mixed_dp45_nt_disk_vol16", "metric_family": "kerr_schild",
            "spin": 0.9, "resolution": [size, size], "r_obs": 100.0, "inclination_deg": round(inclination_deg(), 4),
            "seed": SEED, "fov_deg": 30.0, "tolerance": 1e-8, "escape_radius": 200.0, "horizon_factor": 1.01,
            "disk": [None, 30.0], "volumetric_bins": N_BINS, "precision": "fp32 rhs + fp64 state/projection/island",
            "l2": "inputs are 168-byte frame descriptors; the outputs (4 B image + 64 B spectra per ray) are "
                  "written once per ray; a 256 MiB write flushes the 126 MB L2 between timed steps"}


# --------------------------------------------------------------- clocks ----
class ClockSampler:
    """nvidia-smi samples during the timed region (SM clock, throttle reasons)."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        sm.sort()
        return {"sm_mhz": sm[len(sm) // 2] if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# -------------------------------------------------------------- reference --
def run_reference(args):
    """The reference's own CPU tracer on a bounded strided pixel sample of the frame."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle.pyoracle import Oracle, Reference, ref_available, ref_config_from
    from sirius_b200 import abi
    cfg = workload_config(abi, abi.PRECISION_FP64)
    fr = workload_frame(abi)
    threads = os.cpu_count() or 1
    kind = "reference" if ref_available() else "port"
    if kind == "reference":
        ref = Reference()
        # the reference's TracerConfig: thin disk (it cannot run its volumetric march together with the disk)
        rcfg = ref_config_from(cfg, float(Oracle().isco(0.9)), 30.0)
        rcfg.enable_volumetric = 0

    # calibrate a sample that takes ~4 s per step
    npix = WIDTH * HEIGHT

    def run_sample(n):
        stride = max(npix // n, 1)
        t0 = time.perf_counter()
        recs = []
        if kind == "reference":
            # rows sampled with a stride; each call traces a contiguous block of one row
            rows = max(n // WIDTH, 1)
            row_stride = max(HEIGHT // rows, 1)
            for r in range(rows):
                recs.append(ref.trace_frame(1.0, 0.9, rcfg, fr.camera, (r * row_stride) * WIDTH, WIDTH,
                                            threads=threads))
            n_done = rows * WIDTH
        else:
            orc = Oracle()
            rows = max(n // WIDTH, 1)
            row_stride = max(HEIGHT // rows, 1)
            for r in range(rows):
                recs.append(orc.trace_frame(fr, cfg, (r * row_stride) * WIDTH, WIDTH, threads=threads)[0])
            n_done = rows * WIDTH
        return time.perf_counter() - t0, n_done, recs

    dt, n, _ = run_sample(WIDTH)
    rate = n / dt
    n_step = int(min(max(rate * 4.0, WIDTH), npix))
    times, counts, recs = [], [], []
    for i in range(args.warmup + args.steps):
        dt, n, rr = run_sample(n_step)
        if i >= args.warmup:
            times.append(dt)
            counts.append(n)
            recs += rr
    import numpy as np
    allrec = np.concatenate(recs)
    steps_field = "steps_taken" if kind == "reference" else "steps"
    value = sum(counts) / sum(times) / 1e6
    sample = (f"{counts[0]} pixels per step ({counts[0] // WIDTH} full rows evenly spaced over the 1024^2 frame), "
              f"RenderSession-style atomic pixel queue, {threads} threads, the reference's TracerConfig with the "
              f"workload's tolerances (thin disk; its gray volumetric march replaces the disk, so it is off)")
    line = {"metric": "Mrays/s", "value": value, "unit": "Mrays/s", "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * sum(times) / len(times),
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded camera frame)", "config": workload_desc(),
            "cpu_baseline": {"value": value, "unit": "Mrays/s", "cores": threads, "kind": kind, "sample": sample,
                             "cpu_model": cpu_model(), "steps_per_ray": float(allrec[steps_field].mean()),
                             "outcome_mix": outcome_mix(allrec["outcome"], {0: "escaped", 1: "horizon", 2: "disk",
                                                                            3: "max_steps", 4: "spiraling"})},
            "e2e": {"value": value, "unit": "Mrays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# -------------------------------------------------------------------- ours --
def cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for ln in f:
                if ln.startswith("model name"):
                    return ln.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def outcome_mix(outcomes, names):
    """Counts of each outcome (names: value -> label)."""
    import numpy as np
    vals, counts = np.unique(np.asarray(outcomes), return_counts=True)
    return {names.get(int(v), str(int(v))): int(c) for v, c in zip(vals, counts)}


SAMPLE_ROWS = [(i * 97) % HEIGHT for i in range(HEIGHT)]  # rows spread over the frame, in sampling order


def cpu_baseline_sample(gpu_res, gpu_img, gpu_spc, seconds=12.0):
    """The two CPU numbers on the box's host cores (rank 0, N = 1), each on whole
    rows of the 1024^2 frame spread over its height for about `seconds`:
      reference  the reference's own tracer (oracle/_ref, GeodesicTracer) in
                 RenderSession's pattern; thin disk (its gray volumetric march
                 replaces the disk), stop-on-reject as written;
      oracle     the FP64 restatement in engine semantics (retry on reject, the
                 full workload: NT disk and 16-bin volumetric transfer).
    The oracle's rows also judge the GPU frame (gpu_res, gpu_img, gpu_spc: the
    mixed-precision trace of the full frame): error_vs_oracle, max and p99 of every
    output over those rows (oracle/compare.py)."""
    import numpy as np

    from oracle import compare
    from oracle.pyoracle import Oracle, Reference, ref_available, ref_config_from
    from sirius_b200 import abi
    cfg = workload_config(abi, abi.PRECISION_FP64)
    fr = workload_frame(abi)
    threads = os.cpu_count() or 1
    names = {abi.ESCAPED: "escaped", abi.HORIZON: "horizon", abi.DISK_HIT: "disk", abi.MAX_STEPS: "max_steps",
             abi.SPIRALING: "spiraling", abi.NUMERICAL_FAILURE: "numerical_failure",
             abi.STEP_UNDERFLOW: "step_underflow"}
    out = {}
    orc = Oracle()
    if ref_available():
        ref = Reference()
        rcfg = ref_config_from(cfg, float(orc.isco(0.9)), 30.0)
        rcfg.enable_volumetric = 0
        recs, rows = [], 0
        t0 = time.perf_counter()
        while time.perf_counter() - t0 < seconds and rows < HEIGHT:
            recs.append(ref.trace_frame(1.0, 0.9, rcfg, fr.camera, SAMPLE_ROWS[rows] * WIDTH, WIDTH, threads=threads))
            rows += 1
        dt = time.perf_counter() - t0
        r = np.concatenate(recs)
        out["cpu_baseline"] = {
            "value": rows * WIDTH / dt / 1e6, "unit": "Mrays/s", "cores": threads, "kind": "reference",
            "cpu_model": cpu_model(), "steps_per_ray": float(r["steps_taken"].mean()),
            "outcome_mix": outcome_mix(r["outcome"], {0: "escaped", 1: "horizon", 2: "disk", 3: "max_steps",
                                                      4: "spiraling"}),
            "sample": f"{rows} full rows ({rows * WIDTH} rays) of the 1024^2 frame spread over its height, {dt:.1f} s, "
                      f"RenderSession-style pixel queue over {threads} threads; thin disk only (the reference's gray "
                      f"volumetric march replaces its disk); a rejected step ends a ray as MAX_STEPS "
                      f"(GTRC001A.cpp:272-277), so max_steps counts the rays stop-on-reject cut short"}
    res_o, bins_o, rows_o = [], [], []
    t0 = time.perf_counter()
    while time.perf_counter() - t0 < seconds and len(rows_o) < HEIGHT:
        row = SAMPLE_ROWS[len(rows_o)]
        a, b = orc.trace_frame(fr, cfg, row * WIDTH, WIDTH, threads=threads)
        res_o.append(a)
        bins_o.append(b)
        rows_o.append(row)
    dt = time.perf_counter() - t0
    ro = np.concatenate(res_o)
    bo = np.concatenate(bins_o)
    oracle_line = {"value": len(rows_o) * WIDTH / dt / 1e6, "unit": "Mrays/s", "cores": threads, "kind": "port",
                   "cpu_model": cpu_model(), "steps_per_ray": float(ro["steps"].mean()),
                   "rejected_per_ray": float(ro["rejected"].mean()), "outcome_mix": outcome_mix(ro["outcome"], names),
                   "sample": f"{len(rows_o)} full rows ({len(rows_o) * WIDTH} rays) of the 1024^2 frame, {dt:.1f} s, "
                             f"atomic pixel queue over {threads} threads; the full workload (NT disk + 16-bin "
                             f"volumetric), engine semantics (retry on reject)"}
    if "cpu_baseline" not in out:
        out["cpu_baseline"] = oracle_line
    else:
        out["cpu_baseline_oracle"] = oracle_line
    idx = np.concatenate([np.arange(r * WIDTH, (r + 1) * WIDTH) for r in rows_o])
    rep = compare.report(gpu_res[idx], gpu_img[idx], ro, gpu_spc[idx], bo, escape_radius=200.0)
    rep["rows"] = len(rows_o)
    rep["note"] = ("mixed-precision GPU frame against the FP64 oracle on the oracle's sampled rows; image errors "
                   "relative to the sample's peak, spectra per bin; maxima over the rays whose histories agree "
                   "(split_histories counts the others)")
    out["error_vs_oracle"] = rep
    return out


def batch_frames(abi, seed=3, n=96):
    """The heterogeneous batch: 96 seeded frames, metric family uniform over
    Kerr-Newman (a ~ U[0, 0.998], Q ~ U[0, sqrt(1 - a^2)]), Kerr-de Sitter
    (Lambda ~ LogU[1e-6, 1e-3]), Morris-Thorne (b0 ~ U[0.5, 2]) and Alcubierre
    (v_s ~ U[0.1, 2], sigma = 8, R = 1); square side ~ U{128..1024},
    r_obs ~ U[20, 200], inclination ~ U[10, 89] deg."""
    import numpy as np
    rng = np.random.default_rng(seed)
    frames = []
    for _ in range(n):
        kind = rng.integers(4)
        side = int(rng.integers(128, 1025))
        r = float(rng.uniform(20.0, 200.0))
        th = float(rng.uniform(10.0, 89.0))
        if kind == 0:
            a = float(rng.uniform(0.0, 0.998))
            m = abi.make_metric(a=a, Q=float(rng.uniform(0.0, math.sqrt(1.0 - a * a))))
        elif kind == 1:
            m = abi.make_metric(a=float(rng.uniform(0.0, 0.998)), Lambda=float(10 ** rng.uniform(-6.0, -3.0)))
        elif kind == 2:
            m = abi.make_metric(family=abi.MORRIS_THORNE, b0=float(rng.uniform(0.5, 2.0)))
        else:
            m = abi.make_metric(family=abi.ALCUBIERRE, vs=float(rng.uniform(0.1, 2.0)), sigma=8.0, R=1.0)
        cam = abi.make_camera(r=r, theta_deg=th, width=side, height=side, fov=30.0)
        frames.append(abi.make_frame(m, cam, 0.0, 30.0))
    return frames


def batch_leg(eng, abi, rank=0, world=1, dist=None, dev=None):
    """All 96 frames in one launch (persistent queue, generic kernel) and as
    per-family launches (one thread per ray), mixed precision, thin disk. Under
    torchrun each rank takes whole frames round robin (shard.frames_for_rank) and
    the device time is the maximum over ranks; every rank runs both variants."""
    from sirius_b200.shard import frames_for_rank, max_over_ranks
    all_frames = batch_frames(abi)
    frames = frames_for_rank(all_frames, rank, world)
    total = sum(f.camera.width * f.camera.height for f in all_frames)
    mine = sum(f.camera.width * f.camera.height for f in frames)
    out = {"workload": "96 seeded frames: Kerr-Newman / Kerr-de Sitter / Morris-Thorne / Alcubierre, "
                       "sides U{128..1024}", "rays": total,
           "split": f"whole frames round robin over {world} rank(s)" if world > 1 else "one GPU"}
    for name, bps in (("persistent_one_launch", -1), ("per_family_launches", 0)):
        cfg = workload_config(abi, abi.PRECISION_MIXED)
        cfg.enable_volumetric = 0
        cfg.blocks_per_sm = bps
        eng.configure(cfg)
        eng.trace_frames(frames, results=False, image=True)
        eng.trace_frames(frames, results=False, image=True)
        st = eng.stats()
        ms = max_over_ranks(st.kernel_ms, dist if world > 1 else None, dev)
        out[name] = {"kernel_ms": ms, "mrays_per_s": total / (ms * 1e-3) / 1e6,
                     "kernel_launches": st.kernel_launches, "steps_per_ray": st.accepted_steps / max(mine, 1)}
    return out


def stress_leg(eng, abi, stride=1):
    """The stress configuration: Kerr-Newman a = 0.998, Q = 0.05, equirectangular
    4096 x 2048 sky map at r_obs = 15, Yoshida-4 symplectic d-lambda = 0.01 with
    FP64 re-projection every 8 steps (<= 50k steps), thin disk + 32-bin volumetric
    transfer: the full map in one launch (stride > 1: every stride-th pixel in
    both directions); its outcome mix from the per-ray records."""
    import numpy as np
    w, h = 4096 // stride, 2048 // stride
    cam = abi.make_camera(r=15.0, theta_deg=80.0, width=w, height=h, projection=abi.CAMERA_EQUIRECTANGULAR)
    frame = abi.make_frame(abi.make_metric(a=0.998, Q=0.05), cam, 0.0, 30.0)
    cfg = abi.default_config(integrator=abi.INTEGRATOR_SYMPLECTIC, symplectic_order=4, symplectic_step=0.01,
                             projection_period=8, max_steps=50000, escape_radius=60.0, horizon_factor=1.01,
                             min_step=1e-9, enable_volumetric=1, n_bins=32, precision=abi.PRECISION_MIXED,
                             watchdog_ms=300000)
    eng.configure(cfg)
    res, _, _ = eng.trace_frames([frame], results=True, image=True, spectra=True)
    st = eng.stats()
    names = {abi.ESCAPED: "escaped", abi.HORIZON: "horizon", abi.DISK_HIT: "disk", abi.MAX_STEPS: "max_steps",
             abi.SPIRALING: "spiraling", abi.NUMERICAL_FAILURE: "numerical_failure"}
    return {"workload": f"kerr_newman_a0.998_q0.05_equirect_{w}x{h}_symplectic4_vol32"
                        + (" (sample of 4096x2048)" if stride > 1 else ""),
            "rays": w * h, "kernel_ms": st.kernel_ms, "mrays_per_s": w * h / (st.kernel_ms * 1e-3) / 1e6,
            "steps_per_ray": st.accepted_steps / (w * h), "max_steps_per_ray": int(res["steps"].max()),
            "outcome_mix": outcome_mix(res["outcome"], names),
            "surrogate_gating": "not applied: the network covers charge-free Kerr frames only (this frame has "
                                "Q = 0.05), so every ray is integrated",
            "parity": "tests/test_gpu_symplectic.py compares a 64 x 32 crop of this configuration with the oracle"}


SURROGATE_SIDE = 2048
SURROGATE_WEIGHTS = os.path.join(ROOT, "sirius_b200", "data", "surrogate_kerr.npy")


def surrogate_config(abi, precision):
    """Surrogate workload: thin NT disk only, no volumetric transfer; the gated
    rays integrate in mixed precision without the FP64 near-critical rule and
    with the FP64 island only inside 2 r_+ (island_factor 0): the surrogate's
    error budget is 1e-3 of the image scale, and the image error of the gated
    pixels against FP64 is the same with and without the wider island (measured
    on the 2048^2 frame), while the gated trace runs 8 % faster."""
    return abi.default_config(abs_tolerance=1e-8, rel_tolerance=1e-8, min_step=1e-9, max_step=2.0,
                              initial_step=0.1, escape_radius=200.0, horizon_factor=1.01, max_steps=10000,
                              precision=precision, enable_disk=1, enable_volumetric=0, critical_band=0.0,
                              island_factor=0.0)


def surrogate_leg(eng, abi, np, torch, dev, stream, side=SURROGATE_SIDE, reps=3, inner_gate=0.0):
    """Surrogate-gated rendering of the Kerr a = 0.9 frame at side^2 (gate +-0.3 M
    around the critical curve, the inner-disk gate r_1 < 2.75 r_in from a coarse
    MLP pass on 8 x 8 pixel cells, 1 % audit rays; pixels whose coarse
    neighbourhood predicts no disk crossing take 0 without the per-pixel MLP)
    against the plain FP64 integrator on the same frame; CUDA events on the launch
    stream around whole calls."""
    params = np.load(SURROGATE_WEIGHTS)
    eng.surrogate_load(params)
    frame = workload_frame(abi, side, side)
    n = side * side
    d_img = torch.empty(n, dtype=torch.float32, device=dev)
    d_gate = torch.empty(n, dtype=torch.uint8, device=dev)
    eng.configure(surrogate_config(abi, abi.PRECISION_FP64))
    fp64_ms = []
    for i in range(2):
        _, img64, _ = eng.trace_frames([frame], results=False)
        fp64_ms.append(eng.stats().kernel_ms)
    eng.configure(surrogate_config(abi, abi.PRECISION_MIXED))
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    sc = abi.surrogate_config(inner_gate=inner_gate)
    for _ in range(2):
        eng.render_surrogate_device([frame], d_img.data_ptr(), None, d_gate.data_ptr(), config=sc,
                                    stream=stream.cuda_stream)
    times, stats = [], None
    for _ in range(reps):
        ev0.record(stream)
        stats = eng.render_surrogate_device([frame], d_img.data_ptr(), None, d_gate.data_ptr(), config=sc,
                                            stream=stream.cuda_stream)
        ev1.record(stream)
        torch.cuda.synchronize()
        times.append(ev0.elapsed_time(ev1))
    ms = float(np.mean(times))
    img = d_img.cpu().numpy().astype(np.float64)
    gate = d_gate.cpu().numpy()
    err = np.abs(img - img64) / img64.max()
    t64 = float(np.min(fp64_ms))
    flops = 2.0 * 198912 * n
    # the MLP kernel alone on the frame's features (in the render it shares the
    # SMs with the gated trace, so its stage time there is not the kernel's)
    d_feat = torch.empty((n, 5), dtype=torch.float32, device=dev)
    d_out = torch.empty((n, 4), dtype=torch.float32, device=dev)
    eng.surrogate_features([frame], d_feat.data_ptr(), stream=stream.cuda_stream)
    for _ in range(2):
        eng.surrogate_infer(d_feat.data_ptr(), n, d_out.data_ptr(), stream.cuda_stream)
    mlp_ms = []
    for _ in range(reps):
        ev0.record(stream)
        eng.surrogate_infer(d_feat.data_ptr(), n, d_out.data_ptr(), stream.cuda_stream)
        ev1.record(stream)
        torch.cuda.synchronize()
        mlp_ms.append(ev0.elapsed_time(ev1))
    mlp_alone = float(np.min(mlp_ms))
    peaks = {}
    if os.path.exists(MEASURED_PEAKS):
        with open(MEASURED_PEAKS) as f:
            peaks = json.load(f)
    bf16_peak = float(peaks.get("bf16_tflops", 1590.0))
    return {"workload": f"kerr_a0.9_{side}x{side}_nt_disk_surrogate_gated", "mrays_per_s": n / (ms * 1e-3) / 1e6,
            "ms_per_frame": ms, "fp64_plain_ms": t64, "speedup_vs_fp64_plain": t64 / ms,
            "gate_band_m": 0.3, "inner_gate_r_in": 2.75 if inner_gate == 0.0 else (None if inner_gate < 0 else inner_gate),
            "coarse_stride": 8, "coarse_mlp_rows": int(stats.coarse_rays),
            "audit_fraction": 0.01, "gated_fraction": float(np.mean(gate == 1)),
            "audit_fraction_measured": float(np.mean(gate == 2)), "integrated_rays": int(stats.integrated),
            "empty_fraction": float(np.mean(gate == 3)),
            "stage_ms": {"features_gate": stats.ms_features, "mlp_end": stats.ms_mlp, "shade": stats.ms_shade,
                         "integrate_gated_and_audit": stats.ms_trace,
                         "note": "after the list is built, the gated trace and the MLP run side by side; mlp_end and "
                                 "integrate_gated_and_audit are measured from that point"},
            "error_vs_fp64": {"image_linf_rel": float(err.max()), "image_p99_rel": float(np.percentile(err, 99)),
                              "image_mean_rel": float(err.mean())},
            "audit_judgement": {"pixels": int(stats.audit_count), "rel_l1": float(stats.audit_rel_l1),
                                "rel_max": float(stats.audit_rel_max)},
            "mlp_roofline": {"bound": "tensor", "kernel_ms": mlp_alone, "achieved": flops / (mlp_alone * 1e-3) / 1e12,
                             "peak": bf16_peak, "unit": "TFLOP/s", "frac": flops / (mlp_alone * 1e-3) / 1e12 / bf16_peak,
                             "peak_source": "MEASURED_PEAKS.json bf16_tflops (burst)" if peaks else "fallback",
                             "timing": "the MLP kernel alone on the frame's features (CUDA events)"},
            "weights": "sirius_b200/data/surrogate_kerr.npy (python -m sirius_b200.surrogate_train)"}


def graph_leg(eng, abi, torch, dev, side=128, reps=50):
    """Small frames, where launch overhead shows: the prepared launch sequence
    (memsets, flux tables, trace kernel) issued call by call vs replayed from a
    captured CUDA graph; CUDA events around `reps` back-to-back frames."""
    eng.configure(workload_config(abi, abi.PRECISION_MIXED))
    fr = workload_frame(abi, side, side)
    total = eng.prepare_frames([fr])
    d_img = torch.empty(total, dtype=torch.float32, device=dev)
    s = torch.cuda.Stream(device=dev)
    s.wait_stream(torch.cuda.current_stream(dev))
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(s):
        for _ in range(3):
            eng.launch_prepared(None, d_img.data_ptr(), None, s.cuda_stream)
        ev0.record(s)
        for _ in range(reps):
            eng.launch_prepared(None, d_img.data_ptr(), None, s.cuda_stream)
        ev1.record(s)
    torch.cuda.synchronize(dev)
    direct = ev0.elapsed_time(ev1) / reps
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        eng.launch_prepared(None, d_img.data_ptr(), None, torch.cuda.current_stream(dev).cuda_stream)
    g.replay()
    torch.cuda.synchronize(dev)
    st = torch.cuda.current_stream(dev)
    ev0.record(st)
    for _ in range(reps):
        g.replay()
    ev1.record(st)
    torch.cuda.synchronize(dev)
    replay = ev0.elapsed_time(ev1) / reps
    del g
    return {"workload": f"kerr_a0.9_{side}x{side}_mixed_prepared", "frames": reps, "ms_per_frame_direct": direct,
            "ms_per_frame_graph": replay}


def beam_leg(eng, abi, side=256):
    """Beams (ray + two tangent vectors, FP64 Dormand-Prince) over the Kerr
    a = 0.9 workload camera at side^2; host-timed call (the call synchronises),
    with the magnification range of the escaped rays."""
    import numpy as np
    cfg = abi.default_config(abs_tolerance=1e-8, rel_tolerance=1e-8, min_step=1e-9, max_step=2.0, initial_step=0.1,
                             escape_radius=1000.0, horizon_factor=1.01, max_steps=20000,
                             precision=abi.PRECISION_FP64, enable_disk=0)
    eng.configure(cfg)
    fr = workload_frame(abi, side, side)
    eng.trace_beams([fr])
    t0 = time.perf_counter()
    b = eng.trace_beams([fr])
    dt = time.perf_counter() - t0
    esc = b["outcome"] == abi.ESCAPED
    return {"workload": f"kerr_a0.9_{side}x{side}_beams_fp64", "rays": int(b.size), "seconds": dt,
            "mbeams_per_s": b.size / dt / 1e6, "escaped": int(esc.sum()),
            "magnification_p50_p99": [float(np.percentile(b["magnification"][esc], 50)),
                                      float(np.percentile(b["magnification"][esc], 99))],
            "negative_parity_fraction": float(np.mean(b["parity"][esc] < 0)), "timing": "host clock around the call"}


TRAIN_FLOP_PER_ROW = 3 * 2 * 198912 - 2 * 5 * 256  # forward, dW and dH (no dH for the input layer)
# Algorithmic HBM bytes per training row of one step, from the kernels' operands:
# gather 92 (features, targets, weight in; the BF16 input row, targets, weight
# out); forward 8,240 (layer 1: input 32, Z 1024 FP32, H 512 BF16; layers 2-4:
# H in 512, Z 1024 and H 512 out; output layer: H 512 in, y 16 out); loss 68;
# backward 11,872 (dW5: H4 512 + dY 32; dH4: dY 32, Z4 1024 in, dZ 512 out;
# layers 4..2: dW 512 + 512, dH 512 + Z 1024 in and dZ 512 out; dW1: 512 + 32);
# Adam 5.6 MB of parameters and moments per step over the batch (171 B/row at
# 32768 rows). Weights are re-read from L2 and not counted.
TRAIN_BYTES_PER_ROW = 92 + 8240 + 68 + 11872 + 171


def train_leg(eng, abi, np, torch, dev, rows=1 << 21, batch=32768, steps=64):
    """The surrogate's training step on the tensor cores (gather, forward and
    backward tcgen05 GEMMs, loss, Adam; one CUDA graph replay per step) over a
    seeded synthetic training set of `rows` device-resident rows with the
    surrogate's feature ranges; CUDA-event time of `steps` replayed steps."""
    rng = np.random.default_rng(0)
    X = rng.uniform(-1.0, 1.0, size=(rows, 5)).astype(np.float32)
    hit = (np.hypot(X[:, 2], X[:, 3]) > 0.35).astype(np.float32)
    T = np.stack([hit, hit * (0.5 * X[:, 2] - 0.2 * X[:, 0]), hit * (0.6 + 0.3 * X[:, 3] * X[:, 1]),
                  0.2 * np.sin(3 * X[:, 2]) * X[:, 4]], 1).astype(np.float32)
    W = rng.uniform(0.05, 1.0, size=rows).astype(np.float32)
    dX, dT, dW = (torch.from_numpy(a).to(dev) for a in (X, T, W))
    params = np.load(SURROGATE_WEIGHTS)
    eng.train_init(params, abi.train_config(batch=batch, total_steps=4 * steps, max_lr=1e-4))
    eng.train_steps(dX.data_ptr(), dT.data_ptr(), dW.data_ptr(), rows, 3)  # capture + warm-up
    ms = eng.train_steps(dX.data_ptr(), dT.data_ptr(), dW.data_ptr(), rows, steps)
    rows_per_s = steps * batch / (ms * 1e-3)
    peaks = {}
    if os.path.exists(MEASURED_PEAKS):
        with open(MEASURED_PEAKS) as f:
            peaks = json.load(f)
    bf16_peak = float(peaks.get("bf16_tflops", 1590.0))
    hbm_peak = float(peaks.get("hbm_gbs", 6650.0))
    tflops = rows_per_s * TRAIN_FLOP_PER_ROW / 1e12
    gbs = rows_per_s * TRAIN_BYTES_PER_ROW / 1e9
    # the step moves 20 KB of activations and gradients per row for 1.19 MFLOP:
    # at the measured peaks the bytes take ~4x the tensor-core time, so HBM is the bound
    return {"workload": f"surrogate_mlp_training_batch{batch}", "steps": steps, "ms_per_step": ms / steps,
            "rows_per_s": rows_per_s, "flop_per_row": TRAIN_FLOP_PER_ROW, "bytes_per_row": TRAIN_BYTES_PER_ROW,
            "roofline": {"bound": "hbm", "achieved": gbs, "peak": hbm_peak, "unit": "GB/s", "frac": gbs / hbm_peak,
                         "peak_source": "MEASURED_PEAKS.json hbm_gbs" if "hbm_gbs" in peaks else "fallback 6650 GB/s",
                         "tensor": {"achieved": tflops, "peak": bf16_peak, "unit": "TFLOP/s",
                                    "frac": tflops / bf16_peak}},
            "data": "synthetic rows (seeded), the surrogate's feature ranges"}


def profile_target(target, side, Engine, abi, np):
    """One call of one leg on the workload's camera at side x side, untimed: the
    program ncu captures for the kernel summaries."""
    eng = Engine(0)
    frame = workload_frame(abi, side, side)
    if target in ("trace-mixed", "trace-fp64"):
        eng.configure(workload_config(abi, abi.PRECISION_MIXED if target == "trace-mixed" else abi.PRECISION_FP64))
        eng.trace_frames([frame], results=False)
        st = eng.stats()
        # a first call: its time includes the one-time module load, so none is printed
        print(target, side, f"rays={st.rays}", f"steps_per_ray={st.accepted_steps / st.rays:.1f}")
    elif target == "beams":
        eng.configure(abi.default_config(abs_tolerance=1e-8, rel_tolerance=1e-8, min_step=1e-9, max_step=2.0,
                                         initial_step=0.1, escape_radius=1000.0, horizon_factor=1.01,
                                         max_steps=20000, precision=abi.PRECISION_FP64, enable_disk=0))
        b = eng.trace_beams([frame])
        print(target, side, b.size, float(b["magnification"].mean()))
    elif target == "stress":
        out = stress_leg(eng, abi, stride=max(4096 // side, 1))
        print(target, out["workload"], f"rays={out['rays']}", f"steps_per_ray={out['steps_per_ray']:.1f}")
    else:
        eng.surrogate_load(np.load(SURROGATE_WEIGHTS))
        eng.configure(surrogate_config(abi, abi.PRECISION_MIXED))
        _, _, _, st = eng.render_surrogate([frame])
        print(target, side, f"rays={st.rays}", f"integrated={st.integrated}")
    eng.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-extras", action="store_true", help="skip the FP64 comparator and the CPU baseline")
    ap.add_argument("--surrogate-only", action="store_true",
                    help="run only the surrogate-gated leg (at --surrogate-size) and print its JSON")
    ap.add_argument("--surrogate-size", type=int, default=SURROGATE_SIDE)
    ap.add_argument("--train-only", action="store_true",
                    help="run only the surrogate-training leg and print its JSON")
    ap.add_argument("--train-steps", type=int, default=64)
    ap.add_argument("--max-registers", type=int, default=0,
                    help="register cap of the mixed trace kernel (0: the library default, 128)")
    ap.add_argument("--size", type=int, default=WIDTH,
                    help="frame side (default 1024, the workload; smaller sides are profiling cases)")
    ap.add_argument("--profile-target", default=None,
                    choices=["trace-mixed", "trace-fp64", "beams", "surrogate", "stress"],
                    help="one untimed call of one leg at --size (an ncu target; for stress, --size is the sky "
                         "map's width), then exit")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
        return

    import numpy as np
    import torch
    import torch.distributed as dist

    from sirius_b200 import abi
    from sirius_b200.engine import Engine, flop_count
    from sirius_b200.shard import gather_rows, max_over_ranks, row_block

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream(dev)
    if args.train_only:
        eng = Engine(local)
        print(json.dumps(train_leg(eng, abi, np, torch, dev, steps=args.train_steps)), flush=True)
        eng.close()
        return
    if args.profile_target:
        profile_target(args.profile_target, args.size, Engine, abi, np)
        return
    if args.surrogate_only:
        eng = Engine(local)
        print(json.dumps(surrogate_leg(eng, abi, np, torch, dev, stream, side=args.surrogate_size)), flush=True)
        eng.close()
        return

    main_cfg = workload_config(abi, abi.PRECISION_MIXED)
    main_cfg.max_registers = args.max_registers
    eng = Engine(local, config=main_cfg)
    full_frame = workload_frame(abi, args.size, args.size)
    # the frame is split across ranks as contiguous row blocks (strong scaling);
    # each rank traces its block's row window, and the image rows are gathered to
    # rank 0 every step (the one exchange of a split frame)
    r0, r1 = row_block(args.size, rank, world)
    frame = workload_frame(abi, args.size, args.size)
    if world > 1:
        frame.row_begin, frame.row_count = r0, r1 - r0
    frames = (abi.Frame * 1)(frame)
    frames[0].ray_offset = 0
    total = abi.frame_rays(frame)
    frame_total = args.size * args.size
    fbytes = bytes(frames)
    d_frames = torch.frombuffer(bytearray(fbytes), dtype=torch.uint8).to(dev)
    d_image = torch.empty(total, dtype=torch.float32, device=dev)
    d_spectra = torch.empty(total * N_BINS, dtype=torch.float32, device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    def step():
        eng.trace_frames_device(d_frames.data_ptr(), 1, total, None, d_image.data_ptr(), d_spectra.data_ptr(),
                                stream.cuda_stream)
        if world > 1:
            gather_rows(d_image, args.size, args.size, dist, dev)

    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    kernel_ms, accepted, rejected, fp64, launches = [], 0, 0, 0, 0
    for i in range(args.steps):
        flush.zero_()
        ev[i][0].record(stream)
        step()
        ev[i][1].record(stream)
        st = eng.stats()  # synchronises on the library's stream: per-launch kernel time (CUDA events)
        kernel_ms.append(st.kernel_ms)
        launches += st.kernel_launches
        accepted += st.accepted_steps
        rejected += st.rejected_steps
        fp64 += st.fp64_steps
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clk = clocks.stop()
    step_ms = [a.elapsed_time(b) for a, b in ev]
    # device time of the K steps, the maximum over ranks (each rank traces its row block)
    t_total = max_over_ranks(sum(step_ms), dist if world > 1 else None, dev)
    value = frame_total * args.steps / (t_total * 1e-3) / 1e6

    # end to end through the host entry point: frame descriptor H2D, image + spectra D2H (pinned)
    h_img = torch.empty(total, dtype=torch.float32, pin_memory=True)
    h_spc = torch.empty(total * N_BINS, dtype=torch.float32, pin_memory=True)
    fr_arr = (abi.Frame * 1)(frame)
    for _ in range(2):
        eng.trace_frames_into(C.addressof(fr_arr), 1, None, h_img.data_ptr(), h_spc.data_ptr())
    if world > 1:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        eng.trace_frames_into(C.addressof(fr_arr), 1, None, h_img.data_ptr(), h_spc.data_ptr())
    t_e2e = max_over_ranks(time.perf_counter() - t0, dist if world > 1 else None, dev)
    e2e = frame_total * args.steps / t_e2e / 1e6

    # roofline of the trace kernel: algorithmic operations / kernel time vs the measured FP32 SIMT peak
    rhs_f, att_f, acc_f = flop_count(frame.metric)
    flops = accepted * acc_f + rejected * att_f
    kernel_s = sum(kernel_ms) * 1e-3
    achieved = flops / kernel_s / 1e12
    peak32 = eng.fma_peak(1) / 1e12
    peak64 = eng.fma_peak(0) / 1e12

    line = {"metric": "Mrays/s", "value": value, "unit": "Mrays/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_total / args.steps, "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": "f32+f64",
            "data": "synthetic (seeded camera frame; no dataset)", "config": workload_desc(args.size),
            "e2e": {"value": e2e, "unit": "Mrays/s", "h2d_bytes_per_step": C.sizeof(abi.Frame),
                    "d2h_bytes_per_step": total * 4 * (1 + N_BINS)},
            "gpu_launches": launches,
            "roofline": {"bound": "fp32_simt", "achieved": achieved, "peak": peak32, "unit": "TFLOP/s",
                         "frac": achieved / peak32, "traffic": TRAFFIC_BYTES_PER_RAY * total,
                         "traffic_unit": "bytes per launch (ncu, 512^2 capture scaled by rays)",
                         "peak_source": "measured FMA-chain microbenchmark (sirius_cuda_measure_fma_peak)",
                         "fp64_peak": peak64, "flops_per_accepted_step": acc_f, "flops_per_rhs": rhs_f,
                         "kernel": "trace_kernel<mixed>"},
            "steps_per_ray": accepted / (total * args.steps), "rejected_per_ray": rejected / (total * args.steps),
            "fp64_island_step_fraction": fp64 / max(accepted, 1), "clocks": clk}

    if rank == 0 and world == 1 and not args.no_extras:
        # the mixed frame with per-ray records (untimed), for the error report against the oracle
        res_mixed, _, _ = eng.trace_frames([full_frame], results=True, spectra=False)
        # the plain FP64 GPU integrator on the same frame (one thread per ray), and the error vs it
        img_mixed = d_image.cpu().numpy().astype(np.float64)
        spc_mixed = d_spectra.cpu().numpy().reshape(total, N_BINS).astype(np.float64)
        eng.configure(workload_config(abi, abi.PRECISION_FP64))
        ms64 = []
        for i in range(3):
            step()
            st = eng.stats()
            if i > 0:
                ms64.append(st.kernel_ms)
        img64 = d_image.cpu().numpy().astype(np.float64)
        spc64 = d_spectra.cpu().numpy().reshape(total, N_BINS).astype(np.float64)
        err = np.abs(img_mixed - img64) / img64.max()
        serr = np.abs(spc_mixed - spc64) / spc64.max(axis=0, keepdims=True)
        line["fp64_plain"] = {"kernel_ms": float(np.mean(ms64)),
                              "mrays_per_s": total / (np.mean(ms64) * 1e-3) / 1e6,
                              "speedup_of_mixed": float(np.mean(ms64)) / (sum(kernel_ms) / len(kernel_ms))}
        line["error_vs_fp64"] = {"image_linf_rel": float(err.max()), "image_p99_rel": float(np.percentile(err, 99)),
                                 "spectra_linf_rel": float(serr.max()),
                                 "spectra_p99_rel": float(np.percentile(serr, 99))}
        # the library's default gates (critical-curve band and inner-disk gate), and the
        # critical-curve band alone (faster, with the network's worst case at the inner edge)
        line["surrogate"] = surrogate_leg(eng, abi, np, torch, dev, stream)
        line["surrogate_band_only"] = surrogate_leg(eng, abi, np, torch, dev, stream, inner_gate=-1.0)
        line["surrogate_training"] = train_leg(eng, abi, np, torch, dev)
        line["beams"] = beam_leg(eng, abi)
        line["graph_replay"] = graph_leg(eng, abi, torch, dev)
        line["heterogeneous_batch"] = batch_leg(eng, abi)
        line["stress_symplectic"] = stress_leg(eng, abi)
        line.update(cpu_baseline_sample(res_mixed, img_mixed, spc_mixed))
    if world > 1 and not args.no_extras:
        # the heterogeneous batch split by whole frames (every rank takes part)
        line["heterogeneous_batch"] = batch_leg(eng, abi, rank, world, dist, dev)
    if rank == 0:
        print(json.dumps(line), flush=True)
    eng.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()

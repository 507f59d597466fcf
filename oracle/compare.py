"""Per-output error report of an engine trace against the CPU oracle.

TEST INFRASTRUCTURE ONLY — imported by tests/ and by the CPU-baseline leg of
bench.py, as the checker; never by the product package.

The outputs compared are the ones the task's accuracy bars name (null-constraint
drift, conserved E / L_z / Carter Q, terminal position and direction, outcome
agreement, disk crossings, image intensity). Rays whose histories split at
rounding level between the two integrations are counted and left out of the
per-ray comparisons: a different outcome, a different number of disk crossings
or equatorial crossings (a grazing ray that one integration sends just inside
the horizon or the disk edge and the other just outside). Everything else is
compared ray by ray, and the maxima are over every compared ray.

Null constraint: |g^{mu nu} p_mu p_nu| as the engine returns it, absolute (the
camera normalises E to O(1)) and relative to sum_mu p_mu^2.

Terminal state, over the rays that escape in both traces (final coordinate
radius beyond the escape radius): the escape direction is the angle between the
spatial parts of the final covariant momenta (FP64 in both records); the
terminal position is the final point's offset across the ray (the component of
the position difference perpendicular to the escape direction) relative to its
radius, since the two integrations stop at different points along the same
asymptotic line.

Conserved quantities (computeConservedQuantities, MTTP001A.h:114-132):
  drift      |X_final - X_initial| / max(|X_initial|, floor) per ray of the engine,
             with floor = 1e-3 x the median |X_initial| of the frame (L_z and Q
             vanish on some rays, where a relative drift is meaningless);
  vs_oracle  |X_engine - X_oracle| / max(|X_oracle|, floor) at termination.
"""
import numpy as np


def _stats(v):
    v = np.asarray(v, dtype=np.float64)
    if v.size == 0:
        return {"max": 0.0, "p99": 0.0, "n": 0}
    return {"max": float(v.max()), "p99": float(np.percentile(v, 99)), "n": int(v.size)}


def _rel(a, b, x0):
    floor = 1e-3 * float(np.median(np.abs(x0))) if x0.size else 0.0
    floor = max(floor, 1e-300)
    return np.abs(a - b) / np.maximum(np.abs(x0), floor)


def split_histories(res, ref):
    """Rays whose histories split at rounding level: outcome, disk crossings or
    equatorial crossings differ."""
    return ((res["outcome"] != ref["outcome"]) | (res["n_crossings"] != ref["n_crossings"]) |
            (res["equatorial_crossings"] != ref["equatorial_crossings"]))


def _cartesian(res, spherical):
    """Final positions and spatial momentum directions in Cartesian components.
    Spherical states (t, r, theta, phi; the Morris-Thorne chart) are mapped with
    the orthonormal spherical frame: (p_r, p_theta / r, p_phi / (r sin theta))
    rotated onto (x, y, z) (the far-field direction of an escaped ray)."""
    x = res["final_x"].astype(np.float64)
    p = res["final_p"].astype(np.float64)
    if not spherical:
        return x[:, 1:], p[:, 1:]
    r, th, ph = x[:, 1], x[:, 2], x[:, 3]
    st, ct, sp, cp = np.sin(th), np.cos(th), np.sin(ph), np.cos(ph)
    pos = np.stack([r * st * cp, r * st * sp, r * ct], 1)
    er = np.stack([st * cp, st * sp, ct], 1)
    et = np.stack([ct * cp, ct * sp, -st], 1)
    ep = np.stack([-sp, cp, np.zeros_like(sp)], 1)
    pr, pt, pp = p[:, 1], p[:, 2] / np.maximum(r, 1e-30), p[:, 3] / np.maximum(r * np.abs(st), 1e-30)
    return pos, pr[:, None] * er + pt[:, None] * et + pp[:, None] * ep


def report(res, img, ref, spectra=None, ref_bins=None, escape_radius=None, spherical=False):
    """Errors of an engine trace (results res, image img, optional spectra) against
    the oracle's trace of the same pixels (ref, ref_bins). Images are compared
    relative to the oracle image's peak, spectra per bin relative to the bin's peak.
    escape_radius (None: the smallest final radius of the oracle's escaped rays)
    selects the escaped rays of the terminal-state comparison; spherical: the
    states are in the (t, r, theta, phi) chart."""
    n = len(ref)
    split = split_histories(res, ref)
    same = ~split
    out = {"rays": int(n), "outcome_agreement": float((res["outcome"] == ref["outcome"]).mean()),
           "split_histories": int(split.sum())}
    # null constraint |g^{mu nu} p_mu p_nu| of the engine: the largest value met before a
    # re-projection, and the returned state's
    out["null_before_projection"] = _stats(res["null_drift_max"])
    out["null_final"] = _stats(res["null_final"])
    p2 = np.sum(res["final_p"].astype(np.float64) ** 2, axis=1)
    out["null_final_relative"] = _stats(res["null_final"] / np.maximum(p2, 1e-300))
    # conserved quantities
    for name in ("E", "Lz", "Carter"):
        x0 = res[name + "0"].astype(np.float64)
        out[name] = {"drift": _stats(_rel(res[name], res[name + "0"], x0)),
                     "vs_oracle": _stats(_rel(res[name][same], ref[name][same], ref[name][same]))}
    # terminal state of the rays that escape in both traces
    xg_all, pg_all = _cartesian(res, spherical)
    xo_all, po_all = _cartesian(ref, spherical)
    rg = np.linalg.norm(xg_all, axis=1)
    ro = np.linalg.norm(xo_all, axis=1)
    if escape_radius is None:
        esc0 = ref["outcome"] == 0
        escape_radius = float(ro[esc0].min()) if esc0.any() else np.inf
    esc = same & (rg >= escape_radius) & (ro >= escape_radius)
    out["escaped_compared"] = int(esc.sum())
    pg = pg_all[esc]
    po = po_all[esc]
    ng = pg / np.linalg.norm(pg, axis=1, keepdims=True)
    no = po / np.linalg.norm(po, axis=1, keepdims=True)
    out["escape_direction_rad"] = _stats(np.arctan2(np.linalg.norm(np.cross(ng, no), axis=1), np.sum(ng * no, 1)))
    dx = xg_all[esc] - xo_all[esc]
    perp = dx - np.sum(dx * no, 1, keepdims=True) * no
    out["terminal_position"] = _stats(np.linalg.norm(perp, axis=1) / ro[esc])
    # disk crossings (first crossing of rays that both trace onto the disk)
    hit = same & (ref["n_crossings"] > 0)
    out["disk_r"] = _stats(np.abs(res["disk_r"][hit, 0] - ref["disk_r"][hit, 0]) / ref["disk_r"][hit, 0])
    out["disk_g"] = _stats(np.abs(res["disk_g"][hit, 0] - ref["disk_g"][hit, 0]) /
                           np.maximum(np.abs(ref["disk_g"][hit, 0]), 1e-30))
    # image intensity, relative to the oracle image's peak: every compared ray, and every ray
    scale = max(float(np.abs(ref["intensity"]).max()), 1e-300)
    err = np.abs(np.asarray(img, dtype=np.float64) - ref["intensity"]) / scale
    out["image"] = _stats(err[same])
    out["image_all_rays"] = _stats(err)
    if spectra is not None and ref_bins is not None and ref_bins.size:
        bscale = np.maximum(np.abs(ref_bins).max(axis=0, keepdims=True), 1e-300)
        serr = np.abs(np.asarray(spectra, dtype=np.float64) - ref_bins) / bscale
        out["spectra"] = _stats(serr[same].ravel())
    return out


def summary(rep):
    """One line per output: max and p99."""
    lines = [f"rays {rep['rays']}, outcome agreement {rep['outcome_agreement']:.5f}, "
             f"split histories {rep['split_histories']}, escaped rays compared {rep['escaped_compared']}"]
    for k, v in rep.items():
        if isinstance(v, dict) and "max" in v:
            lines.append(f"{k}: max {v['max']:.3e} p99 {v['p99']:.3e}")
        elif isinstance(v, dict):
            for kk, vv in v.items():
                lines.append(f"{k}.{kk}: max {vv['max']:.3e} p99 {vv['p99']:.3e}")
    return "\n".join(lines)


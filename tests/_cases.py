"""Golden-case plumbing shared by the tests: maps a fixture's CLI arguments
to launch angles and solver parameters the way run_prop does
(main.infraga.3d.cpp:240-306), and parses the fixtures."""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
GOLDEN = os.path.join(HERE, "golden")
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from infraga_b200 import synth  # noqa: E402

# Per-column tolerances for FP64 GPU vs FP64 CPU (same algorithm, different
# FMA contraction and transcendental implementations; rounding differences
# grow along multi-bounce rays to ~1e-9 relative).  Units: deg, deg, -, km,
# km, s, km/s, km, deg, deg, dB, dB.  Launch angles and bounce index exact.
FP64_ATOL = np.array([0, 0, 0, 1e-4, 1e-4, 1e-4, 1e-7, 1e-4, 1e-5, 1e-5, 1e-3, 1e-4])
FP64_RTOL = 1e-8


def load_cases():
    with open(os.path.join(GOLDEN, "cases.json")) as f:
        return json.load(f)


def profile_path(seed: int) -> str:
    return os.path.join(GOLDEN, "profiles", f"gen{seed}.met")


def parse_golden(name: str):
    rows, steps = [], []
    with open(os.path.join(GOLDEN, name + ".txt")) as f:
        for line in f:
            if not line.strip() or line.startswith("#"):
                continue
            if line.startswith("R\t"):
                steps.append(int(line.split("\t")[3]))
            else:
                rows.append([float(x) for x in line.split("\t")])
    return np.array(rows, dtype=np.float64).reshape(-1, 12), np.array(steps, dtype=np.int64)


def case_setup(args, z_ground: float = 0.0, z_top: float = 150.0):
    """Angles and a parameter dict (keys of iga_fan_params / the oracle cfg)
    for a run_prop argument list, with the 3D CLI defaults."""
    kv = dict(a.split("=", 1) for a in args)
    b = lambda s: s.lower() == "true" or (s.lstrip("-").isdigit() and int(s) != 0)  # noqa: E731
    th_min, th_max, th_step = 0.5, 45.0, 0.5
    az_min, az_max, az_step = -90.0, -90.0, 1.0
    if "inclination" in kv:
        th_min = th_max = float(kv["inclination"]); th_step = 1.0
    if "azimuth" in kv:
        az_min = az_max = float(kv["azimuth"]); az_step = 1.0
    th_min = float(kv.get("incl_min", th_min)); th_max = float(kv.get("incl_max", th_max))
    th_step = float(kv.get("incl_step", th_step))
    az_min = float(kv.get("az_min", az_min)); az_max = float(kv.get("az_max", az_max))
    az_step = float(kv.get("az_step", az_step))
    z0 = float(kv.get("z_grnd", z_ground))
    src = (float(kv.get("src_x", 0.0)), float(kv.get("src_y", 0.0)), float(kv.get("src_alt", 0.0)))
    z_src = max(src[2], z0)
    th, ph = synth.fan_angles(th_min, th_max, th_step, az_min, az_max, az_step,
                              src_above_ground=(z_src - z0) >= 0.01)
    p = dict(src=src, ds_min=0.001, ds_max=0.05, s_max=1000.0, alt_max=z_top, rng_max=2000.0,
             x_min=-2000.0, x_max=2000.0, y_min=-2000.0, y_max=2000.0, z_grnd=z0, freq=0.1, tweak_abs=1.0,
             turn_ht_min=0.2, bounces=10, calc_amp=1, write_rays=1)
    p["bounces"] = int(kv.get("bounces", p["bounces"]))
    p["rng_max"] = float(kv.get("max_rng", p["rng_max"]))
    p["freq"] = float(kv.get("freq", p["freq"]))
    p["tweak_abs"] = max(0.0, float(kv.get("abs_coeff", p["tweak_abs"])))
    p["turn_ht_min"] = float(kv.get("turn_ht_min", p["turn_ht_min"]))
    if "calc_amp" in kv:
        p["calc_amp"] = int(b(kv["calc_amp"]))
    if "write_rays" in kv:
        p["write_rays"] = int(b(kv["write_rays"]))
    return th, ph, p


# Spherical fans: columns 3/4 are latitude/longitude in degrees (1e-6 deg is
# about 0.1 m on the ground); the rest as for 3D.
SPH_ATOL = FP64_ATOL.copy()
SPH_ATOL[3] = SPH_ATOL[4] = 1e-6


def case_setup_sph(args, z_ground: float = 0.0, z_top: float = 150.0):
    """Angles and iga_fan_params fields for an infraga-sph run_prop argument
    list (main.infraga.sph.cpp:207-320), with that CLI's defaults."""
    kv = dict(a.split("=", 1) for a in args)
    shared = [a for a in args if a.split("=", 1)[0] not in ("src_lat", "src_lon", "src_alt", "max_rng")]
    _, _, p = case_setup(shared, z_ground, z_top)
    src = (float(kv.get("src_lat", 30.0)), float(kv.get("src_lon", 0.0)), float(kv.get("src_alt", 0.0)))
    z_src = max(src[2], p["z_grnd"])
    th, ph = synth.fan_angles(*_fan_args(kv), src_above_ground=(z_src - p["z_grnd"]) >= 0.01)
    for k in ("x_min", "x_max", "y_min", "y_max"):
        del p[k]
    p.update(geometry=1, src=src, rng_max=float(kv.get("max_rng", 1000.0)),
             lat_min=float(kv.get("min_lat", -90.0)), lat_max=float(kv.get("max_lat", 90.0)),
             lon_min=float(kv.get("min_lon", -180.0)), lon_max=float(kv.get("max_lon", 180.0)),
             time_max=float(kv.get("max_time", 10.0)))
    return th, ph, p


def golden_src(name: str):
    """Source (lat, lon, alt) a range-dependent fixture ran with (its
    ``# src`` line: run_prop puts the default source at the region centre)."""
    with open(os.path.join(GOLDEN, name + ".txt")) as f:
        for line in f:
            if line.startswith("# src "):
                return tuple(float(x) for x in line.split()[2:5])
    raise ValueError(f"{name}: no source line")


def golden_angles(name: str):
    """(theta, phi) of every ray of a fixture, from its ``R`` lines."""
    th, ph = [], []
    with open(os.path.join(GOLDEN, name + ".txt")) as f:
        for line in f:
            if line.startswith("R\t"):
                _, t, p, _ = line.split("\t")
                th.append(float(t)); ph.append(float(p))
    return np.array(th), np.array(ph)


def _fan_args(kv):
    th_min, th_max, th_step = 0.5, 45.0, 0.5
    az_min, az_max, az_step = -90.0, -90.0, 1.0
    if "inclination" in kv:
        th_min = th_max = float(kv["inclination"]); th_step = 1.0
    if "azimuth" in kv:
        az_min = az_max = float(kv["azimuth"]); az_step = 1.0
    return (float(kv.get("incl_min", th_min)), float(kv.get("incl_max", th_max)), float(kv.get("incl_step", th_step)),
            float(kv.get("az_min", az_min)), float(kv.get("az_max", az_max)), float(kv.get("az_step", az_step)))


def compare_arrivals(got: np.ndarray, ref: np.ndarray, atol=FP64_ATOL, rtol=FP64_RTOL, amp_skip_db: float = 60.0):
    """Column-wise comparison; returns (ok, report).  Amplitude is compared
    only where the reference value is above -amp_skip_db (near-caustic
    arrivals, where the Jacobian crosses zero, are flagged, not compared)."""
    if got.shape != ref.shape:
        return False, f"row count differs: got {got.shape[0]}, reference {ref.shape[0]}"
    d = np.abs(got - ref)
    lim = atol[None, :] + rtol * np.abs(ref)
    caustic = ref[:, 10] < -amp_skip_db
    bad = d > lim
    bad[caustic, 10] = False
    if bad.any():
        i, j = np.argwhere(bad)[0]
        return False, f"{bad.sum()} values out of tolerance; first row {i} col {j}: got {got[i, j]!r} ref {ref[i, j]!r}"
    return True, f"max abs diff per column {d.max(axis=0, initial=0.0)}"


# FP32-compensated path vs the FP64 reference.
#
# The north-star bound: ground-intercept range within 10 m, travel time within
# 10 ms and amplitude within 0.1 dB of the FP64 result for non-caustic rays.
# An arrival is non-caustic when its ray has passed no caustic up to it: the
# FP64 run's caustic count (sign changes of the ray-tube Jacobian between
# consecutive RK4 rows, per-arrival diagnostic column 3) is 0.  Without
# calc_amp there is no Jacobian and every arrival counts as non-caustic (range
# and time only).  Arrivals are paired by (ray, bounce); rays whose arrival
# count differs, or whose turning height moves by more than TURN_FLIP_KM, are
# classification flips: counted and reported, not paired.
NS_RANGE_KM = 0.010
NS_TIME_S = 0.010
NS_AMP_DB = 0.1
TURN_FLIP_KM = 1.0


def match_arrivals(rows_a, idx_a, rows_b, idx_b, n_rays, extra_b=None):
    """Pair arrivals of two runs by (ray, bounce).  Returns (a_rows, b_rows,
    extra_b_rows, flipped_ray_ids): rays with differing arrival counts or a
    turning-height change above TURN_FLIP_KM are flips and left out."""
    cnt_a = np.bincount(idx_a, minlength=n_rays)
    cnt_b = np.bincount(idx_b, minlength=n_rays)
    flipped = set(np.nonzero(cnt_a != cnt_b)[0].tolist())
    ok_a = np.isin(idx_a, list(flipped), invert=True)
    ok_b = np.isin(idx_b, list(flipped), invert=True)
    a, b = rows_a[ok_a], rows_b[ok_b]
    ia = idx_a[ok_a]
    turn = np.abs(a[:, 7] - b[:, 7]) > TURN_FLIP_KM
    flipped |= set(ia[turn].tolist())
    keep = np.isin(ia, list(flipped), invert=True)
    ex = extra_b[ok_b][keep] if extra_b is not None else None
    return a[keep], b[keep], ex, np.array(sorted(flipped), dtype=np.int64)


def noncaustic_report(got, ref, caustics, calc_amp=True):
    """North-star check of paired FP32C (got) and FP64 (ref) arrival rows:
    violation counts and maxima over the non-caustic arrivals, percentiles
    over all paired arrivals."""
    nc = caustics == 0
    rng = np.hypot(got[:, 3] - ref[:, 3], got[:, 4] - ref[:, 4])
    dt = np.abs(got[:, 5] - ref[:, 5])
    da = np.abs(got[:, 10] - ref[:, 10]) if calc_amp else np.zeros(got.shape[0])

    def pct(x, q):
        return float(np.percentile(x, q)) if x.size else 0.0
    rep = {"n": int(got.shape[0]), "n_noncaustic": int(nc.sum()),
           "viol_range": int((nc & (rng > NS_RANGE_KM)).sum()), "viol_time": int((nc & (dt > NS_TIME_S)).sum()),
           "viol_amp": int((nc & (da > NS_AMP_DB)).sum()),
           "nc_range_km_max": float(rng[nc].max(initial=0.0)), "nc_time_s_max": float(dt[nc].max(initial=0.0)),
           "nc_amp_db_max": float(da[nc].max(initial=0.0)),
           "nc_turn_ht_km_max": float(np.abs(got[nc, 7] - ref[nc, 7]).max(initial=0.0)),
           "nc_arr_incl_deg_max": float(np.abs(got[nc, 8] - ref[nc, 8]).max(initial=0.0)),
           "nc_atten_db_max": float(np.abs(got[nc, 11] - ref[nc, 11]).max(initial=0.0)),
           "range_km_p50": pct(rng, 50), "range_km_p99": pct(rng, 99), "range_km_max": float(rng.max(initial=0.0)),
           "time_s_p50": pct(dt, 50), "time_s_p99": pct(dt, 99),
           "amp_db_p50": pct(da, 50), "amp_db_p99": pct(da, 99)}
    rep["ok"] = rep["viol_range"] == 0 and rep["viol_time"] == 0 and rep["viol_amp"] == 0
    # the worst non-caustic rows (incl, az, bounce, range err, time err, amp err, reference amp)
    for key, err in (("worst_range", rng), ("worst_amp", da)):
        o = np.argsort(-np.where(nc, err, -1.0))[:4]
        rep[key] = [(float(ref[i, 0]), float(ref[i, 1]), int(ref[i, 2]), float(rng[i]), float(dt[i]), float(da[i]),
                     float(ref[i, 10])) for i in o if nc[i]]
    return rep


def worst_rows(got, ref, extra, col, k=8):
    """Rows with the largest |got - ref| in column col (range when col == 3),
    with the reference-side diagnostics, for reporting."""
    if col == 3:
        e = np.hypot(got[:, 3] - ref[:, 3], got[:, 4] - ref[:, 4])
    else:
        e = np.abs(got[:, col] - ref[:, col])
    o = np.argsort(-e)[:k]
    return [(float(ref[i, 0]), float(ref[i, 1]), int(ref[i, 2]), float(e[i]), float(ref[i, 10]),
             *(float(x) for x in (extra[i] if extra is not None else []))) for i in o]

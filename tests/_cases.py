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
    return True, f"max abs diff per column {d.max(axis=0)}"

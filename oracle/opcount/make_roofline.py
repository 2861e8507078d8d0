"""Writes roofline.json: FLOP-equivalents per RK4 ray-step of the 3D
stratified fan, counted by running the oracle restatement (bit-identical to the
reference solver) with an operation-counting scalar (opcount.cpp) over a
representative fan of the benchmark workload.  Test infrastructure: bench.py
reads the JSON it writes, never this script or the counting build.

    python oracle/opcount/make_roofline.py

Weights (stated in the file): add/sub/mul 1, div/sqrt 4, exp/log/pow/
trigonometric/cbrt 20 FLOP-equivalents.  Representative fan: the benchmark
profiles (seeds 1-4), azimuth 90 deg, inclinations 0.5..60 every 4 deg, 10
bounces, 2000 km -- the config-1 fan's settings on a 15-ray slice.

Variants:
  fp64_amp / fp64_noamp : the reference algorithm as the FP64 kernel runs it
                          (18 or 6 equations, Sutherland-Bass per step);
  fp32c_amp / fp32c_noamp: the same minus the per-step Sutherland-Bass
                          evaluation, which the FP32-compensated kernel reads
                          from a tabulated alpha(z) (a linear interpolation,
                          counted as ALPHA_LERP_FLOPS).
Only the 3D stratified solver has a CPU restatement; the spherical and
range-dependent kernels are not counted here.
"""
from __future__ import annotations

import json
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE = os.path.dirname(HERE)
ROOT = os.path.dirname(ORACLE)
sys.path.insert(0, ROOT)

WEIGHTS = {"add": 1, "mul": 1, "div": 4, "sqrt": 4, "exp": 20, "log": 20, "pow": 20, "trig": 20, "cbrt": 20}
ALPHA_LERP_FLOPS = 6.0   # index scale, floor, weight, lerp (2 mul + 2 add), tweak_abs and ds products
FAN = dict(bounces=10, rng_max=2000.0, incl=(0.5, 60.01, 4.0), azimuth=90.0)
SEEDS = (1, 2, 3, 4)


def weighted(c: dict) -> float:
    return sum(WEIGHTS[k] * v for k, v in c.items())


def compute() -> dict:
    """Build the counting oracle, run it over the sample and return the
    roofline.json content."""
    subprocess.run(["make", "-s", "-C", ORACLE, "opcount"], check=True)
    exe = os.path.join(ORACLE, "_build", "opcount")
    prof_dir = os.path.join(ROOT, "tests", "golden", "profiles")
    out = {"unit": "FLOP-equivalents per accepted RK4 ray-step", "weights": WEIGHTS,
           "alpha_lerp_flops": ALPHA_LERP_FLOPS,
           "sample": (f"3D stratified fan, seeds {list(SEEDS)}, azimuth {FAN['azimuth']} deg, inclinations "
                      f"{FAN['incl'][0]}..{FAN['incl'][1]} step {FAN['incl'][2]} deg, {FAN['bounces']} bounces, "
                      f"{FAN['rng_max']} km"),
           "method": "oracle restatement compiled with an operation-counting scalar (oracle/opcount)",
           "variants": {}, "counts": {}}
    for amp in (1, 0):
        tot_steps, acc_rest, acc_abs = 0, {k: 0.0 for k in WEIGHTS}, {k: 0.0 for k in WEIGHTS}
        for seed in SEEDS:
            met = os.path.join(prof_dir, f"gen{seed}.met")   # the benchmark generator's profiles, committed
            r = subprocess.run([exe, met, str(amp), str(FAN["bounces"]), str(FAN["rng_max"]), *map(str, FAN["incl"]),
                                str(FAN["azimuth"])], check=True, capture_output=True, text=True)
            d = json.loads(r.stdout)
            n = d["ray_steps"]
            tot_steps += n
            for k in WEIGHTS:
                acc_rest[k] += d["rest"][k] * n
                acc_abs[k] += d["absorption"][k] * n
        rest = {k: v / tot_steps for k, v in acc_rest.items()}
        absn = {k: v / tot_steps for k, v in acc_abs.items()}
        tag = "amp" if amp else "noamp"
        out["counts"][tag] = {"ray_steps": tot_steps, "rest": rest, "absorption": absn}
        out["variants"][f"fp64_{tag}"] = round(weighted(rest) + weighted(absn), 1)
        out["variants"][f"fp32c_{tag}"] = round(weighted(rest) + ALPHA_LERP_FLOPS, 1)
    return out


def main() -> int:
    out = compute()
    with open(os.path.join(ROOT, "roofline.json"), "w") as f:
        json.dump(out, f, indent=1)
        f.write("\n")
    print(json.dumps(out["variants"]))
    return 0


if __name__ == "__main__":
    sys.exit(main())

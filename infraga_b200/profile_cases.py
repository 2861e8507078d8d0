"""Small, self-contained runs of each kernel for profiling (ncu captures
summarised under profiles/).  Each case traces one modest workload once per
repetition, so a capture with ``-k regex:<kernel> -c 1`` sees a
representative launch of a few hundred milliseconds at most.

    python -m infraga_b200.profile_cases <case> [--reps N]

cases:
  fansph     spherical stratified fan (fansph_fp64_kernel): 1,440 rays
  fansphr    spherical range-dependent fan with terrain (fansphr_fp64_kernel):
             the 21x21 grid of workloads.py, 408 rays, 1 bounce, 600 km
  fan3dr     3D range-dependent fan with terrain (fan3dr_fp64_kernel): the
             committed 5x5 grid, 1,080 rays, 2 bounces, 600 km
  paths      3D stratified fan with sampled ray paths (PATHS instantiation)
  eig3d      3D eigenray search, 16 pairs (trace3d_fp64_kernel)
  eigsph     spherical eigenray search, 8 pairs (tracesph_fp64_kernel)
"""
from __future__ import annotations

import argparse
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def _golden(*p):
    return os.path.join(ROOT, "tests", "golden", *p)


def case_fansph(ig, wl):
    from infraga_b200 import synth
    atmo = ig.Atmosphere.load(wl.profile_met(1))
    th, ph = synth.fan_angles(0.5, 60.0, 0.5, 0.0, 330.0, 30.0)
    p = atmo.default_params(geometry=ig.GEOM_SPH, bounces=5, rng_max=2000.0, src=(30.0, 0.0, 0.0))
    return lambda: ig.fan_run(atmo, p, th, ph)


def case_fansphr(ig, wl):
    from infraga_b200 import synth
    f = wl.sphr_files()
    atmo = ig.Atmosphere.load_rngdep(f[0], f[1], f[2], topo_file=f[3], geometry=ig.GEOM_SPH)
    th, ph = synth.fan_angles(0.5, 50.0, 3.0, 0.0, 345.0, 15.0)
    p = atmo.default_params(geometry=ig.GEOM_SPH, bounces=1, rng_max=600.0)
    return lambda: ig.fan_run(atmo, p, th, ph)


def case_fan3dr(ig, wl):
    from infraga_b200 import synth
    d = _golden("rngdep3d")
    atmo = ig.Atmosphere.load_rngdep(os.path.join(d, "node"), os.path.join(d, "node_x.dat"),
                                     os.path.join(d, "node_y.dat"), topo_file=os.path.join(d, "topo.dat"),
                                     geometry=ig.GEOM_3D)
    th, ph = synth.fan_angles(0.5, 45.0, 0.5, 0.0, 330.0, 30.0)
    p = atmo.default_params(bounces=2, rng_max=600.0)
    return lambda: ig.fan_run(atmo, p, th, ph)


def case_paths(ig, wl):
    from infraga_b200 import synth
    atmo = ig.Atmosphere.load(wl.profile_met(1))
    th, ph = synth.fan_angles(1.0, 45.0, 1.0, 0.0, 330.0, 30.0)
    p = atmo.default_params(bounces=3, rng_max=1000.0, write_rays=1)
    steps = ig.fan_run(atmo, p, th, ph)["ray_steps"]
    return lambda: ig.fan_paths(atmo, p, th, ph, caustics=True, ray_steps=steps)


def case_eig3d(ig, wl):
    atmo = ig.Atmosphere.load(wl.profile_met(1))
    pairs = wl.eig_pairs(1, 16)
    p = ig.eig_params(atmo, bnc_min=0, bnc_max=2, streams=1)
    return lambda: ig.eig_run(atmo, p, pairs)


def case_eigsph(ig, wl):
    atmo = ig.Atmosphere.load(wl.profile_met(1))
    pairs = [((30.0, 0.0, 0.0), (30.0 + 2.0 * k / 8.0, 2.5 + 0.25 * k)) for k in range(8)]
    p = ig.eig_params(atmo, geometry=ig.GEOM_SPH, bnc_min=0, bnc_max=1, streams=1)
    return lambda: ig.eig_run(atmo, p, pairs)


CASES = {k[len("case_"):]: v for k, v in globals().items() if k.startswith("case_")}


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("case", choices=sorted(CASES))
    ap.add_argument("--reps", type=int, default=1)
    args = ap.parse_args(argv)
    sys.path.insert(0, ROOT)
    import infraga_b200 as ig
    from infraga_b200 import workloads as wl
    run = CASES[args.case](ig, wl)
    for _ in range(args.reps):
        run()
    print(f"{args.case}: ok")
    return 0


if __name__ == "__main__":
    sys.exit(main())

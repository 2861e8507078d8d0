"""Seeded synthetic workloads of the measured configurations, shared by
bench.py's timed legs and its profiling cases (``--profile-case``).

* spherical range-dependent fan: a 21 x 21 node grid at 1 deg (each node a
  751-level profile whose jet amplitudes vary smoothly across the grid),
  fractal terrain 0-3 km on a 0.05 deg grid (401 x 401), a fan of
  inclinations 0.5..50 step 0.25 x azimuths 0..355 step 5 (199 x 72 =
  14,328 rays by the reference's FP64-accumulated loop), 20 bounces,
  3000 km;
* batched eigenray search: per seed 128 source-receiver pairs, receivers on
  the ground at ranges uniform in 50..800 km and azimuths uniform in
  0..360 deg, bounce counts 0..8.

Files are written once into a cache directory and reused.
"""
from __future__ import annotations

import os

import numpy as np

from . import synth

SPHR_GRID = dict(seed=7, n_lat=21, n_lon=21, lat0=30.0, lon0=-110.0, dlat=1.0, dlon=1.0)
SPHR_TERRAIN = dict(seed=8, step=0.05, z_max=3.0)
SPHR_FAN = dict(incl=(0.5, 50.0, 0.25), az=(0.0, 355.0, 5.0), bounces=20, rng_max=3000.0)
EIG = dict(pairs=128, rng=(50.0, 800.0), bnc_max=8)


def default_cache() -> str:
    return os.environ.get("IGA_WORKLOAD_CACHE", os.path.join(os.path.expanduser("~"), ".cache", "infraga_b200"))


def sphr_files(cache: str | None = None):
    """(prefix, lat_file, lon_file, topo_file) of the spherical range-dependent
    workload, generated on first use."""
    d = os.path.join(cache or default_cache(), "sphr_21x21")
    g = SPHR_GRID
    prefix = os.path.join(d, "node")
    lat_f, lon_f = prefix + "_lat.dat", prefix + "_lon.dat"
    topo = os.path.join(d, "topo.dat")
    n_nodes = g["n_lat"] * g["n_lon"]
    if not (os.path.exists(topo) and os.path.exists(f"{prefix}{n_nodes - 1}.met")):
        synth.write_rngdep_grid(d, g["seed"], n_lat=g["n_lat"], n_lon=g["n_lon"], lat0=g["lat0"], lon0=g["lon0"],
                                dlat=g["dlat"], dlon=g["dlon"])
        t = SPHR_TERRAIN
        lat1 = g["lat0"] + g["dlat"] * (g["n_lat"] - 1)
        lon1 = g["lon0"] + g["dlon"] * (g["n_lon"] - 1)
        synth.write_terrain(topo + ".tmp", t["seed"], g["lat0"], lat1, g["lon0"], lon1, t["step"], t["z_max"])
        os.replace(topo + ".tmp", topo)
    return prefix, lat_f, lon_f, topo


def sphr_angles():
    f = SPHR_FAN
    return synth.fan_angles(*f["incl"], *f["az"])


def eig_pairs(seed: int, n: int | None = None):
    """Source at the origin, receivers on the ground (x east, y north, km)."""
    n = n or EIG["pairs"]
    g = np.random.default_rng(1000 + seed)
    r = g.uniform(*EIG["rng"], n)
    a = g.uniform(0.0, 2.0 * np.pi, n)
    return [((0.0, 0.0, 0.0), (float(ri * np.cos(ai)), float(ri * np.sin(ai)))) for ri, ai in zip(r, a)]


def profile_met(seed: int, cache: str | None = None) -> str:
    """The stratified config-0 generator's profile for `seed` (written once)."""
    d = os.path.join(cache or default_cache(), "profiles")
    os.makedirs(d, exist_ok=True)
    path = os.path.join(d, f"gen{seed}.met")
    if not os.path.exists(path):
        synth.write_met(path + ".tmp", seed)
        os.replace(path + ".tmp", path)
    return path

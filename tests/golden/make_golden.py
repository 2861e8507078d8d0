"""Regenerates the golden fixtures in this directory from the reference solver
itself (oracle/_ref, compiled from the reference sources by oracle/Makefile).

    python tests/golden/make_golden.py           # all cases; needs make -C oracle ref
    python tests/golden/make_golden.py NAME...   # only these cases (cases.json is merged)

Each fixture is the full-precision output of the reference's own solver
functions driven by oracle/harness/*.cpp: one line per arrival
(%.17g, the 12 .arrivals.dat columns), ``R`` lines with each ray's RK4 step
count, and a ``#`` summary line.  Profiles are seeded synthetic ones
(infraga_b200.synth), also stored here so the fixtures do not depend on the
random generator.
"""
from __future__ import annotations

import json
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from infraga_b200 import synth  # noqa: E402

PROFILES = os.path.join(HERE, "profiles")
REF = os.path.join(ROOT, "oracle", "_ref")

# name -> (binary, mode, profile seed, argv key=value list)
CASES = {
    "3d_c0_rays": ("iga_ref_3d", "prop", 0, ["incl_min=1", "incl_max=45", "incl_step=1", "azimuth=90", "bounces=5",
                                             "max_rng=1000", "write_rays=true"]),
    "3d_c0_bulk": ("iga_ref_3d", "prop", 0, ["incl_min=1", "incl_max=45", "incl_step=1", "azimuth=90", "bounces=5",
                                             "max_rng=1000", "write_rays=false"]),
    "3d_noamp": ("iga_ref_3d", "prop", 1, ["incl_min=2", "incl_max=40", "incl_step=2", "az_min=0", "az_max=300",
                                           "az_step=60", "bounces=3", "max_rng=800", "calc_amp=false",
                                           "write_rays=false"]),
    "3d_fan_sub": ("iga_ref_3d", "prop", 2, ["incl_min=0.5", "incl_max=60.01", "incl_step=3.5", "az_min=0",
                                             "az_max=270", "az_step=90", "bounces=10", "max_rng=2000",
                                             "write_rays=false"]),
    "3d_elevated": ("iga_ref_3d", "prop", 3, ["incl_min=-30", "incl_max=30", "incl_step=5", "azimuth=45",
                                              "bounces=2", "src_alt=10", "max_rng=600", "write_rays=false"]),
    "3d_zgrnd": ("iga_ref_3d", "prop", 4, ["incl_min=5", "incl_max=35", "incl_step=5", "azimuth=200", "bounces=3",
                                           "z_grnd=0.5", "freq=0.5", "abs_coeff=0.3", "turn_ht_min=10",
                                           "max_rng=900", "write_rays=true"]),
}

# Spherical (global) fans through oracle/harness/harness_sph.cpp; angles in
# degrees as on the infraga-sph command line.
SPH_CASES = {
    "sph_c0_bulk": ("iga_ref_sph", "prop", 0, ["incl_min=1", "incl_max=45", "incl_step=2", "azimuth=90", "bounces=3",
                                               "src_lat=30", "src_lon=10", "write_rays=false"]),
    "sph_rays": ("iga_ref_sph", "prop", 1, ["incl_min=2", "incl_max=38", "incl_step=4", "az_min=0", "az_max=300",
                                            "az_step=60", "bounces=2", "src_lat=-45", "src_lon=-60", "max_rng=800",
                                            "write_rays=true"]),
    "sph_noamp": ("iga_ref_sph", "prop", 2, ["incl_min=3", "incl_max=33", "incl_step=6", "az_min=-90", "az_max=90",
                                             "az_step=90", "bounces=2", "src_lat=10", "src_lon=100", "calc_amp=false",
                                             "write_rays=false"]),
    "sph_elevated": ("iga_ref_sph", "prop", 3, ["incl_min=-30", "incl_max=30", "incl_step=6", "azimuth=45",
                                                "bounces=2", "src_alt=10", "src_lat=0", "src_lon=0", "max_rng=800",
                                                "write_rays=false"]),
    "sph_dateline": ("iga_ref_sph", "prop", 4, ["incl_min=5", "incl_max=35", "incl_step=5", "azimuth=80", "bounces=3",
                                                "src_lat=-20", "src_lon=177", "z_grnd=0.5", "freq=0.5",
                                                "abs_coeff=0.3", "turn_ht_min=10", "max_rng=1500",
                                                "write_rays=true"]),
    "sph_pole": ("iga_ref_sph", "prop", 0, ["incl_min=4", "incl_max=36", "incl_step=8", "az_min=-10", "az_max=10",
                                            "az_step=10", "bounces=6", "src_lat=84", "src_lon=45", "max_rng=3000",
                                            "write_rays=false"]),
    "sph_limits": ("iga_ref_sph", "prop", 1, ["incl_min=5", "incl_max=40", "incl_step=7", "az_min=45", "az_max=135",
                                              "az_step=45", "bounces=4", "src_lat=40", "src_lon=-100",
                                              "max_lat=43", "min_lon=-104", "max_lon=-95", "max_time=0.3",
                                              "write_rays=false"]),
}

# Spherical range-dependent fans through oracle/harness/harness_sphr.cpp over
# a seeded 5 x 5 node grid (1.5 deg spacing, 151 levels) and a seeded fractal
# terrain on a 0.2 deg grid (files under rngdep/).  "TOPO" stands for the
# terrain file.
RNGDEP_DIR = os.path.join(HERE, "rngdep")
RNGDEP_CASES = {
    "sphr_flat": ["incl_min=2", "incl_max=30", "incl_step=4", "az_min=45", "az_max=225", "az_step=180",
                  "bounces=3", "write_rays=false"],
    "sphr_topo": ["topo_file=TOPO", "incl_min=2", "incl_max=30", "incl_step=4", "az_min=90", "az_max=270",
                  "az_step=180", "bounces=3", "write_rays=true"],
    "sphr_topo_noamp": ["topo_file=TOPO", "calc_amp=false", "incl_min=5", "incl_max=25", "incl_step=10",
                        "az_min=0", "az_max=270", "az_step=90", "bounces=2"],
    "sphr_topo_elevated": ["topo_file=TOPO", "src_alt=5", "incl_min=-30", "incl_max=10", "incl_step=10",
                           "az_min=0", "az_max=270", "az_step=90", "bounces=2"],
}


# 3D Cartesian range-dependent fans through oracle/harness/harness_3dr.cpp:
# 5 x 5 nodes at 150 km spacing over [-300, 300] km, terrain on a 20 km grid
# (files under rngdep3d/).
RNGDEP3D_DIR = os.path.join(HERE, "rngdep3d")
RNGDEP3D_CASES = {
    "3dr_flat": ["incl_min=2", "incl_max=30", "incl_step=4", "az_min=45", "az_max=225", "az_step=180",
                 "bounces=3", "write_rays=false"],
    "3dr_topo": ["topo_file=TOPO", "incl_min=2", "incl_max=30", "incl_step=4", "az_min=90", "az_max=270",
                 "az_step=180", "bounces=3", "write_rays=true"],
    "3dr_topo_noamp": ["topo_file=TOPO", "calc_amp=false", "incl_min=5", "incl_max=25", "incl_step=10",
                       "az_min=0", "az_max=270", "az_step=90", "bounces=2"],
    "3dr_topo_elevated": ["topo_file=TOPO", "src_alt=5", "incl_min=-30", "incl_max=10", "incl_step=10",
                          "az_min=0", "az_max=270", "az_step=90", "bounces=2"],
}


def rngdep3d_files():
    return (os.path.join(RNGDEP3D_DIR, "node"), os.path.join(RNGDEP3D_DIR, "node_x.dat"),
            os.path.join(RNGDEP3D_DIR, "node_y.dat"), os.path.join(RNGDEP3D_DIR, "topo.dat"))


def rngdep_files():
    """(prefix, lat_file, lon_file, topo_file) of the committed range-dependent fixtures."""
    return (os.path.join(RNGDEP_DIR, "node"), os.path.join(RNGDEP_DIR, "node_lat.dat"),
            os.path.join(RNGDEP_DIR, "node_lon.dat"), os.path.join(RNGDEP_DIR, "topo.dat"))


# Eigenray searches (run_eig_search through the same driver; the reference
# writes these rows with setprecision(8)).  name -> (profile seed, argv)
EIG_CASES = {
    "3d_eig_a": (0, ["rcvr_x=250", "rcvr_y=40", "bnc_min=0", "bnc_max=2"]),
    "3d_eig_b": (4, ["rcvr_x=330", "rcvr_y=90", "bnc_min=0", "bnc_max=1"]),
    "3d_eig_c": (3, ["rcvr_x=520", "rcvr_y=0", "bnc_min=1", "bnc_max=3"]),
    "3d_eig_none": (2, ["rcvr_x=180", "rcvr_y=-30", "bnc_min=0", "bnc_max=1"]),
}

# Config-3 searches at the full bounce range: the first six receivers of the
# batched eigenray workload's seeds 1 and 2 (infraga_b200.workloads.eig_pairs:
# source at the origin, receivers on the ground 50..800 km away), bounces
# 0..8, on the same seeded profiles.  Run concurrently (minutes per pair).
def _eig8_cases():
    from infraga_b200 import workloads
    cases = {}
    for seed in (1, 2):
        for k, (_, (rx, ry)) in enumerate(workloads.eig_pairs(seed)[:6]):
            cases[f"3d_eig8_s{seed}_p{k}"] = (seed, [f"rcvr_x={rx:.6f}", f"rcvr_y={ry:.6f}", "bnc_min=0", "bnc_max=8"])
    return cases


EIG8_CASES = _eig8_cases()

# Spherical eigenray searches through oracle/harness/harness_sph.cpp (degrees
# as on the infraga-sph command line).  name -> (profile seed, argv)
SPH_EIG_CASES = {
    "sph_eig_a": (0, ["src_lat=30", "src_lon=0", "rcvr_lat=30.5", "rcvr_lon=2.5", "bnc_min=0", "bnc_max=1"]),
    "sph_eig_b": (4, ["src_lat=10", "src_lon=100", "rcvr_lat=12", "rcvr_lon=103", "bnc_min=0", "bnc_max=2"]),
    "sph_eig_c": (0, ["src_lat=30", "src_lon=0", "rcvr_lat=31", "rcvr_lon=5", "bnc_min=1", "bnc_max=1",
                      "incl_min=5", "incl_max=30"]),
    "sph_eig_none": (2, ["src_lat=60", "src_lon=170", "rcvr_lat=60", "rcvr_lon=175", "bnc_min=0", "bnc_max=0"]),
}


def profile_path(seed: int) -> str:
    return os.path.join(PROFILES, f"gen{seed}.met")


def main():
    only = set(sys.argv[1:])
    want = lambda name: not only or name in only  # noqa: E731
    os.makedirs(PROFILES, exist_ok=True)
    for seed in range(5):
        synth.write_met(profile_path(seed), seed)
    meta = {}
    meta_path = os.path.join(HERE, "cases.json")
    if only and os.path.exists(meta_path):
        with open(meta_path) as f:
            meta = json.load(f)
    for name, (binary, mode, seed, args) in CASES.items():
        if not want(name):
            continue
        exe = os.path.join(REF, binary)
        cmd = [exe, mode, profile_path(seed), *args]
        r = subprocess.run(cmd, capture_output=True, text=True, check=True)
        with open(os.path.join(HERE, name + ".txt"), "w") as f:
            f.write(r.stdout)
        meta[name] = {"binary": binary, "mode": mode, "seed": seed, "args": args}
        print(name, r.stdout.strip().splitlines()[-1])
    for name, (binary, mode, seed, args) in SPH_CASES.items():
        if not want(name):
            continue
        cmd = [os.path.join(REF, binary), mode, profile_path(seed), *args]
        r = subprocess.run(cmd, capture_output=True, text=True, check=True)
        with open(os.path.join(HERE, name + ".txt"), "w") as f:
            f.write(r.stdout)
        meta[name] = {"binary": binary, "mode": mode, "seed": seed, "args": args}
        print(name, r.stdout.strip().splitlines()[-1])
    if not only or any(n in only for n in RNGDEP_CASES):
        synth.write_rngdep_grid(RNGDEP_DIR, 5, n_lat=5, n_lon=5, lat0=30.0, lon0=-110.0, dlat=1.5, dlon=1.5,
                                dz=1.0, prefix="node")
        synth.write_terrain(os.path.join(RNGDEP_DIR, "topo.dat"), 5, 30.0, 36.0, -110.0, -104.0, 0.2, 2.0)
    prefix, lat_f, lon_f, topo_f = rngdep_files()
    for name, args in RNGDEP_CASES.items():
        if not want(name):
            continue
        argv = [a.replace("TOPO", topo_f) for a in args]
        cmd = [os.path.join(REF, "iga_ref_sphr"), "prop", prefix, lat_f, lon_f, *argv]
        r = subprocess.run(cmd, capture_output=True, text=True, check=True)
        with open(os.path.join(HERE, name + ".txt"), "w") as f:
            f.write(r.stdout)
        meta[name] = {"binary": "iga_ref_sphr", "mode": "prop", "seed": 5, "args": args}
        print(name, r.stdout.strip().splitlines()[-2])
    if not only or any(n in only for n in RNGDEP3D_CASES):
        synth.write_rngdep_grid(RNGDEP3D_DIR, 9, n_lat=5, n_lon=5, lat0=-300.0, lon0=-300.0, dlat=150.0,
                                dlon=150.0, dz=1.0, prefix="node", axes=("x", "y"))
        synth.write_terrain(os.path.join(RNGDEP3D_DIR, "topo.dat"), 9, -300.0, 300.0, -300.0, 300.0, 20.0, 2.0)
    prefix, x_f, y_f, topo_f = rngdep3d_files()
    for name, args in RNGDEP3D_CASES.items():
        if not want(name):
            continue
        argv = [a.replace("TOPO", topo_f) for a in args]
        cmd = [os.path.join(REF, "iga_ref_3dr"), "prop", prefix, x_f, y_f, *argv]
        r = subprocess.run(cmd, capture_output=True, text=True, check=True)
        with open(os.path.join(HERE, name + ".txt"), "w") as f:
            f.write(r.stdout)
        meta[name] = {"binary": "iga_ref_3dr", "mode": "prop", "seed": 9, "args": args}
        print(name, r.stdout.strip().splitlines()[-2])
    for name, (seed, args) in EIG_CASES.items():
        if not want(name):
            continue
        out = os.path.join(HERE, name + ".txt")
        cmd = [os.path.join(REF, "iga_ref_3d"), "eig", profile_path(seed), *args, "out=" + out,
               "out_id=" + os.path.join("/tmp", name)]
        r = subprocess.run(cmd, capture_output=True, text=True, check=True)
        with open(out, "a") as f:
            f.write(r.stdout)
        meta[name] = {"binary": "iga_ref_3d", "mode": "eig", "seed": seed, "args": args}
        print(name, r.stdout.strip().splitlines()[-1])
    todo = [(n, a) for n, a in EIG8_CASES.items() if want(n)]
    if todo:
        from concurrent.futures import ThreadPoolExecutor

        def run_eig8(item):
            name, (seed, args) = item
            out = os.path.join(HERE, name + ".txt")
            if os.path.exists(out):
                os.remove(out)
            cmd = [os.path.join(REF, "iga_ref_3d"), "eig", profile_path(seed), *args, "out=" + out,
                   "out_id=" + os.path.join("/tmp", name)]
            r = subprocess.run(cmd, capture_output=True, text=True)
            if r.returncode != 0:   # the reference crashes on some inputs: no fixture
                if os.path.exists(out):
                    os.remove(out)
                return name, seed, args, None, f"reference exited with {r.returncode}"
            with open(out, "a") as f:
                f.write(r.stdout)
            return name, seed, args, r.stdout.strip().splitlines()[-1], None
        with ThreadPoolExecutor(max_workers=os.cpu_count() or 1) as ex:
            for name, seed, args, last, err in ex.map(run_eig8, todo):
                if err:
                    meta.pop(name, None)
                    print(name, "skipped:", err)
                    continue
                meta[name] = {"binary": "iga_ref_3d", "mode": "eig", "seed": seed, "args": args}
                print(name, last)
    for name, (seed, args) in SPH_EIG_CASES.items():
        if not want(name):
            continue
        out = os.path.join(HERE, name + ".txt")
        cmd = [os.path.join(REF, "iga_ref_sph"), "eig", profile_path(seed), *args, "out=" + out,
               "out_id=" + os.path.join("/tmp", name)]
        r = subprocess.run(cmd, capture_output=True, text=True, check=True)
        with open(out, "a") as f:
            f.write(r.stdout)
        meta[name] = {"binary": "iga_ref_sph", "mode": "eig", "seed": seed, "args": args}
        print(name, r.stdout.strip().splitlines()[-1])
    with open(meta_path, "w") as f:
        json.dump(meta, f, indent=1)


if __name__ == "__main__":
    main()

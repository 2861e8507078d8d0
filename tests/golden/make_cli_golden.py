"""Regenerates the command-line fixtures under cli/ from the reference's own,
unmodified command-line binaries (oracle/_ref/infraga-*, built from the
reference sources by ``make -C oracle ref``).

    python tests/golden/make_cli_golden.py           # all cases
    python tests/golden/make_cli_golden.py NAME...   # only these cases

Each case runs one binary in a scratch directory laid out by ``stage()``
(the same layout the GPU front-end test uses, so header lines that echo
file names match) and keeps every output file it wrote under cli/NAME/,
with the argument list in cli/cases.json.  Atmospheres are the seeded
synthetic fixtures already in this directory.
"""
from __future__ import annotations

import json
import os
import shutil
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF = os.path.join(ROOT, "oracle", "_ref")
OUT = os.path.join(HERE, "cli")

# name -> (binary, atmosphere kind, seed of the 1D profile, argv after the binary)
# kinds: "1d" = profiles/gen{seed}.met staged as atmo.met;
#        "sphr" / "3dr" = the rngdep/ or rngdep3d/ grid staged as grid/node*, grid/x.dat, grid/y.dat, topo.dat;
#        "1dt" / "1dts" = profiles/gen{seed}.met as atmo.met over the rngdep3d/ (x, y) or rngdep/ (lat, lon)
#        terrain as topo.dat
CASES = {
    "3d_prop": ("infraga-3d", "1d", 0,
                ["-prop", "atmo.met", "incl_min=4", "incl_max=24", "incl_step=10", "az_min=0", "az_max=90",
                 "az_step=90", "bounces=2", "max_rng=600", "max_ds=0.25", "write_caustics=true", "write_topo=true"]),
    "3d_prop_noamp": ("infraga-3d", "1d", 1,
                      ["-p", "atmo.met", "incl_min=10", "incl_max=30.5", "incl_step=0.5", "azimuth=-60", "bounces=1",
                       "max_rng=300", "calc_amp=false", "write_rays=false", "z_grnd=0.25", "freq=0.3"]),
    "3d_eig": ("infraga-3d", "1d", 0,
               ["-eig_search", "atmo.met", "rcvr_x=240", "rcvr_y=30", "bnc_min=0", "bnc_max=1", "incl_min=10",
                "incl_max=17"]),
    "3d_direct": ("infraga-3d", "1d", 0,
                  ["-eig_direct", "atmo.met", "rcvr_x=240", "rcvr_y=30", "incl_est=8", "bounces=0",
                   "output_id=direct"]),
    "3d_back_proj": ("infraga-3d", "1d", 0,
                     ["-back_proj", "atmo.met", "inclination=12", "azimuth=60", "bounces=1", "rcvr_x=10", "max_ds=0.25",
                      "freq=0.2"]),
    "3d_back_proj_dflt": ("infraga-3d", "1d", 1, ["-b", "atmo.met", "max_ds=0.5", "output_id=bp"]),
    "3d_atmo": ("infraga-3d", "1d", 1,
                ["-prop", "atmo.met", "inclination=20", "azimuth=30", "bounces=0", "write_rays=false", "write_atmo=true",
                 "max_alt=120", "z_grnd=0.3"]),
    "3d_direct_atmo": ("infraga-3d", "1d", 0,
                       ["-eig_direct", "atmo.met", "rcvr_x=240", "rcvr_y=30", "incl_est=8", "az_est=80", "bounces=0",
                        "write_atmo=true", "output_id=direct"]),
    "sph_atmo": ("infraga-sph", "1d", 0,
                 ["-prop", "atmo.met", "inclination=20", "azimuth=30", "bounces=0", "write_rays=false",
                  "write_atmo=true", "src_lat=20", "src_lon=-40"]),
    "sph_prop": ("infraga-sph", "1d", 1,
                 ["-prop", "atmo.met", "incl_min=4", "incl_max=24", "incl_step=10", "az_min=0", "az_max=180",
                  "az_step=180", "bounces=1", "src_lat=20", "src_lon=-40", "max_rng=700", "max_ds=0.25", "write_caustics=true",
                  "write_topo=true"]),
    "sph_eig": ("infraga-sph", "1d", 0,
                ["-eig_search", "atmo.met", "src_lat=30", "src_lon=0", "rcvr_lat=30.5", "rcvr_lon=2.5", "bnc_min=0",
                 "bnc_max=0", "incl_min=10", "incl_max=15"]),
    "sph_direct": ("infraga-sph", "1d", 0,
                   ["-eig_direct", "atmo.met", "src_lat=30", "src_lon=0", "rcvr_lat=30.5", "rcvr_lon=2.5",
                    "incl_est=12", "bounces=0", "output_id=direct"]),
    "3dr_prop": ("infraga-3d-rngdep", "3dr", 0,
                 ["-prop", "grid/node", "grid/x.dat", "grid/y.dat", "topo_file=topo.dat", "incl_min=6",
                  "incl_max=26", "incl_step=10", "az_min=90", "az_max=270", "az_step=180", "bounces=1",
                  "max_rng=400", "max_ds=0.25", "write_caustics=true", "write_topo=true"]),
    "3dr_calc_amp": ("infraga-3d-rngdep", "3dr", 0,
                     ["-prop", "grid/node", "grid/x.dat", "grid/y.dat", "inclination=12", "azimuth=100",
                      "bounces=1", "calc_amp=true", "write_rays=false", "output_id=amp"]),
    "3dr_eig": ("infraga-3d-rngdep", "3dr", 0,
                ["-eig_search", "grid/node", "grid/x.dat", "grid/y.dat", "topo_file=topo.dat", "rcvr_x=210",
                 "rcvr_y=0", "incl_min=12", "incl_max=24"]),
    "3dr_back_proj": ("infraga-3d-rngdep", "3dr", 0,
                      ["-back_proj", "grid/node", "grid/x.dat", "grid/y.dat", "inclination=12", "azimuth=60",
                       "bounces=1", "rcvr_x=40", "rcvr_y=-30", "max_ds=0.25"]),
    "3dr_back_proj_topo": ("infraga-3d-rngdep", "3dr", 0,
                           ["-back_proj", "grid/node", "grid/x.dat", "grid/y.dat", "topo_file=topo.dat",
                            "inclination=16", "azimuth=250", "bounces=2", "max_ds=0.25", "output_id=bp"]),
    "3dr_direct": ("infraga-3d-rngdep", "3dr", 0,
                   ["-eig_direct", "grid/node", "grid/x.dat", "grid/y.dat", "topo_file=topo.dat", "rcvr_x=210",
                    "rcvr_y=0", "incl_est=18", "az_est=90", "bounces=0", "output_id=direct"]),
    "3dt_prop": ("infraga-3d", "1dt", 0,
                 ["-prop", "atmo.met", "topo_file=topo.dat", "incl_min=6", "incl_max=26", "incl_step=10", "az_min=90",
                  "az_max=270", "az_step=180", "bounces=1", "max_rng=400", "max_ds=0.25", "write_caustics=true",
                  "write_topo=true"]),
    "3dt_noamp": ("infraga-3d", "1dt", 1,
                  ["-p", "atmo.met", "topo_file=topo.dat", "incl_min=10", "incl_max=30", "incl_step=5", "azimuth=-60",
                   "bounces=2", "max_rng=500", "calc_amp=false", "write_rays=false", "freq=0.3"]),
    "3dt_eig": ("infraga-3d", "1dt", 0,
                ["-eig_search", "atmo.met", "topo_file=topo.dat", "rcvr_x=240", "rcvr_y=0", "incl_min=14",
                 "incl_max=28", "bnc_max=1"]),
    "3dt_direct": ("infraga-3d", "1dt", 0,
                   ["-eig_direct", "atmo.met", "topo_file=topo.dat", "rcvr_x=240", "rcvr_y=0", "incl_est=20",
                    "bounces=0", "output_id=direct"]),
    "spht_prop": ("infraga-sph", "1dts", 0,
                  ["-prop", "atmo.met", "topo_file=topo.dat", "incl_min=6", "incl_max=26", "incl_step=10", "az_min=90",
                   "az_max=270", "az_step=180", "bounces=1", "max_rng=400", "max_ds=0.25", "write_caustics=true",
                   "write_topo=true"]),
    "spht_noamp": ("infraga-sph", "1dts", 1,
                   ["-p", "atmo.met", "topo_file=topo.dat", "incl_min=10", "incl_max=30", "incl_step=5", "azimuth=-60",
                    "bounces=2", "max_rng=500", "calc_amp=false", "write_rays=false", "freq=0.3"]),
    "spht_eig": ("infraga-sph", "1dts", 0,
                 ["-eig_search", "atmo.met", "topo_file=topo.dat", "src_alt=3", "rcvr_lat=32.98", "rcvr_lon=-104.6",
                  "incl_min=10", "incl_max=30"]),
    "3dr_atmo": ("infraga-3d-rngdep", "3dr", 0,
                 ["-prop", "grid/node", "grid/x.dat", "grid/y.dat", "topo_file=topo.dat", "inclination=12",
                  "azimuth=100", "bounces=0", "write_rays=false", "write_atmo=true"]),
    "sphr_atmo": ("infraga-sph-rngdep", "sphr", 0,
                  ["-prop", "grid/node", "grid/x.dat", "grid/y.dat", "topo_file=topo.dat", "inclination=12",
                   "azimuth=100", "bounces=0", "write_rays=false", "write_atmo=true"]),
    "sphr_eig": ("infraga-sph-rngdep", "sphr", 0,
                 ["-eig_search", "grid/node", "grid/x.dat", "grid/y.dat", "topo_file=topo.dat", "src_alt=3",
                  "rcvr_lat=32.98", "rcvr_lon=-104.6", "incl_min=10", "incl_max=30"]),
    "sphr_eig_ground": ("infraga-sph-rngdep", "sphr", 0,
                        ["-s", "grid/node", "grid/x.dat", "grid/y.dat", "topo_file=topo.dat", "rcvr_lat=32.98",
                         "rcvr_lon=-104.6", "output_id=ground"]),
    "sphr_prop": ("infraga-sph-rngdep", "sphr", 0,
                  ["-prop", "grid/node", "grid/x.dat", "grid/y.dat", "topo_file=topo.dat", "incl_min=6",
                   "incl_max=26", "incl_step=10", "az_min=90", "az_max=270", "az_step=180", "bounces=1",
                   "max_rng=400", "max_ds=0.25", "write_caustics=true", "write_topo=true"]),
}


# Console output cases: the lines of the reference's stdout that the
# print_resid diagnostic writes (with the ray lines they follow), kept as
# cli/NAME/stdout.txt.  name -> same tuple as CASES.
STDOUT_CASES = {
    "3d_resid": ("infraga-3d", "1d", 0,
                 ["-prop", "atmo.met", "incl_min=5", "incl_max=35", "incl_step=10", "az_min=0", "az_max=90",
                  "az_step=45", "bounces=2", "max_rng=900", "write_rays=false", "print_resid=true"]),
    "3d_resid_noamp": ("infraga-3d", "1d", 2,
                       ["-prop", "atmo.met", "incl_min=8", "incl_max=20", "incl_step=6", "azimuth=-30", "bounces=3",
                        "max_rng=1200", "calc_amp=false", "write_rays=false", "print_resid=true"]),
}
RESID_MARKERS = ("Calculating ray path", "Residuals at Ray Termination", "Eikonal residual", "Aux. param. residual")

# -wnl_wvfrm cases: the reference's infraga-3d and infraga-sph built against
# oracle/fftshim (oracle/_ref/infraga-{3d,sph}-wnl, ``make -C oracle wnl``)
# write the fixtures; the GPU front end runs as bin/infraga-3d / infraga-sph.  Every output file is kept with
# the waveform console lines (WNL_MARKERS) as cli/NAME/stdout.txt; the
# argument lists go to cli/wnl_cases.json.  Kind "1dw" also stages wave.dat,
# a source waveform file (wave_file()).
WNL_CASES = {
    "3d_wnl": ("infraga-3d-wnl", "1d", 0,
               ["-wnl_wvfrm", "atmo.met", "inclination=12", "azimuth=60", "bounces=0", "wvfrm_len=2048"]),
    "3d_wnl_dflt": ("infraga-3d-wnl", "1d", 2, ["-w", "atmo.met"]),
    "3d_wnl_strong": ("infraga-3d-wnl", "1d", 1,
                      ["-wnl_wvfrm", "atmo.met", "inclination=20", "azimuth=-30", "bounces=1", "wvfrm_len=1024",
                       "wvfrm_p0=500", "wvfrm_opt=Uwave", "write_ray=true", "freq=0.5"]),
    "3d_wnl_nwave": ("infraga-3d-wnl", "1d", 0,
                     ["-wnl_wvfrm", "atmo.met", "inclination=8", "azimuth=60", "bounces=1", "wvfrm_opt=Nwave",
                      "wvfrm_len=1024", "wvfrm_ref=5", "wvfrm_out_step=100", "output_id=nw"]),
    "3d_wnl_file": ("infraga-3d-wnl", "1dw", 3,
                    ["-wnl_wvfrm", "atmo.met", "inclination=18", "azimuth=0", "wvfrm_file=wave.dat", "bounces=0",
                     "z_grnd=0.2", "src_alt=0.5", "abs_coeff=2"]),
    "sph_wnl": ("infraga-sph-wnl", "1d", 0,
                ["-wnl_wvfrm", "atmo.met", "inclination=12", "azimuth=60", "bounces=1", "wvfrm_len=1024"]),
    "sph_wnl_nwave": ("infraga-sph-wnl", "1d", 1,
                      ["-wnl_wvfrm", "atmo.met", "src_lat=40", "src_lon=-100", "inclination=20", "azimuth=-30",
                       "bounces=0", "wvfrm_opt=Nwave", "wvfrm_len=2048", "wvfrm_p0=200", "write_ray=true",
                       "wvfrm_out_step=150", "output_id=sw"]),
}
WNL_MARKERS = ("Defining waveform", "Loading waveform", "Computing waveform", "Generating waveform",
               "Caustic encountered", "Arrival summary", "[km E-W]", "[km N-S]", "latitude [deg] =",
               "longitude [deg] =", "time [s] =", "celerity", "turning height", "arrival inclination",
               "back azimuth", "attenuation (geometric)", "trans. coeff. [dB] =", "absorption [dB]",
               "does not return")


def wave_file() -> str:
    """A 512-sample source waveform file (a Gaussian-windowed two-cycle pulse)
    with a comment header, read through load_wvfrm."""
    import math
    lines = ["# t [s]\tp [Pa]"]
    n = 512
    for i in range(n):
        t = -4.0 + 8.0 * i / n
        p = 25.0 * math.exp(-(t / 0.35) ** 2) * math.sin(2.0 * math.pi * t / 0.4)
        lines.append(f"{t:.10g}\t{p:.10g}")
    return "\n".join(lines) + "\n"


def wnl_lines(stdout: str) -> list[str]:
    return [ln for ln in stdout.splitlines() if any(m in ln for m in WNL_MARKERS)]


def run_case_wnl(binary_dir: str, spec, binary: str | None = None) -> tuple[dict[str, str], str]:
    """Runs one -wnl_wvfrm case; returns ({relative path: text}, console lines)."""
    ref_binary, kind, seed, argv = spec
    with tempfile.TemporaryDirectory() as work:
        stage(work, kind, seed)
        before = inputs(work)
        r = subprocess.run([os.path.join(binary_dir, binary or ref_binary), *argv], cwd=work, stdin=subprocess.DEVNULL,
                           capture_output=True, text=True, check=True, timeout=600)
        files = {}
        for rel in sorted(inputs(work) - before):
            with open(os.path.join(work, rel)) as f:
                files[rel] = f.read()
        return files, "\n".join(wnl_lines(r.stdout)) + "\n"


def resid_lines(stdout: str) -> list[str]:
    return [ln for ln in stdout.splitlines() if any(m in ln for m in RESID_MARKERS)]


def run_case_stdout(binary_dir: str, spec) -> str:
    """Runs one console case; returns its print_resid lines."""
    binary, kind, seed, argv = spec
    with tempfile.TemporaryDirectory() as work:
        stage(work, kind, seed)
        r = subprocess.run([os.path.join(binary_dir, binary), *argv], cwd=work, stdin=subprocess.DEVNULL,
                           capture_output=True, text=True, check=True, timeout=600)
        return "\n".join(resid_lines(r.stdout)) + "\n"


def stage(work: str, kind: str, seed: int) -> None:
    """Input files of a case in `work` under fixed relative names."""
    if kind in ("1d", "1dt", "1dts", "1dw"):
        shutil.copy(os.path.join(HERE, "profiles", f"gen{seed}.met"), os.path.join(work, "atmo.met"))
        if kind == "1dw":
            with open(os.path.join(work, "wave.dat"), "w") as f:
                f.write(wave_file())
        elif kind != "1d":
            shutil.copy(os.path.join(HERE, "rngdep3d" if kind == "1dt" else "rngdep", "topo.dat"),
                        os.path.join(work, "topo.dat"))
        return
    src = os.path.join(HERE, "rngdep" if kind == "sphr" else "rngdep3d")
    ax = ("node_lat.dat", "node_lon.dat") if kind == "sphr" else ("node_x.dat", "node_y.dat")
    os.makedirs(os.path.join(work, "grid"), exist_ok=True)
    for f in os.listdir(src):
        if f.startswith("node") and f.endswith(".met"):
            shutil.copy(os.path.join(src, f), os.path.join(work, "grid", f))
    shutil.copy(os.path.join(src, ax[0]), os.path.join(work, "grid", "x.dat"))
    shutil.copy(os.path.join(src, ax[1]), os.path.join(work, "grid", "y.dat"))
    shutil.copy(os.path.join(src, "topo.dat"), os.path.join(work, "topo.dat"))


def inputs(work: str) -> set[str]:
    out = set()
    for d, _, files in os.walk(work):
        for f in files:
            out.add(os.path.relpath(os.path.join(d, f), work))
    return out


def run_case(binary_dir: str, name: str, spec, keep_dir: str | None = None) -> dict[str, str]:
    """Runs one case in a scratch directory; returns {relative path: text} of
    every file the run wrote."""
    binary, kind, seed, argv = spec
    with tempfile.TemporaryDirectory() as work:
        stage(work, kind, seed)
        before = inputs(work)
        subprocess.run([os.path.join(binary_dir, binary), *argv], cwd=work, stdin=subprocess.DEVNULL,
                       stdout=subprocess.DEVNULL, check=True, timeout=600)
        files = {}
        for rel in sorted(inputs(work) - before):
            with open(os.path.join(work, rel)) as f:
                files[rel] = f.read()
        return files


def main(names: list[str]) -> None:
    todo = {k: v for k, v in CASES.items() if not names or k in names}
    meta_path = os.path.join(OUT, "cases.json")
    meta = json.load(open(meta_path)) if os.path.exists(meta_path) else {}
    for name, spec in todo.items():
        files = run_case(REF, name, spec)
        d = os.path.join(OUT, name)
        if os.path.isdir(d):
            shutil.rmtree(d)
        for rel, text in files.items():
            path = os.path.join(d, rel)
            os.makedirs(os.path.dirname(path), exist_ok=True)
            with open(path, "w") as f:
                f.write(text)
        meta[name] = {"binary": spec[0], "kind": spec[1], "seed": spec[2], "argv": spec[3], "files": sorted(files)}
        print(name, sorted(files), sum(len(t) for t in files.values()), "bytes")
    for name, spec in STDOUT_CASES.items():
        if names and name not in names:
            continue
        text = run_case_stdout(REF, spec)
        d = os.path.join(OUT, name)
        os.makedirs(d, exist_ok=True)
        with open(os.path.join(d, "stdout.txt"), "w") as f:
            f.write(text)
        print(name, text.count("\n"), "console lines")
    os.makedirs(OUT, exist_ok=True)
    with open(meta_path, "w") as f:
        json.dump(meta, f, indent=1, sort_keys=True)
    wnl_path = os.path.join(OUT, "wnl_cases.json")
    wmeta = json.load(open(wnl_path)) if os.path.exists(wnl_path) else {}
    for name, spec in WNL_CASES.items():
        if names and name not in names:
            continue
        files, text = run_case_wnl(REF, spec)
        d = os.path.join(OUT, name)
        if os.path.isdir(d):
            shutil.rmtree(d)
        os.makedirs(d)
        for rel, body in files.items():
            with open(os.path.join(d, rel), "w") as f:
                f.write(body)
        with open(os.path.join(d, "stdout.txt"), "w") as f:
            f.write(text)
        wmeta[name] = {"binary": spec[0].replace("-wnl", ""), "ref_binary": spec[0], "kind": spec[1], "seed": spec[2],
                       "argv": spec[3], "files": sorted(files)}
        print(name, sorted(files), sum(len(t) for t in files.values()), "bytes,", text.count("\n"), "console lines")
    with open(wnl_path, "w") as f:
        json.dump(wmeta, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main(sys.argv[1:])

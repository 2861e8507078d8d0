"""Host-side fault injection through the command-line programs: missing,
truncated and corrupted profile, node-grid and terrain files.  Every case
fails in the host loaders before any device call, so these run without a
GPU; each prints the reference's error line (set_region's "ERROR: Invalid
...", atmo_io.3d.strat.cpp:78-81) with the loader's reason, exits 0 as the
reference does, and writes no output file."""
import os
import shutil
import subprocess

import pytest

from tests._cases import GOLDEN, ROOT

BIN = os.path.join(ROOT, "bin")
GOOD = os.path.join(GOLDEN, "profiles", "gen0.met")


@pytest.fixture(scope="module")
def bins():
    if not all(os.path.exists(os.path.join(BIN, b)) for b in ("infraga-3d", "infraga-3d-rngdep")):
        from infraga_b200 import build
        build.build()
    return BIN


def rows():
    return [ln for ln in open(GOOD) if ln.strip() and not ln.startswith("#")]


def run(bins, tmp, exe, args):
    r = subprocess.run([os.path.join(bins, exe), *args], cwd=tmp, capture_output=True, text=True, timeout=120,
                       stdin=subprocess.DEVNULL)
    assert r.returncode == 0, r.stderr
    outputs = [f for f in os.listdir(tmp) if f.endswith(".dat") and not f.startswith(("topo", "x.", "y."))]
    return r.stdout, outputs


def write(tmp, name, lines):
    with open(os.path.join(tmp, name), "w") as f:
        f.writelines(lines)


CASES = {
    "missing": (None, "Invalid atmospheric specification", "cannot open profile"),
    "nan_row": (lambda r: r[:5] + ["1.0\t280.0\tnan\t4.0\t1.1e-03\t900.0\n"] + r[6:], "Invalid atmospheric specification",
                "non-finite"),
    "decreasing_z": (lambda r: r[:5] + [r[3]] + r[6:], "Invalid atmospheric specification", "increase strictly"),
    "two_rows": (lambda r: r[:2], "Invalid atmospheric specification", "fewer than 3"),
    "text_column": (lambda r: r[:5] + ["1.0\tabc\n"] + r[6:], "Invalid atmospheric specification", "numeric columns"),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_corrupt_profile_is_reported(bins, tmp_path, name):
    mutate, line, reason = CASES[name]
    if mutate is not None:
        write(tmp_path, "atmo.met", mutate(rows()))
    out, files = run(bins, tmp_path, "infraga-3d", ["-prop", "atmo.met", "inclination=10", "azimuth=90"])
    assert line in out and reason in out, out[-600:]
    assert files == []


def test_unknown_profile_format_is_reported(bins, tmp_path):
    shutil.copy(GOOD, tmp_path / "atmo.met")
    out, files = run(bins, tmp_path, "infraga-3d", ["-prop", "atmo.met", "prof_format=zXYZ", "inclination=10"])
    assert "ERROR: loading the atmosphere: invalid argument" in out and files == []


def test_ragged_terrain_is_reported(bins, tmp_path):
    shutil.copy(GOOD, tmp_path / "atmo.met")
    grid = [ln for ln in open(os.path.join(GOLDEN, "rngdep3d", "topo.dat"))]
    write(tmp_path, "topo.dat", grid[:-7])   # drops part of the last x row
    out, files = run(bins, tmp_path, "infraga-3d", ["-prop", "atmo.met", "topo_file=topo.dat", "inclination=10"])
    assert "Invalid terrain file or atmospheric specification" in out and "full" in out, out[-600:]
    assert files == []


def test_missing_node_profile_is_reported(bins, tmp_path):
    src = os.path.join(GOLDEN, "rngdep3d")
    os.makedirs(tmp_path / "grid")
    for f in os.listdir(src):
        if f.startswith("node") and f.endswith(".met") and f != "node5.met":
            shutil.copy(os.path.join(src, f), tmp_path / "grid" / f)
    shutil.copy(os.path.join(src, "node_x.dat"), tmp_path / "grid" / "x.dat")
    shutil.copy(os.path.join(src, "node_y.dat"), tmp_path / "grid" / "y.dat")
    out, files = run(bins, tmp_path, "infraga-3d-rngdep", ["-prop", "grid/node", "grid/x.dat", "grid/y.dat",
                                                            "inclination=10"])
    assert "Invalid grid, profile or terrain files" in out and "node5" in out, out[-600:]
    assert files == [] and not [f for f in os.listdir(tmp_path / "grid") if f.endswith("arrivals.dat")]

"""Command-line front ends without a GPU: the binaries are built and answer
-usage / -version / a short argument list without touching the device, and
the reference-written fixtures they are checked against on the GPU are
complete (and, where the compiled reference is present, reproducible)."""
import json
import os
import subprocess
import sys

import pytest

from tests._cases import GOLDEN, ROOT

sys.path.insert(0, GOLDEN)
import make_cli_golden as mk  # noqa: E402

BIN = os.path.join(ROOT, "bin")
CLI = os.path.join(GOLDEN, "cli")
NAMES = ("infraga-3d", "infraga-sph", "infraga-3d-rngdep", "infraga-sph-rngdep")


@pytest.fixture(scope="module")
def bins():
    missing = [b for b in NAMES if not os.path.exists(os.path.join(BIN, b))]
    if missing:
        from infraga_b200 import build
        build.build()
    return BIN


@pytest.mark.parametrize("name", NAMES)
def test_usage_and_version(bins, name):
    exe = os.path.join(bins, name)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0 and f"Usage: {name}" in r.stdout
    r = subprocess.run([exe, "-version", "x", "y", "z"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0 and "infraga" in r.stdout
    r = subprocess.run([exe, "-nonsense", "a", "b", "c"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0 and "Unrecognized option." in r.stdout


def test_unsupported_modes_say_so(bins):
    # the waveform mode: infraga-3d and infraga-sph over flat ground; the range-dependent binaries and
    # terrain refuse before loading
    for name in ("infraga-3d-rngdep", "infraga-sph-rngdep"):
        r = subprocess.run([os.path.join(bins, name), "-wnl_wvfrm", "a", "b", "c", "d"], capture_output=True, text=True,
                           timeout=60)
        assert r.returncode == 0 and "-wnl_wvfrm is not provided" in r.stdout, name
    for name in ("infraga-3d", "infraga-sph"):
        r = subprocess.run([os.path.join(bins, name), "-w", "x.met", "topo_file=t.dat"], capture_output=True,
                           text=True, timeout=60)
        assert r.returncode == 0 and "-wnl_wvfrm over terrain is not provided" in r.stdout, name
    # back projection: infraga-3d over flat ground and infraga-3d-rngdep; the spherical ones refuse
    # before loading anything
    for name in ("infraga-sph", "infraga-sph-rngdep"):
        r = subprocess.run([os.path.join(bins, name), "-back_proj", "a", "b", "c", "d"], capture_output=True, text=True,
                           timeout=60)
        assert r.returncode == 0 and "-back_proj is not provided" in r.stdout, name
    r = subprocess.run([os.path.join(bins, "infraga-3d"), "-b", "x.met", "topo_file=t.dat"], capture_output=True,
                       text=True, timeout=60)
    assert r.returncode == 0 and "over terrain is not provided" in r.stdout
    for name in ("infraga-3d", "infraga-3d-rngdep"):
        r = subprocess.run([os.path.join(bins, name)], capture_output=True, text=True, timeout=60)
        assert "-back_proj   one ray" in r.stdout, name


def test_wnl_fixtures_complete():
    """The -wnl_wvfrm fixtures (reference waveform mode over oracle/fftshim) match
    make_cli_golden.WNL_CASES, and each waveform file holds its samples."""
    cases = json.load(open(os.path.join(CLI, "wnl_cases.json")))
    assert set(cases) == set(mk.WNL_CASES)
    for name, c in cases.items():
        assert c["argv"] == mk.WNL_CASES[name][3]
        assert any(f.endswith(".wvfrm_out.dat") for f in c["files"]), name
        for rel in c["files"]:
            assert os.path.getsize(os.path.join(CLI, name, rel)) > 0, (name, rel)
        text = open(os.path.join(CLI, name, "stdout.txt")).read()
        assert "Computing waveform at ray length" in text or "Generating waveform at ray length" in text, name


def test_cli_fixtures_complete():
    cases = json.load(open(os.path.join(CLI, "cases.json")))
    assert set(cases) == set(mk.CASES)
    for name, c in cases.items():
        assert c["argv"] == mk.CASES[name][3]
        assert c["files"], name
        for rel in c["files"]:
            assert os.path.getsize(os.path.join(CLI, name, rel)) > 0, (name, rel)
        arr = [f for f in c["files"] if f.endswith(".arrivals.dat")]
        if arr and not name.endswith("_ground"):   # *_ground: a case whose reference result is empty
            rows = [ln for ln in open(os.path.join(CLI, name, arr[0])) if ln.strip() and not ln.startswith("#")]
            assert rows, f"{name}: fixture without arrivals"


REF = os.path.join(ROOT, "oracle", "_ref")


@pytest.mark.skipif(not os.path.exists(os.path.join(REF, "infraga-3d")), reason="compiled reference not present")
@pytest.mark.parametrize("name", ["3d_prop_noamp", "3dr_calc_amp", "3dt_noamp", "spht_noamp", "3d_back_proj_dflt",
                                  "3d_atmo", "sphr_atmo"])
def test_reference_binaries_reproduce_fixtures(name):
    c = mk.CASES[name]
    got = mk.run_case(REF, name, c)
    for rel, text in got.items():
        assert text == open(os.path.join(CLI, name, rel)).read(), rel


@pytest.mark.skipif(not os.path.exists(os.path.join(REF, "infraga-3d")), reason="compiled reference not present")
@pytest.mark.parametrize("name", sorted(mk.STDOUT_CASES))
def test_reference_binaries_reproduce_console_fixtures(name):
    with open(os.path.join(CLI, name, "stdout.txt")) as f:
        assert mk.run_case_stdout(REF, mk.STDOUT_CASES[name]) == f.read()

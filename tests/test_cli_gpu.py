"""The drop-in command-line binaries (bin/infraga-3d, -sph, -3d-rngdep,
-sph-rngdep) against output files of the reference's own binaries
(tests/golden/cli, written by tests/golden/make_cli_golden.py): same files,
identical header and blank-line structure, and every number equal to the
printed precision of the reference (6 significant digits; 8 where the
reference switches its stream to setprecision(8)), up to one unit in the
last printed digit where the FP64 GPU and CPU sums straddle a rounding
boundary, and 1e-9 absolute for values that are rounding noise around 0."""
import json
import math
import os
import subprocess
import sys
import tempfile

import pytest

from tests._cases import GOLDEN, ROOT

sys.path.insert(0, GOLDEN)
import make_cli_golden as mk  # noqa: E402

pytestmark = pytest.mark.gpu

BIN = os.path.join(ROOT, "bin")
CLI = os.path.join(GOLDEN, "cli")
CASES = json.load(open(os.path.join(CLI, "cases.json")))


def sig_digits(tok: str) -> int:
    mant = tok.lstrip("+-").split("e")[0].split("E")[0].replace(".", "").lstrip("0")
    return max(len(mant), 1)


def close(a: str, b: str, col_tol: float) -> bool:
    if a == b:
        return True
    x, y = float(a), float(b)
    if math.isnan(x) or math.isnan(y):
        return False
    if abs(x - y) <= col_tol:
        return True
    # one unit in the last printed digit (the shorter of the two renderings)
    m = max(abs(x), abs(y))
    d = min(sig_digits(a), sig_digits(b))
    ulp = 10.0 ** (math.floor(math.log10(m)) - (d - 1)) if m > 0 else 0.0
    return abs(x - y) <= 1.01 * ulp


def compare_file(got: str, ref: str, name: str) -> list[str]:
    g, r = got.splitlines(), ref.splitlines()
    errs = []
    if len(g) != len(r):
        errs.append(f"{name}: {len(g)} lines, reference {len(r)}")
    for i, (lg, lr) in enumerate(zip(g, r)):
        if lr.startswith("#") or not lr.strip():
            if lg != lr:
                errs.append(f"{name}:{i + 1}: {lg!r} != {lr!r}")
            continue
        tg, tr = lg.split("\t"), lr.split("\t")
        if len(tg) != len(tr):
            errs.append(f"{name}:{i + 1}: {len(tg)} fields, reference {len(tr)}")
            continue
        for j, (a, b) in enumerate(zip(tg, tr)):
            if not close(a, b, 1e-9):
                errs.append(f"{name}:{i + 1} col {j}: {a} vs {b}")
        if len(errs) > 20:
            break
    return errs


@pytest.fixture(scope="module")
def built():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU tests need a CUDA device")
    for b in ("infraga-3d", "infraga-sph", "infraga-3d-rngdep", "infraga-sph-rngdep"):
        assert os.path.exists(os.path.join(BIN, b)), f"bin/{b} missing: run __graft_entry__.build()"
    return True


@pytest.mark.parametrize("name", sorted(CASES))
def test_cli_matches_reference_files(built, name):
    c = CASES[name]
    spec = (c["binary"], c["kind"], c["seed"], c["argv"])
    got = mk.run_case(BIN, name, spec)
    errs = []
    # arrivals first: they say most about a mismatch
    for rel in sorted(c["files"], key=lambda f: not f.endswith(".arrivals.dat")):
        if rel not in got:
            errs.append(f"{rel}: not written")
            continue
        with open(os.path.join(CLI, name, rel)) as f:
            errs += compare_file(got[rel], f.read(), rel)
    errs += [f"{rel}: written, not in the reference output" for rel in sorted(set(got) - set(c["files"]))]
    assert not errs, "\n".join(errs[:30])


def test_cli_unknown_key_prompt_declined(built):
    """An unrecognised key asks to continue; answering n stops before any output."""
    with tempfile.TemporaryDirectory() as work:
        mk.stage(work, "1d", 0)
        r = subprocess.run([os.path.join(BIN, "infraga-3d"), "-prop", "atmo.met", "inclination=10", "azimuth=90",
                            "no_such_key=1"], cwd=work, input="n\n", capture_output=True, text=True, timeout=300)
        assert r.returncode == 0
        assert "Unrecognized parameter entry: no_such_key=1" in r.stdout
        assert not os.path.exists(os.path.join(work, "atmo.arrivals.dat"))


@pytest.mark.parametrize("name", sorted(mk.STDOUT_CASES))
def test_cli_print_resid_matches_reference(built, name):
    """print_resid's console lines (main.infraga.3d.cpp:437-441) against the
    reference binary's: the same ray and segment lines, eikonal residuals within
    1e-13 + 1e-4 relative (they are RK4 truncation error, so the FP64 rounding
    differences between the CPU and the GPU show at the 1e-15 level), auxiliary
    residuals within 1e-4 relative.  Without calc_amp the reference reads its
    auxiliary residual past the end of 6-column solution rows (undefined); the
    GPU front end prints 0 there, so that value is not compared."""
    spec = mk.STDOUT_CASES[name]
    got = mk.run_case_stdout(BIN, spec).splitlines()
    with open(os.path.join(CLI, name, "stdout.txt")) as f:
        ref = f.read().splitlines()
    assert len(got) == len(ref), (len(got), len(ref))
    noamp = "calc_amp=false" in spec[3]
    for g, r in zip(got, ref):
        if ":" not in r or "residual" not in r:
            assert g == r
            continue
        pg, vg = g.rsplit(":", 1)
        pr, vr = r.rsplit(":", 1)
        assert pg == pr
        x, y = float(vg), float(vr)
        if "Aux." in r:
            if noamp:
                assert x == 0.0
            else:
                assert abs(x - y) <= 1e-4 * abs(y) + 1e-12, (g, r)
        else:
            assert abs(x - y) <= 1e-13 + 1e-4 * abs(y), (g, r)

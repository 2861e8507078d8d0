"""infraga-3d and infraga-sph -wnl_wvfrm on the GPU (iga_wnl_run,
infraga_b200/csrc/wnl3d.cu) against the reference's own waveform mode:
oracle/_ref/infraga-{3d,sph}-wnl are the unmodified reference binaries built
against oracle/fftshim (a working FFT behind the FFTW API subset they call),
and their output files for the cases of tests/golden/make_cli_golden.py
WNL_CASES are the fixtures.

Tolerances.  Time columns: the printed 8 significant digits, within one unit
of the last digit (the FP64 travel-time sums of the GPU and the CPU can
straddle a rounding boundary).  Waveform and spectrum columns: within
WAVE_RTOL of the column's largest magnitude.  The Burgers solve runs a few
hundred Heun steps, each an FFT pair; the GPU transforms the weighted sum of
the three non-linear series once where the reference transforms each, and its
FFT (radix-2 over N/2 points with the real split) rounds differently from the
shim's (radix-2 over N points), so the two agree to rounding accumulated over
the steps, not bit for bit.  Ray-path columns: the 6-digit rule of
tests/test_cli_gpu.py.  Console lines: the same lines; ray lengths exact,
altitudes and beta to 1e-5 relative, arrival summary to the printed digits."""
import json
import math
import os

import numpy as np
import pytest

from tests._cases import GOLDEN, ROOT

import sys
sys.path.insert(0, GOLDEN)
import make_cli_golden as mk  # noqa: E402

pytestmark = pytest.mark.gpu

BIN = os.path.join(ROOT, "bin")
CLI = os.path.join(GOLDEN, "cli")
WNL = json.load(open(os.path.join(CLI, "wnl_cases.json")))
WAVE_RTOL = 1e-6


def _num_rows(text):
    hdr, rows = [], []
    for ln in text.splitlines():
        if ln.startswith("#") or not ln.strip():
            hdr.append(ln)
        else:
            rows.append([float(x) for x in ln.split("\t")])
    return hdr, np.array(rows)


def _ulp8(a, b):
    m = np.maximum(np.abs(a), np.abs(b))
    with np.errstate(divide="ignore"):
        e = np.floor(np.log10(np.where(m > 0, m, 1.0)))
    return 1.01 * 10.0 ** (e - 7)


def _compare_wave_file(got, ref, rel):
    hg, g = _num_rows(got)
    hr, r = _num_rows(ref)
    errs = []
    if hg != hr:
        errs.append(f"{rel}: header {hg!r} != {hr!r}")
    if g.shape != r.shape:
        return errs + [f"{rel}: shape {g.shape} != {r.shape}"]
    if rel.startswith("sc_spectrum"):
        fcols, vcols = [0], [1, 2]
    elif rel.endswith(".raypaths.dat"):
        return errs + _compare_6digit(got, ref, rel)
    else:
        fcols, vcols = [0], [1]
    for c in fcols:   # time / frequency axis: printed digits
        bad = np.abs(g[:, c] - r[:, c]) > np.maximum(_ulp8(g[:, c], r[:, c]), 1e-9)
        if rel.startswith("sc_"):   # default 6-digit stream there
            bad = np.abs(g[:, c] - r[:, c]) > 1.01e-5 * np.maximum(np.abs(r[:, c]), 1e-300) + 1e-12
        if bad.any():
            i = int(np.argmax(bad))
            errs.append(f"{rel}: col {c} row {i}: {g[i, c]!r} vs {r[i, c]!r} ({int(bad.sum())} rows)")
    scale = max(np.max(np.abs(r[:, vcols])), 1e-300)
    for c in vcols:
        d = np.abs(g[:, c] - r[:, c])
        if np.max(d) > WAVE_RTOL * scale:
            i = int(np.argmax(d))
            errs.append(f"{rel}: col {c} row {i}: {g[i, c]!r} vs {r[i, c]!r} (max |diff| / max |ref| = "
                        f"{np.max(d) / scale:.3g})")
    return errs


def _compare_6digit(got, ref, rel):
    from tests.test_cli_gpu import compare_file
    return compare_file(got, ref, rel)


def _compare_console(got, ref):
    g, r = got.splitlines(), ref.splitlines()
    assert len(g) == len(r), f"{len(g)} console lines, reference {len(r)}:\n" + "\n".join(g[-5:])
    for lg, lr in zip(g, r):
        if "Computing waveform" in lr or "Generating waveform" in lr:
            fg, fr = lg.split("\t"), lr.split("\t")
            assert fg[1] == fr[1], (lg, lr)   # ray length label
            for a, b in zip(fg[2:], fr[2:]):
                ka, va = a.rsplit(":", 1)
                kb, vb = b.rsplit(":", 1)
                assert ka == kb
                x, y = float(va), float(vb)
                assert abs(x - y) <= 1e-5 * abs(y) + 1e-9, (lg, lr)
        elif " = " in lr:
            ka, va = lg.rsplit("=", 1)
            kb, vb = lr.rsplit("=", 1)
            assert ka == kb, (lg, lr)
            x, y = float(va), float(vb)
            m = max(abs(x), abs(y))
            ulp = 10.0 ** (math.floor(math.log10(m)) - 5) if m > 0 else 0.0
            assert abs(x - y) <= 1.01 * ulp + 1e-9, (lg, lr)
        else:
            assert lg == lr, (lg, lr)


@pytest.fixture(scope="module")
def built():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU tests need a CUDA device")
    assert os.path.exists(os.path.join(BIN, "infraga-3d")), "bin/infraga-3d missing: run __graft_entry__.build()"
    return True


@pytest.mark.parametrize("name", sorted(WNL))
def test_wnl_cli_matches_reference(built, name):
    c = WNL[name]
    spec = (c["ref_binary"], c["kind"], c["seed"], c["argv"])
    got, console = mk.run_case_wnl(BIN, spec, binary=c["binary"])
    errs = []
    for rel in c["files"]:
        if rel not in got:
            errs.append(f"{rel}: not written")
            continue
        with open(os.path.join(CLI, name, rel)) as f:
            errs += _compare_wave_file(got[rel], f.read(), rel)
    errs += [f"{rel}: written, not in the reference output" for rel in sorted(set(got) - set(c["files"]))]
    assert not errs, "\n".join(errs[:30])
    with open(os.path.join(CLI, name, "stdout.txt")) as f:
        _compare_console(console, f.read())


def _atmo(seed):
    import infraga_b200 as ig
    return ig.Atmosphere.load(os.path.join(GOLDEN, "profiles", f"gen{seed}.met"))


def _impulse(n=1024, p0=10.0, t0=0.1, alpha=4.0):
    # wvfrm::build_wvfrm "impulse" with N_rise 10, N_period 40 (waveforms.cpp:67-84)
    dur = t0 * n * max(((1 + alpha) - math.sqrt(1 + alpha)) / 10, 2 * 3.14159 * math.sqrt(1 + alpha) / 40)
    t = np.array([-dur / 2 + dur * i / n for i in range(n)])
    x = np.where(t >= 0, t / t0, 0.0)
    xp = (alpha + 1) - math.sqrt(alpha + 1)
    p = np.where(t >= 0, x ** alpha * (1 - x / (1 + alpha)) * np.exp(-x), 0.0)
    p = p0 * p / (xp ** alpha * (1 - xp / (1 + alpha)) * math.exp(-xp))
    return t, p


def test_wnl_batch_equals_single_rays(built):
    """One launch over several rays (one CTA each) gives every ray exactly the
    waveform it gets alone."""
    import infraga_b200 as ig
    atmo = _atmo(0)
    p = ig.wnl_params(atmo, bounces=1)
    t, pw = _impulse(512)
    th = np.array([8.0, 12.0, 20.0, 30.0, 12.0])
    ph = np.array([60.0, 60.0, -30.0, 90.0, 200.0])
    batch = ig.wnl_run(atmo, p, th, ph, t, pw, event_cap=512)
    assert np.all(batch["status"] == 0)
    assert np.all(batch["steps"] > 50)
    for i in range(th.size):
        one = ig.wnl_run(atmo, p, th[i:i + 1], ph[i:i + 1], t, pw, event_cap=512)
        np.testing.assert_array_equal(one["u"][0], batch["u"][i])
        np.testing.assert_array_equal(one["info"][0], batch["info"][i])
        k = int(one["events"][0].shape[0] if one["info"][0][3] > 512 else one["info"][0][3])
        np.testing.assert_array_equal(one["events"][0][:k], batch["events"][i][:k])
        assert not np.any(batch["events"][i][k:])
    atmo.close()


def test_wnl_linear_limit_conserves_shape(built):
    """With a vanishing source amplitude the scheme is linear: scaling p0 by
    10 changes nothing in u = p / p0 beyond the (vanishing) non-linear term,
    the step size stays at its 1 km clamp, and the waveform energy only
    decays (absorption, filters, window)."""
    import infraga_b200 as ig
    atmo = _atmo(1)
    p = ig.wnl_params(atmo)
    t, pw = _impulse(1024, p0=1e-12)
    a = ig.wnl_run(atmo, p, [15.0], [90.0], t, pw)
    b = ig.wnl_run(atmo, p, [15.0], [90.0], t, pw * 10.0)
    assert a["status"][0] == 0 and b["status"][0] == 0
    assert a["steps"][0] == b["steps"][0]
    np.testing.assert_allclose(a["u"][0], b["u"][0], rtol=0, atol=1e-8 * np.max(np.abs(a["u"][0])))
    e0 = np.sum((pw / np.max(np.abs(pw))) ** 2)
    assert np.sum(a["u"][0] ** 2) <= e0 * (1 + 1e-12)
    atmo.close()


def test_wnl_rejects_unsupported(built):
    import infraga_b200 as ig
    atmo = _atmo(0)
    p = ig.wnl_params(atmo)
    t, pw = _impulse(1000)   # not a power of two
    with pytest.raises(ig.IgaError):
        ig.wnl_run(atmo, p, [15.0], [90.0], t, pw)
    atmo.close()

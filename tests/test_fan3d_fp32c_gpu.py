"""FP32-compensated fan (IGA_FP32C) against FP64: the north-star bound --
ground-intercept range within 10 m, travel time within 10 ms, amplitude within
0.1 dB -- on every non-caustic arrival (no caustic passed by the ray up to that
arrival), with zero violations, on every 3D golden case (against the
reference's own output) and on the full 71,520-ray config-1 fan of each of the
four benchmark seeds (against the FP64 kernel, which follows the reference to
1e-9).  Classification flips (arrival count or turning layer) are counted and
must stay rare.  Rays that reach a focusing arrival before their first caustic
are traced again with FP64 auxiliaries (IGA_RAY_AUX_FP64 in their status):
they are counted, must stay a small fraction of the fan, and their arrivals
must follow the FP64 kernel to rounding."""
import numpy as np
import pytest

import infraga_b200 as ig
from infraga_b200 import synth
from tests._cases import case_setup, load_cases, match_arrivals, noncaustic_report, parse_golden, profile_path

pytestmark = pytest.mark.gpu

CASES = {k: v for k, v in load_cases().items() if v["binary"] == "iga_ref_3d" and v["mode"] == "prop"}


@pytest.fixture(scope="module")
def dev():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU tests need a CUDA device")
    ig.lib()
    return torch


def ray_ids(rows, th, ph):
    key = {(a, b): i for i, (a, b) in enumerate(zip(th, ph))}
    return np.array([key[(r[0], r[1])] for r in rows], dtype=np.int64)


@pytest.mark.parametrize("name", sorted(CASES))
def test_fp32c_north_star_bound_on_reference_cases(dev, name):
    """Against the reference's own FP64 output (golden fixtures); the caustic
    count of each arrival comes from the FP64 GPU run, whose arrivals are the
    golden rows (tests/test_fan3d_gpu.py)."""
    c = CASES[name]
    th, ph, p = case_setup(c["args"])
    atmo = ig.Atmosphere.load(profile_path(c["seed"]))
    r64 = ig.fan_run(atmo, atmo.default_params(**p), th, ph, with_aux=True)
    ref, _ = parse_golden(name)
    assert r64["arrivals"].shape == ref.shape
    r32 = ig.fan_run(atmo, atmo.default_params(**p, precision=ig.FP32C), th, ph)
    got, want, aux, flipped = match_arrivals(r32["arrivals"], r32["ray_index"].astype(np.int64), ref,
                                             ray_ids(ref, th, ph), th.size, r64["aux"])
    rep = noncaustic_report(got, want, aux[:, 3], calc_amp=bool(p["calc_amp"]))
    print(name, "flips", flipped.size, rep)
    assert flipped.size <= max(1, th.size // 100), f"classification flips on rays {flipped}"
    assert rep["ok"], rep


@pytest.mark.parametrize("seed", [1, 2, 3, 4])
def test_fp32c_north_star_bound_full_fan(dev, seed):
    """The config-1 fan (596 x 120 = 71,520 rays, 10 bounces, 2000 km) of one
    benchmark seed: zero violations on the non-caustic arrivals."""
    th, ph = synth.fan_angles(0.5, 60.01, 0.1, 0, 357, 3)
    atmo = ig.Atmosphere.load(profile_path(seed))
    kw = dict(bounces=10, rng_max=2000.0, write_rays=0)
    r64 = ig.fan_run(atmo, atmo.default_params(**kw), th, ph, with_aux=True)
    r32 = ig.fan_run(atmo, atmo.default_params(**kw, precision=ig.FP32C), th, ph)
    got, want, aux, flipped = match_arrivals(r32["arrivals"], r32["ray_index"].astype(np.int64), r64["arrivals"],
                                             r64["ray_index"].astype(np.int64), th.size, r64["aux"])
    rep = noncaustic_report(got, want, aux[:, 3])
    steps_rel = abs(r32["total_steps"] - r64["total_steps"]) / r64["total_steps"]
    st = r32["ray_status"]
    redo = (st & ig.RAY_AUX_FP64) != 0
    print(f"seed {seed}: flips {flipped.size} ({100 * flipped.size / th.size:.4f}%) steps rel {steps_rel:.2e} "
          f"re-traced with FP64 auxiliaries {redo.sum()} ({100 * redo.mean():.2f}%)", rep)
    assert rep["n_noncaustic"] > 1000
    assert rep["ok"], rep
    assert flipped.size < 1e-3 * th.size
    assert steps_rel < 1e-4
    # the flag only marks rays: the termination reason is the FP64 kernel's
    assert np.mean((st & 0xFF) == r64["ray_status"]) > 1 - 1e-3
    assert 0 < redo.sum() < 0.03 * th.size
    # a re-traced ray's non-caustic arrivals: FP64 ray equations and auxiliaries
    ids = np.where(redo)[0]
    s32, s64 = np.isin(r32["ray_index"], ids), np.isin(r64["ray_index"], ids)
    g2, w2, x2, _ = match_arrivals(r32["arrivals"][s32], r32["ray_index"][s32].astype(np.int64),
                                   r64["arrivals"][s64], r64["ray_index"][s64].astype(np.int64), th.size,
                                   r64["aux"][s64])
    nc2 = x2[:, 3] == 0
    assert nc2.sum() > 0
    assert np.abs(g2[nc2, 10] - w2[nc2, 10]).max() < 1e-3
    assert np.hypot(g2[nc2, 3] - w2[nc2, 3], g2[nc2, 4] - w2[nc2, 4]).max() < 1e-4


@pytest.mark.parametrize("seed", [1, 2])
def test_fp32c_flagged_form(dev, seed):
    """IGA_FP32C_FLAGGED: the fan kernel alone.  Rays that met a focusing arrival
    carry IGA_RAY_FOCUS (the rays the default form re-traces); every other ray
    is bit-identical to the default form, and the north-star bound holds on
    its non-caustic arrivals."""
    th, ph = synth.fan_angles(0.5, 60.01, 0.1, 0, 357, 3)
    atmo = ig.Atmosphere.load(profile_path(seed))
    kw = dict(bounces=10, rng_max=2000.0, write_rays=0)
    r64 = ig.fan_run(atmo, atmo.default_params(**kw), th, ph, with_aux=True)
    r32 = ig.fan_run(atmo, atmo.default_params(**kw, precision=ig.FP32C), th, ph)
    rf = ig.fan_run(atmo, atmo.default_params(**kw, precision=ig.FP32C_FLAGGED), th, ph)
    redo = (r32["ray_status"] & ig.RAY_AUX_FP64) != 0
    foc = (rf["ray_status"] & ig.RAY_FOCUS) != 0
    np.testing.assert_array_equal(foc, redo)
    np.testing.assert_array_equal(rf["ray_status"] & 0xFF, r32["ray_status"] & 0xFF)
    keep = np.where(~foc)[0]
    s32, sf = np.isin(r32["ray_index"], keep), np.isin(rf["ray_index"], keep)
    np.testing.assert_array_equal(rf["arrivals"][sf], r32["arrivals"][s32])
    s64 = np.isin(r64["ray_index"], keep)
    got, want, aux, flipped = match_arrivals(rf["arrivals"][sf], rf["ray_index"][sf].astype(np.int64),
                                             r64["arrivals"][s64], r64["ray_index"][s64].astype(np.int64), th.size,
                                             r64["aux"][s64])
    rep = noncaustic_report(got, want, aux[:, 3])
    print(f"seed {seed}: flagged {foc.sum()} rays", rep)
    assert rep["ok"], rep

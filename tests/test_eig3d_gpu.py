"""GPU eigenray search (iga_eig_run) against the reference's own
est_eigenray/find_eigenray output (tests/golden/3d_eig_*, written by the
reference with 8 significant digits)."""
import ctypes

import numpy as np
import pytest

import infraga_b200 as ig
from tests._cases import load_cases, parse_golden, profile_path

pytestmark = pytest.mark.gpu

CASES = {k: v for k, v in load_cases().items() if v["mode"] == "eig" and v["binary"] == "iga_ref_3d"}

# The search stops once the ray lands within tolerance (0.1 km) of the
# receiver, so rounding differences can end it one Newton step apart; the
# bounds below are set by that stopping rule, not by the integration.
# Columns: incl, az [deg], n_b, x, y [km], time [s], cel [km/s], turning ht [km],
# arrival incl, back az [deg], amplitude, absorption [dB].
EIG_ATOL = np.array([2e-3, 2e-3, 0, 0.1, 0.1, 0.5, 2e-4, 0.05, 2e-3, 2e-3, 0.2, 0.05])


def eig_setup(args):
    kv = dict(a.split("=", 1) for a in args)
    src = (float(kv.get("src_x", 0.0)), float(kv.get("src_y", 0.0)), float(kv.get("src_alt", 0.0)))
    rcvr = (float(kv.get("rcvr_x", -250.0)), float(kv.get("rcvr_y", 0.0)))
    over = dict(bnc_min=int(kv.get("bnc_min", 0)), bnc_max=int(kv.get("bnc_max", 0)))
    return src, rcvr, over


@pytest.fixture(scope="module")
def dev():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU tests need a CUDA device")
    ig.lib()
    return torch


@pytest.mark.parametrize("name", sorted(CASES))
def test_eigenrays_match_reference(dev, name):
    c = CASES[name]
    src, rcvr, over = eig_setup(c["args"])
    atmo = ig.Atmosphere.load(profile_path(c["seed"]))
    params = ig.eig_params(atmo, **over)
    r = ig.eig_run(atmo, params, [(src, rcvr)])
    ref, _ = parse_golden(name)
    got = r["eigenrays"]
    print(name, "reference", ref.shape[0], "gpu", got.shape[0], "steps", r["total_steps"])
    assert got.shape == ref.shape, (got[:, :3], ref[:, :3])
    d = np.abs(got - ref)
    print("  max |diff| per column:", np.array2string(d.max(axis=0, initial=0.0), precision=3))
    np.testing.assert_array_equal(got[:, 2], ref[:, 2])
    bad = d > EIG_ATOL[None, :] + 1e-7 * np.abs(ref)
    assert not bad.any(), (np.argwhere(bad)[:5], got[bad], ref[bad])
    # every eigenray lands within the search tolerance of the receiver for
    # bounce counts the Newton iteration follows (the reference's Newton loop
    # traces at most one reflection, so n_b >= 2 rows are not eigenrays)
    one = got[:, 2] <= 1
    assert np.all(np.hypot(got[one, 3] - rcvr[0], got[one, 4] - rcvr[1]) < params.tolerance + 1e-9)


def test_eigen_batch_equals_single_pairs(dev):
    """Searching several pairs in one call gives each pair's single-call result."""
    atmo = ig.Atmosphere.load(profile_path(4))
    params = ig.eig_params(atmo, bnc_min=0, bnc_max=1)
    pairs = [((0.0, 0.0, 0.0), (330.0, 90.0)), ((0.0, 0.0, 0.0), (250.0, -40.0)), ((10.0, 5.0, 0.0), (300.0, 60.0))]
    batch = ig.eig_run(atmo, params, pairs)
    for i, p in enumerate(pairs):
        single = ig.eig_run(atmo, params, [p])
        np.testing.assert_array_equal(batch["eigenrays"][batch["pair_index"] == i], single["eigenrays"])


def test_eigen_pair_groups_equal_one_stream(dev):
    """Pair groups searched concurrently on their own streams give exactly the
    single-stream rows, in pair order."""
    atmo = ig.Atmosphere.load(profile_path(0))
    g = np.random.default_rng(5)
    rng, az = g.uniform(150.0, 400.0, 10), g.uniform(0.0, 2 * np.pi, 10)
    pairs = [((0.0, 0.0, 0.0), (float(r * np.cos(a)), float(r * np.sin(a)))) for r, a in zip(rng, az)]
    one = ig.eig_run(atmo, ig.eig_params(atmo, bnc_min=0, bnc_max=1, streams=1), pairs)
    many = ig.eig_run(atmo, ig.eig_params(atmo, bnc_min=0, bnc_max=1, streams=4), pairs)
    assert one["eigenrays"].shape[0] > 0
    np.testing.assert_array_equal(many["eigenrays"], one["eigenrays"])
    np.testing.assert_array_equal(many["pair_index"], one["pair_index"])
    assert many["total_steps"] == one["total_steps"]


# FP32C search: sweep traces in the FP32-compensated kernel (FP64 ray
# equations), Newton and record traces with FP64 auxiliaries, bracket and
# Newton updates in FP64 on the host.  Its eigenrays are the reference's
# within the search tolerance: the Newton iteration stops anywhere within
# 0.1 km of the receiver, so rounding differences of 1e-9 km can end it at a
# slightly different launch angle, and where the amplitude changes fast with
# the launch angle (the middle branch of a triplication, between two
# caustics) the reference's and the FP32C eigenray then differ by up to a few
# dB while both are correct to the search tolerance.  The amplitude is
# therefore checked against an FP64 fan ray launched at the FP32C eigenray's
# own angles (the arithmetic error), and against the reference only in bulk.
FP32C_EIG_TOL = {"incl": 0.05, "az": 0.05, "time": 0.5, "amp_db_same_angle": 0.1, "amp_db_ref": 3.0}


@pytest.mark.parametrize("name", sorted(CASES))
def test_fp32c_eigenrays_match_reference(dev, name):
    c = CASES[name]
    src, rcvr, over = eig_setup(c["args"])
    atmo = ig.Atmosphere.load(profile_path(c["seed"]))
    params = ig.eig_params(atmo, **over)
    params.fan.precision = ig.FP32C
    r = ig.eig_run(atmo, params, [(src, rcvr)])
    ref, _ = parse_golden(name)
    got = r["eigenrays"]
    print(name, "reference", ref.shape[0], "fp32c", got.shape[0])
    for row in ref[ref[:, 2] <= 1]:
        cand = got[got[:, 2] == row[2]]
        assert cand.shape[0] > 0, row[:3]
        j = np.argmin(np.abs(cand[:, 0] - row[0]) + np.abs(cand[:, 1] - row[1]))
        m = cand[j]
        assert abs(m[0] - row[0]) < FP32C_EIG_TOL["incl"] and abs(m[1] - row[1]) < FP32C_EIG_TOL["az"], (m[:3], row[:3])
        assert abs(m[5] - row[5]) < FP32C_EIG_TOL["time"]
        assert abs(m[10] - row[10]) < FP32C_EIG_TOL["amp_db_ref"]
        assert np.hypot(m[3] - rcvr[0], m[4] - rcvr[1]) < params.tolerance + 1e-3
    # every FP32C eigenray against an FP64 ray at its own launch angles
    for m in got:
        pf = ig.FanParams.from_buffer_copy(params.fan)
        pf.precision, pf.bounces, pf.write_rays, pf.calc_amp = ig.FP64, int(m[2]), 0, 1
        pf.src = (ctypes.c_double * 3)(*src)
        f = ig.fan_run(atmo, pf, np.array([m[0]]), np.array([m[1]]))
        a = f["arrivals"][f["arrivals"][:, 2] == m[2]]
        assert a.shape[0] == 1, m[:3]
        assert np.hypot(a[0, 3] - m[3], a[0, 4] - m[4]) < 1e-4, (a[0, 3:5], m[3:5])
        if np.isfinite(a[0, 10]):
            assert abs(a[0, 10] - m[10]) < FP32C_EIG_TOL["amp_db_same_angle"], (a[0, 10], m[10], m[:3])

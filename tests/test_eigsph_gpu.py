"""GPU spherical eigenray search (iga_eig_run with fan.geometry = IGA_GEOM_SPH)
against the reference's own est_eigenray / find_eigenray output for
infraga-sph (tests/golden/sph_eig_*, written by oracle/harness/harness_sph.cpp
with the reference's 8 significant digits)."""
import numpy as np
import pytest

import infraga_b200 as ig
from tests._cases import load_cases, parse_golden, profile_path

pytestmark = pytest.mark.gpu

CASES = {k: v for k, v in load_cases().items() if v["mode"] == "eig" and v["binary"] == "iga_ref_sph"}

# Same stopping-rule bounds as the 3D search (the search ends once the ray
# lands within 0.1 km of the receiver, so rounding can end it one Newton
# step apart); latitude/longitude of the landing point in degrees
# (0.1 km ~ 1e-3 deg).  The amplitude bound is 0.5 dB: one sph_eig_c
# eigenray sits next to a caustic (-78 dB), where the amplitude moves
# ~0.03 dB per 1e-6 deg of launch angle and the two searches stopped
# 9e-6 deg apart (0.23 dB).  Columns: incl, az, n_b, lat, lon, time, cel,
# turning ht, arrival incl, back az, amplitude, absorption.
EIG_ATOL = np.array([2e-3, 2e-3, 0, 1e-3, 1e-3, 0.5, 2e-4, 0.05, 2e-3, 2e-3, 0.5, 0.05])
R_EARTH = 6370.0


def gc_dist(lat1, lon1, lat2, lon2):
    lat1, lon1, lat2, lon2 = map(np.radians, (lat1, lon1, lat2, lon2))
    h = np.sin((lat2 - lat1) / 2) ** 2 + np.cos(lat1) * np.cos(lat2) * np.sin((lon2 - lon1) / 2) ** 2
    return 2.0 * R_EARTH * np.arcsin(np.sqrt(h))


def eig_setup(args):
    kv = dict(a.split("=", 1) for a in args)
    src = (float(kv.get("src_lat", 30.0)), float(kv.get("src_lon", 0.0)), float(kv.get("src_alt", 0.0)))
    rcvr = (float(kv.get("rcvr_lat", 30.0)), float(kv.get("rcvr_lon", -2.5)))
    over = dict(bnc_min=int(kv.get("bnc_min", 0)), bnc_max=int(kv.get("bnc_max", 0)))
    for k in ("incl_min", "incl_max"):
        if k in kv:
            over[k] = float(kv[k])
    return src, rcvr, over


@pytest.fixture(scope="module")
def dev():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU tests need a CUDA device")
    ig.lib()
    return torch


@pytest.mark.parametrize("name", sorted(CASES))
def test_sph_eigenrays_match_reference(dev, name):
    c = CASES[name]
    src, rcvr, over = eig_setup(c["args"])
    atmo = ig.Atmosphere.load(profile_path(c["seed"]))
    params = ig.eig_params(atmo, geometry=ig.GEOM_SPH, **over)
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
    # the spherical Newton iteration follows every bounce: each row is an eigenray
    assert np.all(gc_dist(got[:, 3], got[:, 4], rcvr[0], rcvr[1]) < params.tolerance + 1e-6)


def test_sph_eigen_batch_equals_single_pairs(dev):
    atmo = ig.Atmosphere.load(profile_path(0))
    params = ig.eig_params(atmo, geometry=ig.GEOM_SPH, bnc_min=0, bnc_max=0, incl_min=5.0, incl_max=20.0)
    pairs = [((30.0, 0.0, 0.0), (30.5, 2.5)), ((30.0, 0.0, 0.0), (31.0, 2.0)), ((-20.0, 50.0, 0.0), (-19.5, 52.5))]
    batch = ig.eig_run(atmo, params, pairs)
    for i, p in enumerate(pairs):
        single = ig.eig_run(atmo, params, [p])
        np.testing.assert_array_equal(batch["eigenrays"][batch["pair_index"] == i], single["eigenrays"])


def test_sph_eig_direct_and_fp32c_rejected(dev):
    atmo = ig.Atmosphere.load(profile_path(0))
    params = ig.eig_params(atmo, geometry=ig.GEOM_SPH, bnc_min=0, bnc_max=0, incl_min=10.0, incl_max=13.0)
    res = ig.eig_run(atmo, params, [((30.0, 0.0, 0.0), (30.5, 2.5))])
    assert res["eigenrays"].shape[0] >= 1
    row = res["eigenrays"][0]
    d = ig.eig_direct(atmo, params, (30.0, 0.0, 0.0), (30.5, 2.5), row[0], row[1], 0)
    assert d is not None and gc_dist(d[3], d[4], 30.5, 2.5) < params.tolerance
    params.fan.precision = ig.FP32C
    with pytest.raises(ig.IgaError):
        ig.eig_run(atmo, params, [((30.0, 0.0, 0.0), (30.5, 2.5))])

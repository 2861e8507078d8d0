"""Sampled ray paths, terrain samples and caustics (iga_fan_paths) and the
Newton-only eigenray refinement (iga_eig_direct) through the Python binding.
File-level parity with the reference binaries is in test_cli_gpu.py; these
check the invariants of the sampled output on the golden fans."""
import numpy as np
import pytest

import infraga_b200 as ig
from tests._cases import case_setup, case_setup_sph, load_cases, profile_path

pytestmark = pytest.mark.gpu

CASES = load_cases()


@pytest.fixture(scope="module")
def dev():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU tests need a CUDA device")
    ig.lib()
    return torch


def _setup(name):
    c = CASES[name]
    atmo = ig.Atmosphere.load(profile_path(c["seed"]))
    if c["binary"] == "iga_ref_sph":
        th, ph, p = case_setup_sph(c["args"])
    else:
        th, ph, p = case_setup(c["args"])
    return atmo, th, ph, atmo.default_params(**p)


@pytest.mark.parametrize("name", ["3d_c0_rays", "sph_rays"])
def test_path_rows_follow_each_ray(dev, name):
    atmo, th, ph, params = _setup(name)
    params.write_rays = 1
    fan = ig.fan_run(atmo, params, th, ph)
    out = ig.fan_paths(atmo, params, th, ph, caustics=True, ray_steps=fan["ray_steps"])
    rows, start = out["paths"], out["path_start"]
    assert start[-1] == rows.shape[0] and np.all(np.diff(start) >= 1)
    arr, idx = fan["arrivals"], fan["ray_index"]
    for i in range(th.size):
        r = rows[start[i]:start[i + 1]]
        assert np.all(np.diff(r[:, 5]) > 0.0)          # time grows along the ray
        assert np.all(np.diff(r[:, 6]) >= 0.0)         # bounce index never decreases
        assert np.all(r[:, 4] <= 0.0)                  # -2 x absorption
        for b_row in arr[idx == i]:
            seg = r[r[:, 6] == b_row[2]]
            assert seg.size and seg[-1, 5] <= b_row[5]  # sampled rows precede the arrival
    # caustics: ordered by ray, times inside the ray's sampled span
    cr = out["caustic_ray"]
    assert np.all(np.diff(cr) >= 0)
    # the step-count pass inside the call gives the same rows as the caller's counts
    again = ig.fan_paths(atmo, params, th, ph, caustics=True)
    np.testing.assert_array_equal(again["paths"], rows)
    np.testing.assert_array_equal(again["caustics"], out["caustics"])


def test_terrain_samples_on_flat_ground(dev):
    atmo, th, ph, params = _setup("3d_c0_rays")
    out = ig.fan_paths(atmo, params, th[:3], ph[:3], mode=ig.PATH_TERRAIN)
    assert np.all(out["paths"][:, 2] == params.z_grnd)


def test_eig_direct_reproduces_search_result(dev):
    atmo = ig.Atmosphere.load(profile_path(0))
    p = ig.eig_params(atmo, bnc_min=0, bnc_max=1)
    res = ig.eig_run(atmo, p, [((0.0, 0.0, 0.0), (250.0, 40.0))])
    assert res["eigenrays"].shape[0] > 0
    for row in res["eigenrays"]:
        d = ig.eig_direct(atmo, p, (0.0, 0.0, 0.0), (250.0, 40.0), row[0], row[1], int(row[2]))
        assert d is not None
        assert np.hypot(d[3] - 250.0, d[4] - 40.0) < p.tolerance
        assert abs(d[0] - row[0]) < 0.05 and abs(d[1] - row[1]) < 0.05


def test_paths_reject_fp32c_and_caustics_without_amp(dev):
    atmo, th, ph, params = _setup("3d_c0_rays")
    params.precision = ig.FP32C
    with pytest.raises(ig.IgaError):
        ig.fan_paths(atmo, params, th[:2], ph[:2], ray_steps=np.array([10, 10]))
    params.precision = ig.FP64
    params.calc_amp = 0
    with pytest.raises(ig.IgaError):
        ig.fan_paths(atmo, params, th[:2], ph[:2], caustics=True, ray_steps=np.array([10, 10]))


def test_projection_rows_match_fan_and_reject_other_solvers(dev):
    """IGA_PATH_PROJ (-back_proj rows): 15 columns, time growing along the ray,
    the last row before each arrival at most the arrival time; other handles,
    caustics and calc_amp = 0 are refused.  File-level parity with the
    reference's .projection.dat is in test_cli_gpu.py (3d_back_proj*)."""
    atmo = ig.Atmosphere.load(profile_path(0), reverse_winds=True)
    params = atmo.default_params(bounces=1, src=(10.0, 0.0, 0.0), turn_ht_min=-1e30)
    params.write_rays = 1
    th, ph = np.array([12.0]), np.array([60.0])
    fan = ig.fan_run(atmo, params, th, ph)
    rows = ig.fan_paths(atmo, params, th, ph, mode=ig.PATH_PROJ, ray_steps=fan["ray_steps"])["paths"]
    assert rows.shape[1] == ig.PROJ_COLS and rows.shape[0] > 10
    assert np.all(np.diff(rows[:, 3]) > 0.0) and np.all(rows[:, 2] >= 0.0)
    assert rows[-1, 3] <= fan["arrivals"][-1, 5]
    with pytest.raises(ig.IgaError):
        ig.fan_paths(atmo, params, th, ph, mode=ig.PATH_PROJ, caustics=True, ray_steps=fan["ray_steps"])
    params.calc_amp = 0
    with pytest.raises(ig.IgaError):
        ig.fan_paths(atmo, params, th, ph, mode=ig.PATH_PROJ, ray_steps=fan["ray_steps"])
    sph = atmo.default_params(geometry=ig.GEOM_SPH)
    with pytest.raises(ig.IgaError):
        ig.fan_paths(atmo, sph, th, ph, mode=ig.PATH_PROJ, ray_steps=np.array([100]))

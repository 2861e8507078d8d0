"""GPU parity of the spherical (global) stratified ray fan (FP64) through the
C ABI, against the reference's own full-precision output (tests/golden,
written by oracle/harness/harness_sph.cpp around the unmodified infraga-sph
solver)."""
import ctypes

import numpy as np
import pytest

import infraga_b200 as ig
from tests._cases import SPH_ATOL, FP64_RTOL, case_setup_sph, compare_arrivals, load_cases, parse_golden, profile_path

pytestmark = pytest.mark.gpu

CASES = {k: v for k, v in load_cases().items() if v["binary"] == "iga_ref_sph" and v["mode"] == "prop"}


@pytest.fixture(scope="module")
def dev():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU tests need a CUDA device")
    ig.lib()
    return torch


def run_case(args, seed, with_aux=False, **over):
    th, ph, p = case_setup_sph(args)
    p.update(over)
    atmo = ig.Atmosphere.load(profile_path(seed))
    params = atmo.default_params(**p)
    return th, ph, params, atmo, ig.fan_run(atmo, params, th, ph, with_aux=with_aux)


@pytest.mark.parametrize("name", sorted(CASES))
def test_sph_fan_matches_reference_golden(dev, name):
    c = CASES[name]
    th, ph, params, atmo, r = run_case(c["args"], c["seed"])
    ref, ref_steps = parse_golden(name)
    np.testing.assert_array_equal(r["ray_steps"], ref_steps)
    ok, msg = compare_arrivals(r["arrivals"], ref, atol=SPH_ATOL, rtol=FP64_RTOL)
    print(name, msg)
    assert ok, msg
    assert r["total_steps"] == int(ref_steps.sum())


def test_sph_ray_order_and_repeat_invariance(dev):
    """Each ray's result depends only on that ray: a shuffled fan gives the
    same per-ray rows, and a repeated run is bit-identical."""
    c = CASES["sph_rays"]
    th, ph, params, atmo, r = run_case(c["args"], c["seed"])
    r2 = ig.fan_run(atmo, params, th, ph)
    np.testing.assert_array_equal(r["arrivals"], r2["arrivals"])
    perm = np.random.default_rng(3).permutation(th.size)
    rp = ig.fan_run(atmo, params, th[perm], ph[perm])
    np.testing.assert_array_equal(rp["ray_steps"], r["ray_steps"][perm])
    for new_i, old_i in enumerate(perm):
        a = r["arrivals"][r["ray_index"] == old_i]
        b = rp["arrivals"][rp["ray_index"] == new_i]
        np.testing.assert_array_equal(a, b)


def test_sph_noamp_paths_equal_amp_paths(dev):
    """The 6 ray equations do not depend on the 12 auxiliary ones: without
    amplitudes every column but the transmission coefficient is unchanged."""
    c = CASES["sph_c0_bulk"]
    th, ph, params, atmo, r = run_case(c["args"], c["seed"])
    params.calc_amp = 0
    r0 = ig.fan_run(atmo, params, th, ph)
    np.testing.assert_array_equal(r0["ray_steps"], r["ray_steps"])
    cols = [i for i in range(12) if i != 10]
    np.testing.assert_array_equal(r0["arrivals"][:, cols], r["arrivals"][:, cols])
    assert np.all(r0["arrivals"][:, 10] == 0.0)


def test_sph_device_entry_matches_host_entry(dev):
    torch = dev
    c = CASES["sph_elevated"]
    th, ph, params, atmo, r = run_case(c["args"], c["seed"])
    n = th.size
    nb = params.bounces + 1
    d_th = torch.tensor(th, dtype=torch.float64, device="cuda")
    d_ph = torch.tensor(ph, dtype=torch.float64, device="cuda")
    d_arr = torch.zeros((n, nb, 12), dtype=torch.float64, device="cuda")
    d_n = torch.zeros(n, dtype=torch.int32, device="cuda")
    d_steps = torch.zeros(n, dtype=torch.int64, device="cuda")
    d_ws = torch.zeros(ig.fan_workspace_bytes(), dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream()
    ig.fan_run_device(atmo, params, d_th.data_ptr(), d_ph.data_ptr(), n, d_arr.data_ptr(), d_n.data_ptr(),
                      d_steps.data_ptr(), 0, d_ws.data_ptr(), stream.cuda_stream)
    torch.cuda.synchronize()
    rows = np.concatenate([d_arr[i, : int(d_n[i])].cpu().numpy() for i in range(n)])
    np.testing.assert_array_equal(rows, r["arrivals"])
    np.testing.assert_array_equal(d_steps.cpu().numpy(), r["ray_steps"])


def test_sph_status_codes(dev):
    """Termination reasons of the edge-case fixtures: travel-time cap and
    region limits (sph_limits), and every ray of a fan has a status."""
    c = CASES["sph_limits"]
    th, ph, params, atmo, r = run_case(c["args"], c["seed"])
    st = r["ray_status"]
    assert set(np.unique(st)).issubset(set(ig.RAY_STATUS))
    assert (st == 1).any()          # left the lat/lon box
    # a short time cap ends long multi-bounce rays at the bounce that exceeds it
    params.time_max = 0.05
    rt = ig.fan_run(atmo, params, th, ph)
    assert (rt["ray_status"] == 6).any()
    assert np.all(rt["arrivals"][:, 5] / 3600.0 <= 0.05)


def test_sph_aux_columns(dev):
    """Per-arrival diagnostics are finite where amplitudes are, the Jacobian
    sign agrees with the amplitude's |D|, and caustic counts never decrease
    along a ray."""
    c = CASES["sph_c0_bulk"]
    th, ph, params, atmo, r = run_case(c["args"], c["seed"], with_aux=True)
    aux = r["aux"]
    assert aux.shape == (r["arrivals"].shape[0], 4)
    assert np.all(np.isfinite(aux[:, :3]))
    assert np.all(aux[:, 0] > 0.0)
    for i in np.unique(r["ray_index"]):
        cnt = aux[r["ray_index"] == i, 3]
        assert np.all(np.diff(cnt) >= 0)


def test_sph_rejects_fp32c_and_bad_latitude(dev):
    atmo = ig.Atmosphere.load(profile_path(0))
    p = atmo.default_params(geometry=ig.GEOM_SPH, precision=ig.FP32C)
    with pytest.raises(ig.IgaError):
        ig.fan_run(atmo, p, np.array([10.0]), np.array([90.0]))
    p = atmo.default_params(geometry=ig.GEOM_SPH, src=(91.0, 0.0, 0.0))
    with pytest.raises(ig.IgaError):
        ig.fan_run(atmo, p, np.array([10.0]), np.array([90.0]))


def test_sph_defaults_follow_infraga_sph(dev):
    atmo = ig.Atmosphere.load(profile_path(0))
    p = atmo.default_params(geometry=ig.GEOM_SPH)
    assert p.geometry == ig.GEOM_SPH
    assert tuple(p.src) == (30.0, 0.0, 0.0)
    assert p.rng_max == 1000.0 and p.time_max == 10.0
    assert (p.lat_min, p.lat_max, p.lon_min, p.lon_max) == (-90.0, 90.0, -180.0, 180.0)

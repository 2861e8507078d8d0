"""FP32-compensated spherical range-dependent fan (IGA_FP32C on a node grid,
fansphr_fp32c.cu) against FP64: the north-star bound -- ground-intercept range
within 10 m, travel time within 10 ms, amplitude within 0.1 dB -- on every
non-caustic arrival (no caustic passed up to it, counted by the FP64 run),
with zero violations, on the reference's own golden cases and on the config-2
workload (21 x 21 node grid, 0.05-deg fractal terrain, 14,328 rays, 20
bounces, 3000 km) against the FP64 kernel.  Rays re-traced with FP64
auxiliaries after a focusing arrival are counted and must stay few."""
import numpy as np
import pytest

import infraga_b200 as ig
from infraga_b200 import workloads as wl
from tests._cases import golden_angles, match_arrivals, noncaustic_report, parse_golden
from tests.test_fansphr_gpu import CASES, atmo, params_for

pytestmark = pytest.mark.gpu

R_EARTH = 6370.0


@pytest.fixture(scope="module")
def dev():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU tests need a CUDA device")
    ig.lib()
    return torch


def as_km(rows):
    """Arrival rows with lat/lon [deg] replaced by ground distances [km] from
    the first row's point: the bound is on the intercept range in km."""
    out = rows.copy()
    lat, lon = np.radians(rows[:, 3]), np.radians(rows[:, 4])
    out[:, 3] = R_EARTH * lat
    out[:, 4] = R_EARTH * np.cos(lat) * lon
    return out


def ray_ids(rows, th, ph):
    key = {(a, b): i for i, (a, b) in enumerate(zip(th, ph))}
    return np.array([key[(r[0], r[1])] for r in rows], dtype=np.int64)


def check(r32, r64, n_rays, calc_amp=True):
    got, want, aux, flipped = match_arrivals(as_km(r32["arrivals"]), r32["ray_index"].astype(np.int64),
                                             as_km(r64["arrivals"]), r64["ray_index"].astype(np.int64), n_rays,
                                             r64["aux"])
    rep = noncaustic_report(got, want, aux[:, 3], calc_amp=calc_amp)
    redo = (r32["ray_status"] & ig.RAY_AUX_FP64) != 0
    return rep, flipped, redo


@pytest.mark.parametrize("name", sorted(CASES))
def test_sphr_fp32c_bound_on_reference_cases(dev, name):
    topo = any(x.startswith("topo_file=") for x in CASES[name]["args"])
    a = atmo(topo)
    p = params_for(name, a)
    p.write_rays = 0
    th, ph = golden_angles(name)
    r64 = ig.fan_run(a, p, th, ph, with_aux=True)
    ref, _ = parse_golden(name)
    assert r64["arrivals"].shape == ref.shape
    p.precision = ig.FP32C
    r32 = ig.fan_run(a, p, th, ph)
    rep, flipped, redo = check(r32, r64, th.size, calc_amp=bool(p.calc_amp))
    print(name, "flips", flipped.size, "re-traced", redo.sum(), rep)
    assert flipped.size <= max(1, th.size // 100)
    assert rep["ok"], rep


def test_sphr_fp32c_bound_config2(dev):
    files = wl.sphr_files()
    a = ig.Atmosphere.load_rngdep(files[0], files[1], files[2], topo_file=files[3], geometry=ig.GEOM_SPH)
    th, ph = wl.sphr_angles()
    f = wl.SPHR_FAN
    kw = dict(geometry=ig.GEOM_SPH, bounces=f["bounces"], rng_max=f["rng_max"], write_rays=0)
    r64 = ig.fan_run(a, a.default_params(**kw), th, ph, with_aux=True)
    r32 = ig.fan_run(a, a.default_params(**kw, precision=ig.FP32C), th, ph)
    rep, flipped, redo = check(r32, r64, th.size)
    steps_rel = abs(r32["total_steps"] - r64["total_steps"]) / r64["total_steps"]
    print(f"config 2: rays {th.size} flips {flipped.size} re-traced {redo.sum()} steps rel {steps_rel:.2e}", rep)
    assert rep["n_noncaustic"] > 1000
    assert rep["ok"], rep
    assert flipped.size < 2e-3 * th.size
    assert redo.sum() < 0.05 * th.size
    assert steps_rel < 1e-3
    a.close()

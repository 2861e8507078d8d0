"""GPU parity of the spherical range-dependent ray fan (hybrid 3D atmosphere
splines, flat ground or terrain; FP64) through the C ABI, against the
reference's own full-precision output (tests/golden, written by
oracle/harness/harness_sphr.cpp around the unmodified infraga-sph-rngdep
solver)."""
import os

import numpy as np
import pytest

import infraga_b200 as ig
from tests._cases import (FP64_RTOL, GOLDEN, SPH_ATOL, compare_arrivals, golden_angles, golden_src, load_cases,
                          parse_golden)

pytestmark = pytest.mark.gpu

CASES = {k: v for k, v in load_cases().items() if v["binary"] == "iga_ref_sphr"}
RNG = os.path.join(GOLDEN, "rngdep")
FILES = (os.path.join(RNG, "node"), os.path.join(RNG, "node_lat.dat"), os.path.join(RNG, "node_lon.dat"))
TOPO = os.path.join(RNG, "topo.dat")

# Range-dependent tolerances: the node tables combine the reference's
# per-evaluation finite differences ahead of time (same arithmetic in a
# different order), which moves results by ~1e-12 relative per evaluation.
RD_ATOL = SPH_ATOL.copy()


@pytest.fixture(scope="module")
def dev():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU tests need a CUDA device")
    ig.lib()
    return torch


_ATMO = {}


def atmo(topo: bool):
    if topo not in _ATMO:
        _ATMO[topo] = ig.Atmosphere.load_rngdep(*FILES, topo_file=TOPO if topo else None)
    return _ATMO[topo]


def params_for(name, a):
    kv = dict(x.split("=", 1) for x in CASES[name]["args"])
    p = a.default_params(geometry=ig.GEOM_SPH)
    p.src = type(p.src)(*golden_src(name))
    p.write_rays = int(kv.get("write_rays", "true") == "true")
    p.calc_amp = int(kv.get("calc_amp", "true") == "true")
    p.bounces = int(kv.get("bounces", 2))
    return p


@pytest.mark.parametrize("name", sorted(CASES))
def test_sphr_fan_matches_reference_golden(dev, name):
    topo = any(x.startswith("topo_file=") for x in CASES[name]["args"])
    a = atmo(topo)
    p = params_for(name, a)
    th, ph = golden_angles(name)
    r = ig.fan_run(a, p, th, ph)
    ref, ref_steps = parse_golden(name)
    np.testing.assert_array_equal(r["ray_steps"], ref_steps)
    ok, msg = compare_arrivals(r["arrivals"], ref, atol=RD_ATOL, rtol=FP64_RTOL)
    print(name, msg)
    assert ok, msg


def test_sphr_region_and_defaults(dev):
    a = atmo(True)
    lat0, lat1, lon0, lon1 = a.region()
    assert abs(lat0 - 30.001) < 1e-9 and abs(lat1 - 35.999) < 1e-9
    assert abs(lon0 - (-109.999)) < 1e-9 and abs(lon1 - (-104.001)) < 1e-9
    p = a.default_params(geometry=ig.GEOM_SPH)
    assert p.bounces == 2
    assert abs(p.src[0] - 33.0) < 1e-9 and abs(p.src[1] - (-107.0)) < 1e-9


def test_sphr_rejects_unsupported(dev):
    a = atmo(False)
    for over in (dict(geometry=ig.GEOM_3D),):
        p = a.default_params(**over)
        with pytest.raises(ig.IgaError):
            ig.fan_run(a, p, np.array([10.0]), np.array([90.0]))


def test_sphr_repeat_is_bit_identical(dev):
    a = atmo(True)
    p = params_for("sphr_topo", a)
    th, ph = golden_angles("sphr_topo")
    r1 = ig.fan_run(a, p, th, ph)
    r2 = ig.fan_run(a, p, th[::-1].copy(), ph[::-1].copy())
    np.testing.assert_array_equal(r1["ray_steps"], r2["ray_steps"][::-1])
    for i in range(th.size):
        np.testing.assert_array_equal(r1["arrivals"][r1["ray_index"] == i],
                                      r2["arrivals"][r2["ray_index"] == th.size - 1 - i])

"""GPU parity of the 3D Cartesian range-dependent ray fan (hybrid 3D
atmosphere splines on an x/y grid in km, flat ground or terrain; FP64)
through the C ABI, against the reference's own full-precision output
(tests/golden, written by oracle/harness/harness_3dr.cpp around the unmodified
infraga-3d-rngdep solver)."""
import os

import numpy as np
import pytest

import infraga_b200 as ig
from tests._cases import (FP64_ATOL, FP64_RTOL, GOLDEN, compare_arrivals, golden_angles, golden_src, load_cases,
                          parse_golden)

pytestmark = pytest.mark.gpu

CASES = {k: v for k, v in load_cases().items() if v["binary"] == "iga_ref_3dr"}
RNG = os.path.join(GOLDEN, "rngdep3d")
FILES = (os.path.join(RNG, "node"), os.path.join(RNG, "node_x.dat"), os.path.join(RNG, "node_y.dat"))
TOPO = os.path.join(RNG, "topo.dat")


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
        _ATMO[topo] = ig.Atmosphere.load_rngdep(*FILES, topo_file=TOPO if topo else None, geometry=ig.GEOM_3D)
    return _ATMO[topo]


def params_for(name, a):
    kv = dict(x.split("=", 1) for x in CASES[name]["args"])
    p = a.default_params(geometry=ig.GEOM_3D)
    p.src = type(p.src)(*golden_src(name))
    p.write_rays = int(kv.get("write_rays", "true") == "true")
    p.calc_amp = int(kv.get("calc_amp", "true") == "true")
    p.bounces = int(kv.get("bounces", 10))
    return p


@pytest.mark.parametrize("name", sorted(CASES))
def test_3dr_fan_matches_reference_golden(dev, name):
    topo = any(x.startswith("topo_file=") for x in CASES[name]["args"])
    a = atmo(topo)
    p = params_for(name, a)
    th, ph = golden_angles(name)
    r = ig.fan_run(a, p, th, ph)
    ref, ref_steps = parse_golden(name)
    np.testing.assert_array_equal(r["ray_steps"], ref_steps)
    ok, msg = compare_arrivals(r["arrivals"], ref, atol=FP64_ATOL, rtol=FP64_RTOL)
    print(name, msg)
    assert ok, msg


def test_3dr_region_and_defaults(dev):
    a = atmo(True)
    x0, x1, y0, y1 = a.region()
    assert abs(x0 - (-299.999)) < 1e-9 and abs(x1 - 299.999) < 1e-9
    assert abs(y0 - (-299.999)) < 1e-9 and abs(y1 - 299.999) < 1e-9
    p = a.default_params(geometry=ig.GEOM_3D)
    assert (p.x_min, p.x_max, p.y_min, p.y_max) == (x0, x1, y0, y1)
    assert p.src[0] == 0.0 and p.src[1] == 0.0 and p.rng_max == 1000.0 and p.bounces == 10


def test_3dr_rejects_other_geometry(dev):
    a = atmo(False)
    p = a.default_params(geometry=ig.GEOM_SPH)
    with pytest.raises(ig.IgaError):
        ig.fan_run(a, p, np.array([10.0]), np.array([90.0]))


def test_3dr_aux_consistent_with_amplitude(dev):
    """|D| from the diagnostics reproduces the amplitude's Jacobian: rays with
    larger |d(x,y)/d incl| spread more and arrive weaker, and caustic counts
    never decrease along a ray."""
    a = atmo(True)
    p = params_for("3dr_topo", a)
    th, ph = golden_angles("3dr_topo")
    r = ig.fan_run(a, p, th, ph, with_aux=True)
    aux = r["aux"]
    assert np.all(np.isfinite(aux)) and np.all(aux[:, 0] > 0)
    for i in np.unique(r["ray_index"]):
        assert np.all(np.diff(aux[r["ray_index"] == i, 3]) >= 0)

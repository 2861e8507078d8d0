"""Launch shape: every fan kernel gives bit-identical results for every CTA
size the autotuner may pick (a ray's arithmetic does not depend on which
thread or CTA traces it), and iga_fan_tune returns one of its candidates
with a time for each."""
import os

import numpy as np
import pytest

import infraga_b200 as ig
from infraga_b200 import synth
from tests._cases import GOLDEN, profile_path

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dev():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU tests need a CUDA device")
    ig.lib()
    return torch


def fans():
    th, ph = synth.fan_angles(1.0, 45.0, 2.0, 0.0, 300.0, 60.0)
    a3 = ig.Atmosphere.load(profile_path(0))
    yield "3d-fp64", a3, a3.default_params(bounces=3, rng_max=800.0), th, ph
    yield "3d-fp32c", a3, a3.default_params(bounces=3, rng_max=800.0, precision=ig.FP32C), th, ph
    yield "sph", a3, a3.default_params(geometry=ig.GEOM_SPH, bounces=2, rng_max=800.0), th, ph
    d = os.path.join(GOLDEN, "rngdep3d")
    r3 = ig.Atmosphere.load_rngdep(os.path.join(d, "node"), os.path.join(d, "node_x.dat"), os.path.join(d, "node_y.dat"),
                                   topo_file=os.path.join(d, "topo.dat"), geometry=ig.GEOM_3D)
    yield "3dr", r3, r3.default_params(bounces=2, rng_max=500.0), th, ph
    d = os.path.join(GOLDEN, "rngdep")
    rs = ig.Atmosphere.load_rngdep(os.path.join(d, "node"), os.path.join(d, "node_lat.dat"),
                                   os.path.join(d, "node_lon.dat"), topo_file=os.path.join(d, "topo.dat"))
    yield "sphr", rs, rs.default_params(geometry=ig.GEOM_SPH, bounces=2, rng_max=500.0), th, ph


def test_block_sizes_give_identical_fans(dev):
    for name, atmo, p, th, ph in fans():
        ref = None
        for block in (0, 32, 64, 96, 128):
            p.block = block
            r = ig.fan_run(atmo, p, th, ph)
            if ref is None:
                ref = r
                assert r["arrivals"].shape[0] > 0, name
                continue
            np.testing.assert_array_equal(r["arrivals"], ref["arrivals"], err_msg=f"{name} block {block}")
            np.testing.assert_array_equal(r["ray_steps"], ref["ray_steps"], err_msg=f"{name} block {block}")


def test_tuner_picks_a_candidate(dev):
    for name, atmo, p, th, ph in fans():
        p.block = 0
        best, secs = ig.fan_tune(atmo, p, th, ph)
        assert best in (32, 64, 96, 128), name
        assert all(t > 0.0 for t in secs.values()), (name, secs)
        assert secs[best] == min(secs.values())


def test_invalid_block_rejected(dev):
    atmo = ig.Atmosphere.load(profile_path(0))
    p = atmo.default_params()
    for bad in (16, 48, 160, -32):
        p.block = bad
        with pytest.raises(ig.IgaError):
            ig.fan_run(atmo, p, np.array([10.0]), np.array([90.0]))

"""Synthetic workload generator: deterministic profiles and the reference's
launch-angle enumeration (main.infraga.3d.cpp:407-421)."""
import os
import tempfile

import numpy as np

from infraga_b200 import synth
from tests._cases import profile_path


def test_profiles_regenerate_identically():
    with tempfile.TemporaryDirectory() as d:
        for seed in range(5):
            p = synth.write_met(os.path.join(d, f"g{seed}.met"), seed)
            assert open(p).read() == open(profile_path(seed)).read()


def test_profile_shape_and_units():
    z, T, u, v, rho, p = synth.profile_columns(0)
    assert z.size == 751 and z[0] == 0.0 and abs(z[-1] - 150.0) < 1e-12
    c = np.sqrt(0.1 * 1.4 * p / rho)          # m/s, the reference's conversion
    np.testing.assert_allclose(c, np.sqrt(1.4 * 287.058 * T), rtol=1e-12)
    assert abs(np.sqrt(np.mean((v) ** 2)) - 5.0) < 2.0


def test_fan_counts():
    th, ph = synth.fan_angles(0.5, 60.0, 0.1, 0, 357, 3)
    assert th.size == 595 * 120                # FP64 accumulation stops at 59.9000000000006
    th, ph = synth.fan_angles(0.5, 60.01, 0.1, 0, 357, 3)
    assert th.size == 596 * 120 == 71520
    assert th[595] == th[-1] and abs(th[-1] - 60.0) < 1e-9
    th, ph = synth.fan_angles(1, 45, 1, 90, 90, 1)
    assert th.size == 45
    th, _ = synth.fan_angles(-30, 30, 5, 45, 45, 1, src_above_ground=True)
    assert th[0] == -30 and th.size == 13
    th, _ = synth.fan_angles(-30, 30, 5, 45, 45, 1, src_above_ground=False)
    assert th[0] == 0.1

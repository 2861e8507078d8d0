"""infraga-3d's and infraga-sph's stratified profiles over terrain
(iga_atmo_load_topo): the eigenray searches against the reference binaries'
own tables (tests/golden/cli/3dt_eig and spht_eig, written by
tests/golden/make_cli_golden.py; the fan and file outputs are compared in
test_cli_gpu.py), and a flat terrain against the flat-ground stratified
solvers, which share no kernel with the terrain ones."""
import os

import numpy as np
import pytest

import infraga_b200 as ig
from tests._cases import GOLDEN, profile_path

pytestmark = pytest.mark.gpu

CLI = os.path.join(GOLDEN, "cli")
TOPO = os.path.join(GOLDEN, "rngdep3d", "topo.dat")
TOPO_SPH = os.path.join(GOLDEN, "rngdep", "topo.dat")
# stopping-rule bounds of the other eigenray searches (tests/test_eigrngdep_gpu.py);
# 3D columns 3-4 in km, spherical in degrees
ATOL_3D = np.array([2e-3, 2e-3, 0, 0.1, 0.1, 0.5, 2e-4, 0.05, 2e-3, 2e-3, 0.5, 0.05])
ATOL_SPH = np.array([2e-3, 2e-3, 0, 1e-3, 1e-3, 0.5, 2e-4, 0.05, 2e-3, 2e-3, 0.5, 0.05])


@pytest.fixture(scope="module")
def dev():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU tests need a CUDA device")
    ig.lib()
    return torch


def rows_of(path):
    rows = [[float(x) for x in ln.split("\t")] for ln in open(path) if ln.strip() and not ln.startswith("#")]
    return np.array(rows, dtype=np.float64).reshape(-1, 12)


def check(got, ref, atol):
    print("reference", ref.shape[0], "gpu", got.shape[0])
    assert got.shape == ref.shape, (got[:, :3], ref[:, :3])
    np.testing.assert_array_equal(got[:, 2], ref[:, 2])
    d = np.abs(got - ref)
    print("  max |diff| per column:", np.array2string(d.max(axis=0, initial=0.0), precision=3))
    bad = d > atol[None, :] + 1e-7 * np.abs(ref)
    assert not bad.any(), (np.argwhere(bad)[:5], got[bad], ref[bad])


def centre(atmo):
    a0, a1, b0, b1 = atmo.region()
    return (a1 + a0) / 2.0, (b1 + b0) / 2.0


def test_eigenrays_over_terrain_match_reference(dev):
    atmo = ig.Atmosphere.load_topo(profile_path(0), TOPO)
    x, y = centre(atmo)
    p = ig.eig_params(atmo, incl_min=14.0, incl_max=28.0, bnc_min=0, bnc_max=1)
    got = ig.eig_run(atmo, p, [((x, y, 0.0), (240.0, 0.0))])["eigenrays"]
    check(got, rows_of(os.path.join(CLI, "3dt_eig", "atmo.arrivals.dat")), ATOL_3D)
    assert np.all(np.hypot(got[:, 3] - 240.0, got[:, 4]) < p.tolerance + 1e-6)


def test_sph_eigenrays_over_terrain_match_reference(dev):
    atmo = ig.Atmosphere.load_topo(profile_path(0), TOPO_SPH, geometry=ig.GEOM_SPH)
    lat, lon = centre(atmo)
    p = ig.eig_params(atmo, incl_min=10.0, incl_max=30.0)
    assert p.fan.geometry == ig.GEOM_SPH
    got = ig.eig_run(atmo, p, [((lat, lon, 3.0), (32.98, -104.6))])["eigenrays"]
    check(got, rows_of(os.path.join(CLI, "spht_eig", "atmo.arrivals.dat")), ATOL_SPH)


@pytest.mark.parametrize("calc_amp", [1, 0])
def test_flat_terrain_matches_flat_ground(dev, tmp_path, calc_amp):
    """Terrain at z = 0 everywhere against the flat-ground solver at z_grnd = 0.
    The terrain solver puts its ground-check ceiling 0.1 km and its
    boundary-layer top 2.1 km above the terrain maximum where the flat one has
    0 and 2 km (topo::set_bndlyr of each), which moves the 2.0-2.1 km steps by
    ~1e-6 of ds and the winds there by ~1e-9: the arrivals agree to ~1e-6."""
    xs = np.linspace(-500.0, 500.0, 11)
    with open(tmp_path / "flat.dat", "w") as f:
        for x in xs:
            for y in xs:
                f.write(f"{x:.6f}\t{y:.6f}\t0.0\n")
    flat = ig.Atmosphere.load(profile_path(1))
    topo = ig.Atmosphere.load_topo(profile_path(1), str(tmp_path / "flat.dat"))
    th = np.repeat(np.arange(4.0, 40.0, 3.0), 3)
    ph = np.tile([30.0, 100.0, -135.0], th.size // 3)
    pf = flat.default_params(bounces=2, calc_amp=calc_amp, rng_max=450.0, src=(0.0, 0.0, 0.0), turn_ht_min=-1.0)
    pt = topo.default_params(bounces=2, calc_amp=calc_amp, rng_max=450.0, src=(0.0, 0.0, 0.0), turn_ht_min=-1.0)
    a = ig.fan_run(flat, pf, th, ph)
    b = ig.fan_run(topo, pt, th, ph)
    ka = {tuple(r[:3]): r for r in a["arrivals"]}
    kb = {tuple(r[:3]): r for r in b["arrivals"]}
    assert len(ka) > 20 and set(ka) == set(kb)
    tol = np.array([0, 0, 0, 1e-3, 1e-3, 1e-3, 1e-6, 1e-3, 1e-4, 1e-4, 1e-2, 1e-3])
    worst = np.zeros(12)
    for k, ra in ka.items():
        worst = np.maximum(worst, np.abs(kb[k] - ra))
    print("max |diff| per column:", np.array2string(worst, precision=3))
    assert np.all(worst <= tol)


@pytest.mark.parametrize("calc_amp", [1, 0])
def test_sph_flat_terrain_matches_flat_ground(dev, tmp_path, calc_amp):
    """As above on the globe: terrain at 0 km over 20-46 N, 120-94 W against
    infraga-sph's flat ground (ceilings 0.01 and 2.01 km against 0 and 2)."""
    with open(tmp_path / "flat.dat", "w") as f:
        for la in np.linspace(20.0, 46.0, 14):
            for lo in np.linspace(-120.0, -94.0, 14):
                f.write(f"{la:.6f}\t{lo:.6f}\t0.0\n")
    flat = ig.Atmosphere.load(profile_path(1))
    topo = ig.Atmosphere.load_topo(profile_path(1), str(tmp_path / "flat.dat"), geometry=ig.GEOM_SPH)
    th = np.repeat(np.arange(4.0, 40.0, 3.0), 3)
    ph = np.tile([30.0, 100.0, -135.0], th.size // 3)
    kw = dict(bounces=2, calc_amp=calc_amp, rng_max=450.0, src=(33.0, -107.0, 0.0), turn_ht_min=-1.0)
    a = ig.fan_run(flat, flat.default_params(geometry=ig.GEOM_SPH, **kw), th, ph)
    b = ig.fan_run(topo, topo.default_params(geometry=ig.GEOM_SPH, **kw), th, ph)
    ka = {tuple(r[:3]): r for r in a["arrivals"]}
    kb = {tuple(r[:3]): r for r in b["arrivals"]}
    assert len(ka) > 20 and set(ka) == set(kb)
    tol = np.array([0, 0, 0, 1e-5, 1e-5, 1e-3, 1e-6, 1e-3, 1e-4, 1e-4, 1e-2, 1e-3])
    worst = np.zeros(12)
    for k, ra in ka.items():
        worst = np.maximum(worst, np.abs(kb[k] - ra))
    print("max |diff| per column:", np.array2string(worst, precision=3))
    assert np.all(worst <= tol)


def test_topo_handles_are_fp64_only(dev):
    for path, geom in ((TOPO, ig.GEOM_3D), (TOPO_SPH, ig.GEOM_SPH)):
        atmo = ig.Atmosphere.load_topo(profile_path(0), path, geometry=geom)
        p = atmo.default_params(geometry=geom, precision=ig.FP32C)
        with pytest.raises(ig.IgaError):
            ig.fan_run(atmo, p, np.array([10.0]), np.array([90.0]))

"""GPU eigenray search on the range-dependent solvers with terrain (iga_eig_run
on handles from iga_atmo_load_rngdep) against the eigenray tables the
reference's own infraga-3d-rngdep / infraga-sph-rngdep binaries wrote
(tests/golden/cli/{3dr,sphr}_eig*, 8 significant digits, written by
tests/golden/make_cli_golden.py)."""
import os

import numpy as np
import pytest

import infraga_b200 as ig
from tests._cases import GOLDEN

pytestmark = pytest.mark.gpu

CLI = os.path.join(GOLDEN, "cli")
# stopping-rule bounds as for the stratified searches (tests/test_eig3d_gpu.py,
# tests/test_eigsph_gpu.py); 3D columns 3-4 in km, spherical in degrees
ATOL_3D = np.array([2e-3, 2e-3, 0, 0.1, 0.1, 0.5, 2e-4, 0.05, 2e-3, 2e-3, 0.5, 0.05])
ATOL_SPH = np.array([2e-3, 2e-3, 0, 1e-3, 1e-3, 0.5, 2e-4, 0.05, 2e-3, 2e-3, 0.5, 0.05])


def rows_of(path):
    rows = [[float(x) for x in ln.split("\t")] for ln in open(path) if ln.strip() and not ln.startswith("#")]
    return np.array(rows, dtype=np.float64).reshape(-1, 12)


@pytest.fixture(scope="module")
def dev():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU tests need a CUDA device")
    ig.lib()
    return torch


def load(kind):
    d = os.path.join(GOLDEN, "rngdep3d" if kind == "3dr" else "rngdep")
    ax = ("node_x.dat", "node_y.dat") if kind == "3dr" else ("node_lat.dat", "node_lon.dat")
    return ig.Atmosphere.load_rngdep(os.path.join(d, "node"), os.path.join(d, ax[0]), os.path.join(d, ax[1]),
                                     topo_file=os.path.join(d, "topo.dat"),
                                     geometry=ig.GEOM_3D if kind == "3dr" else ig.GEOM_SPH)


def centre(atmo):
    a0, a1, b0, b1 = atmo.region()
    return (a1 + a0) / 2.0, (b1 + b0) / 2.0


def check(got, ref, atol):
    assert got.shape == ref.shape, (got[:, :3], ref[:, :3])
    np.testing.assert_array_equal(got[:, 2], ref[:, 2])
    d = np.abs(got - ref)
    print("  max |diff| per column:", np.array2string(d.max(axis=0, initial=0.0), precision=3))
    bad = d > atol[None, :] + 1e-7 * np.abs(ref)
    assert not bad.any(), (np.argwhere(bad)[:5], got[bad], ref[bad])


def test_3dr_eigenrays_match_reference(dev):
    atmo = load("3dr")
    x, y = centre(atmo)
    p = ig.eig_params(atmo, incl_min=12.0, incl_max=24.0)
    got = ig.eig_run(atmo, p, [((x, y, 0.0), (210.0, 0.0))])["eigenrays"]
    ref = rows_of(os.path.join(CLI, "3dr_eig", "grid", "node.arrivals.dat"))
    print("3dr reference", ref.shape[0], "gpu", got.shape[0])
    check(got, ref, ATOL_3D)
    assert np.all(np.hypot(got[:, 3] - 210.0, got[:, 4]) < p.tolerance + 1e-6)


def test_sphr_eigenrays_match_reference(dev):
    atmo = load("sphr")
    lat, lon = centre(atmo)
    p = ig.eig_params(atmo, incl_min=10.0, incl_max=30.0)
    assert p.fan.geometry == ig.GEOM_SPH
    got = ig.eig_run(atmo, p, [((lat, lon, 3.0), (32.98, -104.6))])["eigenrays"]
    ref = rows_of(os.path.join(CLI, "sphr_eig", "grid", "node.arrivals.dat"))
    print("sphr reference", ref.shape[0], "gpu", got.shape[0])
    check(got, ref, ATOL_SPH)


def test_sphr_ground_source_over_terrain_finds_none(dev):
    """Over terrain the spherical search's ground launch limit is a degree
    value compared with radians (kept as the reference has it), so a source on
    sloping ground starts its sweep above the inclination range."""
    atmo = load("sphr")
    lat, lon = centre(atmo)
    p = ig.eig_params(atmo)
    got = ig.eig_run(atmo, p, [((lat, lon, 0.0), (32.98, -104.6))])
    assert got["eigenrays"].shape[0] == 0
    assert rows_of(os.path.join(CLI, "sphr_eig_ground", "ground.arrivals.dat")).shape[0] == 0


def test_rngdep_pairs_must_share_the_source(dev):
    atmo = load("3dr")
    p = ig.eig_params(atmo)
    with pytest.raises(ig.IgaError):
        ig.eig_run(atmo, p, [((0.0, 0.0, 2.0), (200.0, 0.0)), ((10.0, 0.0, 2.0), (200.0, 0.0))])

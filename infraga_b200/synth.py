"""Seeded synthetic atmospheres in the reference's ``.met`` formats.

The reference ships only example profiles (examples/ToyAtmo.met and the 4x4
``examples/profs`` grid); the benchmark workloads use generated profiles of
the same shape instead:

* 751 levels, z = 0..150 km every 0.2 km, column format ``zTuvdp``
  (the reference's default, parsed by atmo_io.3d.strat.cpp:85-93);
* T piecewise linear through (0, 288), (11, 217), (20, 217), (50, 270),
  (85, 190), (150, 1000) K;
* u = 30 exp(-(z-12)^2 / 18) + 60 exp(-(z-60)^2 / 200) m/s, v = 0, plus for u
  and v each a seeded sum of 20 sinusoids (vertical wavelength U[2, 20] km,
  phase U[0, 2 pi)) with equal amplitudes giving 5 m/s total rms;
* rho = 1.225e-3 exp(-z / 7) g/cm^3;
* p = rho R T (ideal gas, in mbar) so that the reference's sound-speed
  conversion c = sqrt(0.1 gamma p / rho) (atmo_io.3d.strat.cpp:114) gives
  c = sqrt(gamma R T).  A literally hydrostatic p with this rho would give a
  constant or unbounded c; the ideal-gas reading is the one used here.
"""
from __future__ import annotations

import os
from typing import Sequence

import numpy as np

R_AIR = 287.058      # atmo_state.3d.strat.cpp:26
T_KNOTS = ((0.0, 288.0), (11.0, 217.0), (20.0, 217.0), (50.0, 270.0), (85.0, 190.0), (150.0, 1000.0))


def profile_columns(seed: int, z_top: float = 150.0, dz: float = 0.2,
                    jet_scale: Sequence[float] = (1.0, 1.0), n_waves: int = 20,
                    wave_rms: float = 5.0, rng: np.random.Generator | None = None):
    """Return (z, T, u, v, rho, p) arrays for one seeded profile (units of the .met file)."""
    n = int(round(z_top / dz)) + 1
    z = np.round(np.arange(n) * dz, 10)
    tz, tv = zip(*T_KNOTS)
    T = np.interp(z, tz, tv)
    u = jet_scale[0] * 30.0 * np.exp(-(z - 12.0) ** 2 / (2 * 3.0 ** 2)) \
        + jet_scale[1] * 60.0 * np.exp(-(z - 60.0) ** 2 / (2 * 10.0 ** 2))
    v = np.zeros_like(z)
    g = rng if rng is not None else np.random.default_rng(seed)
    amp = wave_rms / np.sqrt(n_waves / 2.0)
    for comp in (u, v):
        lam = g.uniform(2.0, 20.0, n_waves)
        ph = g.uniform(0.0, 2 * np.pi, n_waves)
        comp += amp * np.sin(2 * np.pi * z[:, None] / lam[None, :] + ph[None, :]).sum(axis=1)
    rho = 1.225e-3 * np.exp(-z / 7.0)
    p = rho * 1.0e3 * R_AIR * T / 100.0
    return z, T, u, v, rho, p


def write_met(path: str, seed: int, **kw) -> str:
    """Write one seeded ``zTuvdp`` profile to ``path`` and return the path."""
    z, T, u, v, rho, p = profile_columns(seed, **kw)
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    with open(path, "w") as f:
        f.write(f"# synthetic infraga-b200 profile, seed {seed}\n")
        f.write("# z [km]\tT [K]\tu [m/s]\tv [m/s]\trho [g/cm^3]\tp [mbar]\n")
        for row in zip(z, T, u, v, rho, p):
            f.write("\t".join(f"{x:.10e}" for x in row) + "\n")
    return path


def fan_angles(incl_min: float, incl_max: float, incl_step: float,
               az_min: float, az_max: float, az_step: float,
               src_above_ground: bool = False):
    """Launch angles in the order the reference CLI traces them.

    Reproduces the FP64 accumulated loops of run_prop
    (main.infraga.3d.cpp:407-421): ``for (phi = min; phi <= max; phi += step)``
    outer, ``for (theta = max(min, th_grnd); theta <= max(max, th_grnd);
    theta += step)`` inner, with th_grnd = 0.1 deg for a ground source on flat
    ground and -89.9 deg for an elevated source.
    Returns (theta_deg, phi_deg) float64 arrays.
    """
    th_grnd = -89.9 if src_above_ground else 0.1
    th_out, ph_out = [], []
    phi = float(az_min)
    while phi <= az_max:
        th = max(float(incl_min), th_grnd)
        th_hi = max(float(incl_max), th_grnd)
        while th <= th_hi:
            th_out.append(th)
            ph_out.append(phi)
            th += incl_step
        phi += az_step
    return np.asarray(th_out, dtype=np.float64), np.asarray(ph_out, dtype=np.float64)


def write_rngdep_grid(out_dir: str, seed: int, n_lat: int = 21, n_lon: int = 21, lat0: float = 30.0,
                      lon0: float = -110.0, dlat: float = 1.0, dlon: float = 1.0, prefix: str = "node",
                      z_top: float = 150.0, dz: float = 0.2, node_rms: float = 1.0, axes=("lat", "lon")):
    """Range-dependent grid in the layout set_region reads for the range-
    dependent solvers (atmo_io.sph.rngdep.cpp:61-131): a latitude list, a
    longitude list (degrees, one per line) and one ``zTuvdp`` profile per node
    named ``{prefix}{n}.met`` with n = i_lat * n_lon + i_lon.  For the 3D
    Cartesian solver the same layout holds with x/y node lists in km
    (``axes=("x", "y")``, atmo_io.3d.rngdep.cpp:86-110).

    Each node is the single-profile generator above with jet amplitudes that
    vary smoothly across the grid (seeded phases, +-30 %), the same 20 gravity
    waves everywhere (so horizontal differences stay smooth) and a small
    node-specific perturbation (``node_rms`` m/s rms, 8 waves).
    Returns (prefix_path, lat_file, lon_file).
    """
    os.makedirs(out_dir, exist_ok=True)
    g = np.random.default_rng(seed)
    ph = g.uniform(0.0, 2 * np.pi, 4)
    lats = lat0 + dlat * np.arange(n_lat)
    lons = lon0 + dlon * np.arange(n_lon)
    lat_file = os.path.join(out_dir, f"{prefix}_{axes[0]}.dat")
    lon_file = os.path.join(out_dir, f"{prefix}_{axes[1]}.dat")
    with open(lat_file, "w") as f:
        f.write("".join(f"{x:.6f}\n" for x in lats))
    with open(lon_file, "w") as f:
        f.write("".join(f"{x:.6f}\n" for x in lons))
    for i in range(n_lat):
        for j in range(n_lon):
            a = i / max(n_lat - 1, 1)
            b = j / max(n_lon - 1, 1)
            js = (1.0 + 0.3 * np.sin(2 * np.pi * a + ph[0]) * np.cos(np.pi * b + ph[1]),
                  1.0 + 0.3 * np.cos(np.pi * a + ph[2]) * np.sin(2 * np.pi * b + ph[3]))
            z, T, u, v, rho, p = profile_columns(seed, z_top=z_top, dz=dz, jet_scale=js,
                                                 rng=np.random.default_rng(seed))
            if node_rms > 0.0:
                gn = np.random.default_rng([seed, i, j])
                amp = node_rms / np.sqrt(8 / 2.0)
                for comp in (u, v):
                    lam = gn.uniform(2.0, 20.0, 8)
                    phs = gn.uniform(0.0, 2 * np.pi, 8)
                    comp += amp * np.sin(2 * np.pi * z[:, None] / lam[None, :] + phs[None, :]).sum(axis=1)
            path = os.path.join(out_dir, f"{prefix}{i * n_lon + j}.met")
            with open(path, "w") as f:
                f.write(f"# synthetic infraga-b200 range-dependent node ({i}, {j}), seed {seed}\n")
                for row in zip(z, T, u, v, rho, p):
                    f.write("\t".join(f"{x:.10e}" for x in row) + "\n")
    return os.path.join(out_dir, prefix), lat_file, lon_file


def fractal_terrain(seed: int, n_lat: int, n_lon: int, z_max: float = 3.0, slope: float = -2.0):
    """Seeded fractal terrain: white noise shaped to a power spectrum
    proportional to k^slope, rescaled to [0, z_max] km."""
    g = np.random.default_rng(seed)
    w = g.standard_normal((n_lat, n_lon))
    ky = np.fft.fftfreq(n_lat)[:, None]
    kx = np.fft.fftfreq(n_lon)[None, :]
    k = np.sqrt(kx * kx + ky * ky)
    k[0, 0] = 1.0
    amp = k ** (slope / 2.0)
    amp[0, 0] = 0.0
    z = np.real(np.fft.ifft2(np.fft.fft2(w) * amp))
    z -= z.min()
    z *= z_max / max(z.max(), 1e-30)
    return z


def write_terrain(path: str, seed: int, lat0: float, lat1: float, lon0: float, lon1: float, step: float,
                  z_max: float = 3.0):
    """Terrain file for topo_file= (atmo_io.sph.rngdep.cpp:213-225): rows
    ``lat lon z`` [deg, deg, km], latitude-major, longitude increasing fastest
    (for the 3D solvers ``x y z`` in km, atmo_io.3d.rngdep.cpp:209-223)."""
    lats = np.round(np.arange(lat0, lat1 + step * 0.5, step), 8)
    lons = np.round(np.arange(lon0, lon1 + step * 0.5, step), 8)
    z = fractal_terrain(seed, lats.size, lons.size, z_max)
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    with open(path, "w") as f:
        for i, la in enumerate(lats):
            f.write("".join(f"{la:.8f}\t{lo:.8f}\t{z[i, j]:.8e}\n" for j, lo in enumerate(lons)))
    return path

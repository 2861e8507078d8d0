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

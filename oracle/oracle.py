"""ctypes binding of the CPU oracle (test infrastructure only).

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s cpu_baseline
leg import this module, and only as the checker / timed CPU baseline.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")
ARR_COLS = 12
_lib = None


class FanCfg(ctypes.Structure):
    _fields_ = [
        ("src", ctypes.c_double * 3),
        ("ds_min", ctypes.c_double), ("ds_max", ctypes.c_double), ("s_max", ctypes.c_double),
        ("alt_max", ctypes.c_double), ("rng_max", ctypes.c_double),
        ("x_min", ctypes.c_double), ("x_max", ctypes.c_double),
        ("y_min", ctypes.c_double), ("y_max", ctypes.c_double),
        ("z_grnd", ctypes.c_double), ("freq", ctypes.c_double),
        ("tweak_abs", ctypes.c_double), ("turn_ht_min", ctypes.c_double),
        ("bounces", ctypes.c_int), ("calc_amp", ctypes.c_int), ("write_rays", ctypes.c_int),
        ("reverse_winds", ctypes.c_int), ("n_threads", ctypes.c_int),
    ]


def build() -> None:
    """Compile the oracle restatement and, where the reference checkout is present
    (IGA_REFERENCE_DIR, default /root/reference), oracle/_ref from its sources."""
    subprocess.run(["make", "-s", "-C", HERE, "port"], check=True)
    ref = os.environ.get("IGA_REFERENCE_DIR", "/root/reference")
    if os.path.isdir(os.path.join(ref, "src")):
        subprocess.run(["make", "-s", "-C", HERE, "ref", f"REF={ref}"], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            subprocess.run(["make", "-s", "-C", HERE, "port"], check=True)
        _lib = ctypes.CDLL(LIB_PATH)
        _lib.orc_fan_3d.restype = ctypes.c_int
    return _lib


def default_cfg(**kw) -> FanCfg:
    """Fan configuration with the 3D CLI defaults for a flat-ground profile
    spanning 0..150 km (set_limits, atmo_io.3d.strat.cpp:24-37)."""
    c = FanCfg()
    vals = dict(src=(0.0, 0.0, 0.0), ds_min=0.001, ds_max=0.05, s_max=1000.0, alt_max=150.0,
                rng_max=2000.0, x_min=-2000.0, x_max=2000.0, y_min=-2000.0, y_max=2000.0,
                z_grnd=0.0, freq=0.1, tweak_abs=1.0, turn_ht_min=0.2, bounces=10, calc_amp=1,
                write_rays=0, reverse_winds=0, n_threads=1)
    vals.update(kw)
    for k, v in vals.items():
        if k == "src":
            c.src = (ctypes.c_double * 3)(*v)
        else:
            setattr(c, k, v)
    return c


AUX_COLS = 4


def fan_3d(met_path: str, theta_deg, phi_deg, fmt: str = "zTuvdp", with_aux: bool = False, **cfg_kw):
    """Run the oracle 3D stratified fan.  Returns (arrivals [n_rows, 12], steps
    per ray), plus the per-arrival diagnostics [n_rows, 4] when with_aux."""
    th = np.ascontiguousarray(theta_deg, dtype=np.float64)
    ph = np.ascontiguousarray(phi_deg, dtype=np.float64)
    cfg = default_cfg(**cfg_kw)
    n = th.size
    nb = cfg.bounces + 1
    arr = np.zeros((n * nb, ARR_COLS), dtype=np.float64)
    n_arr = np.zeros(n, dtype=np.int32)
    steps = np.zeros(n, dtype=np.int64)
    aux = np.zeros((n * nb, AUX_COLS), dtype=np.float64)
    P = ctypes.POINTER
    rc = lib().orc_fan_3d(met_path.encode(), fmt.encode(), ctypes.byref(cfg),
                          th.ctypes.data_as(P(ctypes.c_double)), ph.ctypes.data_as(P(ctypes.c_double)),
                          ctypes.c_int(n), arr.ctypes.data_as(P(ctypes.c_double)),
                          n_arr.ctypes.data_as(P(ctypes.c_int)), steps.ctypes.data_as(P(ctypes.c_longlong)),
                          aux.ctypes.data_as(P(ctypes.c_double)))
    if rc != 0:
        raise RuntimeError(f"oracle fan failed ({rc}) for {met_path}")
    sel = np.concatenate([np.arange(i * nb, i * nb + n_arr[i]) for i in range(n)]).astype(np.int64) if n else []
    rows = arr[sel]
    if with_aux:
        return rows, steps, aux[sel]
    return rows, steps


def parse_ref_output(text: str):
    """Parse the full-precision reference driver output (oracle/harness)."""
    rows, steps, meta = [], [], {}
    for line in text.splitlines():
        if not line.strip():
            continue
        if line.startswith("#"):
            parts = line[1:].split()
            for i in range(0, len(parts) - 1, 2):
                try:
                    meta[parts[i]] = float(parts[i + 1])
                except ValueError:
                    pass
            continue
        if line.startswith("R\t"):
            steps.append(int(line.split("\t")[3]))
            continue
        rows.append([float(x) for x in line.split("\t")])
    return np.array(rows, dtype=np.float64).reshape(-1, ARR_COLS), np.array(steps, dtype=np.int64), meta

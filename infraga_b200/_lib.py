"""ctypes binding of libinfraga_gpu.so (the C ABI in include/infraga_gpu.h).

There is no CPU fallback: if the shared library is missing or cannot be
loaded, every call raises ``NativeLibraryError``.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libinfraga_gpu.so")
ARRIVAL_COLS = 12
AUX_COLS = 4

IGA_OK, IGA_E_INVALID, IGA_E_IO, IGA_E_NOMEM, IGA_E_CUDA, IGA_E_NODEVICE, IGA_E_TRUNCATED, IGA_E_UNSUPPORTED = \
    0, -1, -2, -3, -4, -5, -6, -7
GEOM_3D, GEOM_SPH = 0, 1
FP64, FP32C, FP32C_FLAGGED = 0, 1, 2
RAY_STATUS = {0: "bounces", 1: "escaped", 2: "low_turn", 3: "short", 4: "nonfinite", 5: "stepcap", 6: "time_max"}
# flag OR'ed into an FP32C ray's status: traced again with FP64 auxiliaries
# after a focusing arrival (IGA_RAY_AUX_FP64); status & 0xff is the reason
RAY_AUX_FP64 = 0x100
# flag OR'ed into an FP32C_FLAGGED ray's status: met a focusing arrival and kept
# its FP32 auxiliaries (IGA_RAY_FOCUS)
RAY_FOCUS = 0x200


class NativeLibraryError(RuntimeError):
    pass


class IgaError(RuntimeError):
    def __init__(self, code: int, what: str):
        self.code = code
        super().__init__(f"{what}: {strerror(code)} ({code}) {last_cuda_error()}".rstrip())


class FanParams(ctypes.Structure):
    """Mirror of iga_fan_params."""
    _fields_ = [
        ("geometry", ctypes.c_int), ("precision", ctypes.c_int), ("bounces", ctypes.c_int),
        ("calc_amp", ctypes.c_int), ("write_rays", ctypes.c_int), ("block", ctypes.c_int),
        ("src", ctypes.c_double * 3),
        ("ds_min", ctypes.c_double), ("ds_max", ctypes.c_double), ("s_max", ctypes.c_double),
        ("alt_max", ctypes.c_double), ("rng_max", ctypes.c_double),
        ("x_min", ctypes.c_double), ("x_max", ctypes.c_double),
        ("y_min", ctypes.c_double), ("y_max", ctypes.c_double),
        ("z_grnd", ctypes.c_double), ("freq", ctypes.c_double), ("tweak_abs", ctypes.c_double),
        ("turn_ht_min", ctypes.c_double),
        ("lat_min", ctypes.c_double), ("lat_max", ctypes.c_double),
        ("lon_min", ctypes.c_double), ("lon_max", ctypes.c_double),
        ("time_max", ctypes.c_double),
    ]


class EigParams(ctypes.Structure):
    """Mirror of iga_eig_params."""
    _fields_ = [("fan", FanParams), ("incl_min", ctypes.c_double), ("incl_max", ctypes.c_double),
                ("incl_step_min", ctypes.c_double), ("incl_step_max", ctypes.c_double),
                ("damping", ctypes.c_double), ("tolerance", ctypes.c_double), ("az_err_lim", ctypes.c_double),
                ("bnc_min", ctypes.c_int), ("bnc_max", ctypes.c_int), ("iterations", ctypes.c_int),
                ("chunk", ctypes.c_int), ("streams", ctypes.c_int)]


class WnlParams(ctypes.Structure):
    """Mirror of iga_wnl_params."""
    _fields_ = [("fan", FanParams), ("ds_wvfrm", ctypes.c_double), ("wvfrm_ref", ctypes.c_double),
                ("out_step", ctypes.c_double),
                ("filt1_g", ctypes.c_double), ("filt1_n1", ctypes.c_double), ("filt1_n2", ctypes.c_double),
                ("filt2_g", ctypes.c_double), ("filt2_n1", ctypes.c_double), ("filt2_n2", ctypes.c_double),
                ("max_steps", ctypes.c_longlong)]


WNL_INFO = 17
WNL_INFO_NAMES = ("status", "steps", "shifts", "events", "snaps", "t_ref", "p0", "scale", "length", "c0", "rho0",
                  "nu0", "cg0", "D0", "oob", "beta0", "time")
WNL_EVENT_COLS = 4


class EigPair(ctypes.Structure):
    _fields_ = [("src", ctypes.c_double * 3), ("rcvr", ctypes.c_double * 2)]


class ServerConfig(ctypes.Structure):
    """Mirror of iga_server_config."""
    _fields_ = [("device", ctypes.c_int), ("max_inflight", ctypes.c_int), ("eig_workers", ctypes.c_int),
                ("small_rays", ctypes.c_int), ("big_fan_sm_frac", ctypes.c_double), ("hbm_budget", ctypes.c_size_t)]


class ServerStats(ctypes.Structure):
    """Mirror of iga_server_stats."""
    _fields_ = [("completed", ctypes.c_longlong), ("pending", ctypes.c_longlong),
                ("p50_s", ctypes.c_double), ("p99_s", ctypes.c_double),
                ("fan_p50_s", ctypes.c_double), ("fan_p99_s", ctypes.c_double),
                ("eig_p50_s", ctypes.c_double), ("eig_p99_s", ctypes.c_double),
                ("ray_steps", ctypes.c_longlong), ("rays", ctypes.c_longlong), ("eigenrays", ctypes.c_longlong),
                ("wall_s", ctypes.c_double), ("bytes_in_use", ctypes.c_size_t)]


class Profile(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int), ("z", ctypes.POINTER(ctypes.c_double)), ("c", ctypes.POINTER(ctypes.c_double)),
                ("u", ctypes.POINTER(ctypes.c_double)), ("v", ctypes.POINTER(ctypes.c_double)),
                ("rho", ctypes.POINTER(ctypes.c_double))]


_lib = None
_P = ctypes.POINTER
_D = ctypes.c_double
_I = ctypes.c_int
_LL = ctypes.c_longlong
_VP = ctypes.c_void_p

# name -> (restype, argtypes)
_SIGS = {
    "iga_strerror": (ctypes.c_char_p, [_I]),
    "iga_last_cuda_error": (ctypes.c_char_p, []),
    "iga_version": (_I, []),
    "iga_device_count": (_I, [_P(_I)]),
    "iga_atmo_load": (_I, [ctypes.c_char_p, ctypes.c_char_p, _I, _P(_VP)]),
    "iga_atmo_create": (_I, [_P(Profile), _P(_VP)]),
    "iga_atmo_limits": (_I, [_VP, _P(_D), _P(_D)]),
    "iga_atmo_destroy": (_I, [_VP]),
    "iga_atmo_load_rngdep": (_I, [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p,
                                  _I, _I, _P(_VP)]),
    "iga_atmo_region": (_I, [_VP, _P(_D), _P(_D), _P(_D), _P(_D)]),
    "iga_atmo_load_topo": (_I, [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p, _I, _I, _P(_VP)]),
    "iga_atmo_sample": (_I, [_VP, _P(FanParams), _D, _D, _P(_D), _I, _P(_D)]),
    "iga_server_config_default": (_I, [_P(ServerConfig)]),
    "iga_server_create": (_I, [_P(ServerConfig), _P(_VP)]),
    "iga_server_submit_fan": (_I, [_VP, _VP, _P(FanParams), _P(_D), _P(_D), _I, _P(_LL)]),
    "iga_server_submit_eig": (_I, [_VP, _VP, _P(EigParams), _P(EigPair), _I, _P(_LL)]),
    "iga_server_wait": (_I, [_VP, _LL, _D, _P(_I)]),
    "iga_server_fetch": (_I, [_VP, _LL, _P(_D), _I, _P(_I), _P(_I), _P(_LL), _P(_D)]),
    "iga_server_get_stats": (_I, [_VP, _P(ServerStats)]),
    "iga_server_destroy": (_I, [_VP]),
    "iga_fan_params_default": (_I, [_VP, _P(FanParams)]),
    "iga_fan_params_init": (_I, [_VP, _I, _P(FanParams)]),
    "iga_fan_run": (_I, [_VP, _P(FanParams), _P(_D), _P(_D), _I, _P(_D), _I, _P(_I), _P(_I), _P(_LL), _P(_I), _P(_LL),
                         _P(_D)]),
    "iga_fan_workspace_bytes": (ctypes.c_size_t, []),
    "iga_fan_run_device": (_I, [_VP, _P(FanParams), _VP, _VP, _I, _VP, _VP, _VP, _VP, _VP, _VP, _VP]),
    "iga_fan_run_device_noalloc": (_I, [_VP, _P(FanParams), _VP, _VP, _I, _VP, _VP, _VP, _VP, _VP, _VP]),
    "iga_eig_params_default": (_I, [_VP, _P(EigParams)]),
    "iga_eig_run": (_I, [_VP, _P(EigParams), _P(EigPair), _I, _P(_D), _I, _P(_I), _P(_I), _P(_LL)]),
    "iga_eig_direct": (_I, [_VP, _P(EigParams), _P(EigPair), _D, _D, _I, _P(_D), _P(_I), _P(_LL)]),
    "iga_fan_paths": (_I, [_VP, _P(FanParams), _P(_D), _P(_D), _I, _I, _P(_LL), _P(_D), _LL, _P(_LL), _P(_LL),
                           _P(_D), _LL, _P(_LL), _P(_I)]),
    "iga_atmo_terrain": (_I, [_VP, _D, _D, _P(_D), _P(_D), _P(_D)]),
    "iga_fan_tune": (_I, [_VP, _P(FanParams), _P(_D), _P(_D), _I, _P(_I), _P(_D)]),
    "iga_wnl_params_default": (_I, [_VP, _P(WnlParams)]),
    "iga_wnl_run": (_I, [_VP, _P(WnlParams), _P(_D), _P(_D), _I, _P(_D), _P(_D), _I, _P(_D), _P(_D), _P(_D), _P(_I),
                         _P(_I), _P(_D), _I, _P(_D), _I]),
}


def exported_symbols() -> list[str]:
    return list(_SIGS)


def lib():
    """Load libinfraga_gpu.so (building it first only if the sources are present and it is absent)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        try:
            from . import build as _build
            _build.build_lib()
        except Exception as e:  # pragma: no cover - depends on toolchain
            raise NativeLibraryError(f"libinfraga_gpu.so is missing and could not be built: {e}") from e
    try:
        L = ctypes.CDLL(LIB_PATH)
    except OSError as e:
        raise NativeLibraryError(f"cannot load {LIB_PATH}: {e}") from e
    for name, (res, args) in _SIGS.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def strerror(code: int) -> str:
    return lib().iga_strerror(code).decode()


def last_cuda_error() -> str:
    return lib().iga_last_cuda_error().decode()


def _check(rc: int, what: str):
    if rc != IGA_OK:
        raise IgaError(rc, what)


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(_P(_D))


class Atmosphere:
    """A stratified atmosphere resident on the current CUDA device
    (the reference's set_region, atmo_io.3d.strat.cpp:55-143)."""

    def __init__(self, handle):
        self._h = handle

    @classmethod
    def load(cls, met_path: str, fmt: str = "zTuvdp", reverse_winds: bool = False) -> "Atmosphere":
        h = _VP()
        _check(lib().iga_atmo_load(str(met_path).encode(), fmt.encode(), int(reverse_winds), ctypes.byref(h)),
               f"iga_atmo_load({met_path})")
        return cls(h)

    @classmethod
    def load_rngdep(cls, prefix: str, x_file: str, y_file: str, topo_file: str | None = None,
                    fmt: str = "zTuvdp", reverse_winds: bool = False, geometry: int = GEOM_SPH) -> "Atmosphere":
        """Range-dependent grid ({prefix}{n}.met node profiles on the node
        lists: lat/lon in degrees for GEOM_SPH, x/y in km for GEOM_3D) with
        optional terrain (the range-dependent set_region,
        atmo_io.sph.rngdep.cpp:61-311 and atmo_io.3d.rngdep.cpp:58-330)."""
        h = _VP()
        _check(lib().iga_atmo_load_rngdep(str(prefix).encode(), str(x_file).encode(), str(y_file).encode(),
                                          str(topo_file).encode() if topo_file else None, fmt.encode(),
                                          int(reverse_winds), int(geometry), ctypes.byref(h)),
               f"iga_atmo_load_rngdep({prefix})")
        return cls(h)

    @classmethod
    def load_topo(cls, met_path: str, topo_file: str, fmt: str = "zTuvdp", reverse_winds: bool = False,
                  geometry: int = GEOM_3D) -> "Atmosphere":
        """A .met profile over a terrain file: infraga-3d's set_region with
        topo_file (atmo_io.3d.strat.cpp:146-258; rows "x y z" in km) or, with
        geometry=GEOM_SPH, infraga-sph's (rows "lat lon z" in deg, deg, km).
        The handle runs FP64 fans and eigenray searches of that geometry like a
        range-dependent one."""
        h = _VP()
        _check(lib().iga_atmo_load_topo(str(met_path).encode(), str(topo_file).encode(), fmt.encode(),
                                        int(reverse_winds), int(geometry), ctypes.byref(h)),
               f"iga_atmo_load_topo({met_path}, {topo_file})")
        return cls(h)

    def sample(self, params: FanParams, x: float, y: float, z) -> np.ndarray:
        """atmo::c, u, v, rho at (x, y) [km; lat, lon in deg for GEOM_SPH params]
        and altitudes z [km], as the reference's point functions return them
        (host FP64; the write_atmo profile).  Returns [n, 4]."""
        zz = np.ascontiguousarray(z, dtype=np.float64)
        out = np.zeros((max(zz.size, 1), 4), dtype=np.float64)
        _check(lib().iga_atmo_sample(self._h, ctypes.byref(params), float(x), float(y), _dptr(zz), zz.size, _dptr(out)),
               "iga_atmo_sample")
        return out[:zz.size]

    def region(self):
        """(lat_min, lat_max, lon_min, lon_max) [deg] of geoac::set_limits."""
        v = [_D() for _ in range(4)]
        _check(lib().iga_atmo_region(self._h, *[ctypes.byref(x) for x in v]), "iga_atmo_region")
        return tuple(x.value for x in v)

    @classmethod
    def from_arrays(cls, z, c, u, v, rho) -> "Atmosphere":
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (z, c, u, v, rho)]
        pr = Profile(len(arrs[0]), *[_dptr(a) for a in arrs])
        h = _VP()
        _check(lib().iga_atmo_create(ctypes.byref(pr), ctypes.byref(h)), "iga_atmo_create")
        return cls(h)

    @property
    def handle(self):
        return self._h

    def limits(self):
        lo, hi = _D(), _D()
        _check(lib().iga_atmo_limits(self._h, ctypes.byref(lo), ctypes.byref(hi)), "iga_atmo_limits")
        return lo.value, hi.value

    def default_params(self, geometry: int = GEOM_3D, **overrides) -> FanParams:
        """run_prop defaults for ``geometry`` (GEOM_3D or GEOM_SPH) with
        keyword overrides of any iga_fan_params field."""
        p = FanParams()
        _check(lib().iga_fan_params_init(self._h, int(geometry), ctypes.byref(p)), "iga_fan_params_init")
        for k, v in overrides.items():
            if k == "src":
                p.src = (_D * 3)(*v)
            else:
                setattr(p, k, v)
        return p

    def close(self):
        if self._h:
            lib().iga_atmo_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def fan_run(atmo: Atmosphere, params: FanParams, theta_deg, phi_deg, with_aux: bool = False):
    """Trace a ray fan (host buffers).  Returns a dict with ``arrivals``
    [n_rows, 12] in the reference's .arrivals.dat column order, ``ray_index``,
    ``ray_steps``, ``ray_status``, ``total_steps`` and, with ``with_aux``,
    ``aux`` [n_rows, 4]: |d(x,y)/d incl|, |d(x,y)/d az| [km/rad], the Jacobian
    D and the caustic count of each arrival."""
    th = np.ascontiguousarray(theta_deg, dtype=np.float64)
    ph = np.ascontiguousarray(phi_deg, dtype=np.float64)
    n = int(th.size)
    cap = n * (params.bounces + 1)
    arr = np.zeros((max(cap, 1), ARRIVAL_COLS), dtype=np.float64)
    ray_index = np.zeros(max(cap, 1), dtype=np.int32)
    steps = np.zeros(max(n, 1), dtype=np.int64)
    status = np.zeros(max(n, 1), dtype=np.int32)
    aux = np.zeros((max(cap, 1), AUX_COLS), dtype=np.float64) if with_aux else None
    n_out = _I()
    tot = _LL()
    rc = lib().iga_fan_run(atmo.handle, ctypes.byref(params), _dptr(th), _dptr(ph), n, _dptr(arr), cap,
                           ctypes.byref(n_out), ray_index.ctypes.data_as(_P(_I)), steps.ctypes.data_as(_P(_LL)),
                           status.ctypes.data_as(_P(_I)), ctypes.byref(tot),
                           _dptr(aux) if with_aux else None)
    _check(rc, "iga_fan_run")
    m = n_out.value
    out = {"arrivals": arr[:m], "ray_index": ray_index[:m], "ray_steps": steps[:n], "ray_status": status[:n],
           "total_steps": int(tot.value)}
    if with_aux:
        out["aux"] = aux[:m]
    return out


def eig_params(atmo: Atmosphere, geometry: int = GEOM_3D, **overrides) -> EigParams:
    """iga_eig_params with the run_eig_search defaults; keyword overrides go to
    the eigen fields or, for propagation settings, to params.fan.  For a
    spherical search (geometry=GEOM_SPH) params.fan takes infraga-sph's
    propagation defaults and pairs are given in degrees."""
    p = EigParams()
    _check(lib().iga_eig_params_default(atmo.handle, ctypes.byref(p)), "iga_eig_params_default")
    if geometry != GEOM_3D:
        _check(lib().iga_fan_params_init(atmo.handle, int(geometry), ctypes.byref(p.fan)), "iga_fan_params_init")
    eig_fields = {f for f, _ in EigParams._fields_}
    for k, v in overrides.items():
        if k in eig_fields:
            setattr(p, k, v)
        else:
            setattr(p.fan, k, v)
    return p


def eig_run(atmo: Atmosphere, params: EigParams, pairs):
    """Eigenray search for a list of ((sx, sy, sz), (rx, ry)) pairs.  Returns
    a dict with ``eigenrays`` [n, 12] (the reference's eigenray arrival rows),
    ``pair_index`` and ``total_steps``."""
    arr = (EigPair * max(1, len(pairs)))()
    for i, (src, rcv) in enumerate(pairs):
        arr[i].src = (_D * 3)(*src)
        arr[i].rcvr = (_D * 2)(*rcv)
    cap = max(16, 64 * len(pairs) * (params.bnc_max - params.bnc_min + 1))
    while True:
        out = np.zeros((cap, ARRIVAL_COLS), dtype=np.float64)
        idx = np.zeros(cap, dtype=np.int32)
        n_out = _I()
        tot = _LL()
        rc = lib().iga_eig_run(atmo.handle, ctypes.byref(params), arr, len(pairs), _dptr(out), cap,
                               ctypes.byref(n_out), idx.ctypes.data_as(_P(_I)), ctypes.byref(tot))
        if rc == IGA_E_TRUNCATED:
            cap = n_out.value
            continue
        _check(rc, "iga_eig_run")
        m = n_out.value
        return {"eigenrays": out[:m], "pair_index": idx[:m], "total_steps": int(tot.value)}


def eig_direct(atmo: Atmosphere, params: EigParams, src, rcvr, incl_est: float, az_est: float, bounces: int):
    """find_eigenray alone from a launch estimate (degrees).  Returns the
    eigenray row [12] or None when the refinement did not converge."""
    pair = EigPair()
    pair.src = (_D * 3)(*src)
    pair.rcvr = (_D * 2)(*rcvr)
    row = np.zeros(ARRIVAL_COLS, dtype=np.float64)
    found = _I()
    tot = _LL()
    _check(lib().iga_eig_direct(atmo.handle, ctypes.byref(params), ctypes.byref(pair), float(incl_est), float(az_est),
                                int(bounces), _dptr(row), ctypes.byref(found), ctypes.byref(tot)), "iga_eig_direct")
    return row if found.value else None


PATH_RAYS, PATH_TERRAIN, PATH_PROJ, PATH_RESID = 0, 1, 2, 3
PATH_COLS, CAUSTIC_COLS, PROJ_COLS = 7, 5, 15


def fan_paths(atmo: Atmosphere, params: FanParams, theta_deg, phi_deg, mode: int = PATH_RAYS,
              caustics: bool = False, ray_steps=None):
    """Sampled ray-path rows (run_prop's write_rays / write_topo rows, or
    run_back_proj's projection rows with mode=PATH_PROJ, or print_resid's
    per-segment residual rows with mode=PATH_RESID) and, with
    ``caustics``, caustic points of a fan.  Returns a dict with ``paths``
    [n, 7] ([n, 15] for PATH_PROJ), ``path_start`` [n_rays + 1] and, with
    caustics, ``caustics`` [m, 5] and ``caustic_ray`` [m]."""
    th = np.ascontiguousarray(theta_deg, dtype=np.float64)
    ph = np.ascontiguousarray(phi_deg, dtype=np.float64)
    n = th.size
    if ray_steps is None:
        ray_steps = fan_run(atmo, params, th, ph)["ray_steps"]
    steps = np.ascontiguousarray(ray_steps, dtype=np.int64)
    if mode == PATH_RESID:
        cap = int(n * (params.bounces + 1))
    else:
        div = {PATH_RAYS: 15, PATH_TERRAIN: 10, PATH_PROJ: 5}[mode]
        cap = int(np.sum(params.bounces + 1 + steps // div + 1))
    rows = np.zeros((max(cap, 1), PROJ_COLS if mode == PATH_PROJ else PATH_COLS), dtype=np.float64)
    start = np.zeros(n + 1, dtype=np.int64)
    n_path = _LL()
    ccap = 4096 if caustics else 0
    while True:
        crow = np.zeros((max(ccap, 1), CAUSTIC_COLS), dtype=np.float64)
        cray = np.zeros(max(ccap, 1), dtype=np.int32)
        n_caus = _LL()
        rc = lib().iga_fan_paths(atmo.handle, ctypes.byref(params), _dptr(th), _dptr(ph), n, int(mode),
                                 steps.ctypes.data_as(_P(_LL)), _dptr(rows), cap, ctypes.byref(n_path),
                                 start.ctypes.data_as(_P(_LL)), _dptr(crow) if caustics else None, ccap,
                                 ctypes.byref(n_caus) if caustics else None,
                                 cray.ctypes.data_as(_P(_I)) if caustics else None)
        if rc == IGA_E_TRUNCATED and caustics and n_caus.value > ccap:
            ccap = n_caus.value
            continue
        _check(rc, "iga_fan_paths")
        out = {"paths": rows[:n_path.value], "path_start": start}
        if caustics:
            out["caustics"] = crow[:n_caus.value]
            out["caustic_ray"] = cray[:n_caus.value]
        return out


def fan_tune(atmo: Atmosphere, params: FanParams, theta_deg, phi_deg):
    """Times the fan at each candidate CTA size; returns (best block, {block: seconds})."""
    th = np.ascontiguousarray(theta_deg, dtype=np.float64)
    ph = np.ascontiguousarray(phi_deg, dtype=np.float64)
    best = _I()
    secs = np.zeros(4, dtype=np.float64)
    _check(lib().iga_fan_tune(atmo.handle, ctypes.byref(params), _dptr(th), _dptr(ph), th.size, ctypes.byref(best),
                              _dptr(secs)), "iga_fan_tune")
    return int(best.value), dict(zip((32, 64, 96, 128), secs.tolist()))


def fan_workspace_bytes() -> int:
    return int(lib().iga_fan_workspace_bytes())


def fan_run_device(atmo: Atmosphere, params: FanParams, d_theta: int, d_phi: int, n_rays: int, d_arrivals: int,
                   d_n_arr: int, d_steps: int, d_status: int, d_workspace: int, stream: int = 0,
                   d_aux: int = 0) -> None:
    """Device-pointer form (pointers as integers, e.g. ``tensor.data_ptr()``)."""
    rc = lib().iga_fan_run_device(atmo.handle, ctypes.byref(params), _VP(d_theta), _VP(d_phi), int(n_rays),
                                  _VP(d_arrivals), _VP(d_n_arr), _VP(d_steps), _VP(d_status) if d_status else None,
                                  _VP(d_aux) if d_aux else None, _VP(d_workspace), _VP(stream) if stream else None)
    _check(rc, "iga_fan_run_device")


class Server:
    """Continuous-batching request server (iga_server_*): submit fan and
    eigenray requests from any thread, wait for and fetch their results."""

    def __init__(self, **config):
        cfg = ServerConfig()
        _check(lib().iga_server_config_default(ctypes.byref(cfg)), "iga_server_config_default")
        for k, v in config.items():
            setattr(cfg, k, v)
        self._h = _VP()
        _check(lib().iga_server_create(ctypes.byref(cfg), ctypes.byref(self._h)), "iga_server_create")
        self._kind = {}

    def submit_fan(self, atmo: Atmosphere, params: FanParams, theta_deg, phi_deg) -> int:
        th = np.ascontiguousarray(theta_deg, dtype=np.float64)
        ph = np.ascontiguousarray(phi_deg, dtype=np.float64)
        rid = _LL()
        _check(lib().iga_server_submit_fan(self._h, atmo.handle, ctypes.byref(params), _dptr(th), _dptr(ph),
                                           int(th.size), ctypes.byref(rid)), "iga_server_submit_fan")
        self._kind[rid.value] = ("fan", int(th.size) * (params.bounces + 1))
        return rid.value

    def submit_eig(self, atmo: Atmosphere, params: EigParams, pairs) -> int:
        arr = (EigPair * max(len(pairs), 1))()
        for i, (src, rcvr) in enumerate(pairs):
            arr[i].src = (_D * 3)(*src)
            arr[i].rcvr = (_D * 2)(*rcvr)
        rid = _LL()
        _check(lib().iga_server_submit_eig(self._h, atmo.handle, ctypes.byref(params), arr, len(pairs),
                                           ctypes.byref(rid)), "iga_server_submit_eig")
        self._kind[rid.value] = ("eig", 0)
        return rid.value

    def wait(self, rid: int, timeout_s: float = -1.0) -> bool:
        done = _I()
        _check(lib().iga_server_wait(self._h, rid, float(timeout_s), ctypes.byref(done)), "iga_server_wait")
        return bool(done.value)

    def fetch(self, rid: int):
        """Results of a finished request: dict with rows [n, 12], index,
        total_steps and latency_s (submit -> results on the host)."""
        cap = max(self._kind.get(rid, ("", 0))[1], 64)
        while True:
            rows = np.zeros((cap, ARRIVAL_COLS), dtype=np.float64)
            idx = np.zeros(cap, dtype=np.int32)
            n, steps, lat = _I(), _LL(), _D()
            rc = lib().iga_server_fetch(self._h, rid, _dptr(rows), cap, ctypes.byref(n), idx.ctypes.data_as(_P(_I)),
                                        ctypes.byref(steps), ctypes.byref(lat))
            if rc == -6:   # IGA_E_TRUNCATED: request kept, retry with the count it reported
                cap = n.value
                continue
            _check(rc, "iga_server_fetch")
            self._kind.pop(rid, None)
            m = n.value
            return {"rows": rows[:m], "index": idx[:m], "total_steps": int(steps.value), "latency_s": lat.value}

    def stats(self) -> dict:
        st = ServerStats()
        _check(lib().iga_server_get_stats(self._h, ctypes.byref(st)), "iga_server_get_stats")
        return {name: getattr(st, name) for name, _ in ServerStats._fields_}

    def close(self):
        if self._h:
            lib().iga_server_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def wnl_params(atmo: "Atmosphere", geometry: int = GEOM_3D, **overrides) -> WnlParams:
    """iga_wnl_params_default (fan from iga_fan_params_init for GEOM_SPH), then
    fields by name (fan fields too: bounces=, src=, freq= ...)."""
    p = WnlParams()
    _check(lib().iga_wnl_params_default(atmo.handle, ctypes.byref(p)), "iga_wnl_params_default")
    if geometry != GEOM_3D:
        _check(lib().iga_fan_params_init(atmo.handle, int(geometry), ctypes.byref(p.fan)), "iga_fan_params_init")
    for k, v in overrides.items():
        if hasattr(p, k) and k != "fan":
            setattr(p, k, v)
        elif k == "src":
            for i in range(3):
                p.fan.src[i] = float(v[i])
        else:
            setattr(p.fan, k, v)
    return p


def wnl_run(atmo: "Atmosphere", params: WnlParams, theta_deg, phi_deg, wv_t, wv_p, event_cap: int = 0,
            snap_cap: int = 0):
    """Weakly non-linear waveforms along rays (iga_wnl_run).  Returns a dict:
    ``u`` [n, len] (p = u * p0 * scale), ``info`` [n, WNL_INFO] (also by name),
    ``arrivals`` [n, bounces + 1, 12], ``n_arr``, ``ray_status`` and, with
    caps, ``events`` / ``snaps``."""
    th = np.ascontiguousarray(np.atleast_1d(theta_deg), dtype=np.float64)
    ph = np.ascontiguousarray(np.atleast_1d(phi_deg), dtype=np.float64)
    t = np.ascontiguousarray(wv_t, dtype=np.float64)
    pw = np.ascontiguousarray(wv_p, dtype=np.float64)
    n, N = th.size, t.size
    nb = params.fan.bounces + 1
    u = np.zeros((n, N))
    info = np.zeros((n, WNL_INFO))
    arr = np.zeros((n, nb, ARRIVAL_COLS))
    n_arr = np.zeros(n, dtype=np.int32)
    status = np.zeros(n, dtype=np.int32)
    ev = np.zeros((n, max(event_cap, 1), WNL_EVENT_COLS))
    snap_w = 1 + N + 2 * (N // 2 + 1)
    sn = np.zeros((n, max(snap_cap, 1), snap_w))
    rc = lib().iga_wnl_run(atmo.handle, ctypes.byref(params), _dptr(th), _dptr(ph), n, _dptr(t), _dptr(pw), N,
                           _dptr(u), _dptr(info), _dptr(arr), n_arr.ctypes.data_as(_P(_I)),
                           status.ctypes.data_as(_P(_I)), _dptr(ev) if event_cap else None, int(event_cap),
                           _dptr(sn) if snap_cap else None, int(snap_cap))
    _check(rc, "iga_wnl_run")
    out = {"u": u, "info": info, "arrivals": arr, "n_arr": n_arr, "ray_status": status}
    for i, name in enumerate(WNL_INFO_NAMES):
        out[name] = info[:, i]
    if event_cap:
        out["events"] = ev
    if snap_cap:
        out["snaps"] = sn
    return out

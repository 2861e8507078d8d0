/*
 * infraga_gpu.h — C ABI of the B200 ray-fan / eigenray library
 * (libinfraga_gpu.so).
 *
 * The reference has no library boundary: its CLI mains call the geoac/atmo
 * C++ namespace functions directly, one ray at a time, on global state.
 * Each entry point below replaces a group of those calls for a whole batch
 * of rays; the comment on each names the reference interface it replaces
 * (paths relative to the reference project).
 *
 * Conventions: plain C types only; the caller owns every input and output
 * array; the library owns device copies of atmospheres (handle lifetime =
 * create .. destroy).  Every function returns IGA_OK (0) or a negative
 * iga_status; no exceptions cross the ABI.  Handles are immutable after
 * creation and may be shared between threads.
 */
#ifndef INFRAGA_GPU_H_
#define INFRAGA_GPU_H_

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define IGA_ABI_VERSION 3

/* ---- status codes ---- */
enum iga_status {
    IGA_OK = 0,
    IGA_E_INVALID = -1,      /* bad argument or parameter */
    IGA_E_IO = -2,           /* profile / terrain file missing or malformed */
    IGA_E_NOMEM = -3,        /* host or device allocation failed */
    IGA_E_CUDA = -4,         /* CUDA runtime error (see iga_last_cuda_error) */
    IGA_E_NODEVICE = -5,     /* no CUDA device / extension not usable */
    IGA_E_TRUNCATED = -6,    /* output capacity too small; n_out holds the needed count */
    IGA_E_UNSUPPORTED = -7   /* combination not implemented (e.g. terrain on this geometry) */
};

/* ---- per-ray termination status (why a ray stopped) ---- */
enum iga_ray_status {
    IGA_RAY_BOUNCES = 0,     /* all requested bounces traced */
    IGA_RAY_ESCAPED = 1,     /* left the region: range, x/y, altitude or s_max (break_check) */
    IGA_RAY_LOW_TURN = 2,    /* turning height below turn_ht_min (main.infraga.3d.cpp:503) */
    IGA_RAY_SHORT = 3,       /* ground reached in < 2 steps (main.infraga.3d.cpp:507) */
    IGA_RAY_NONFINITE = 4,   /* state became NaN/Inf */
    IGA_RAY_STEPCAP = 5,     /* s_max/ds_min steps without a stop (prop_rk4 array bound) */
    IGA_RAY_TIME = 6,        /* travel time above time_max (spherical run_prop,
                                main.infraga.sph.cpp:515) */
    /* Flag OR'ed into the reason above (status & 0xff) for IGA_FP32C rays
     * with amplitudes that were traced again, from launch, with FP64
     * auxiliaries: a ray whose tube Jacobian at an arrival falls below 0.2 of
     * the largest |D| along its path before its first caustic.  Near such a
     * focus the amplitude is ill-conditioned and FP32 auxiliaries would miss
     * it by tenths of a dB. */
    IGA_RAY_AUX_FP64 = 0x100,
    /* Flag OR'ed into the reason for IGA_FP32C_FLAGGED rays that met such a
     * focusing arrival and were not traced again. */
    IGA_RAY_FOCUS = 0x200
};

/* geometry / precision selectors */
enum iga_geometry { IGA_GEOM_3D = 0, IGA_GEOM_SPH = 1 };
/* IGA_FP32C: FP32-compensated form (FP64 ray equations, FP32 Jacobian
 * auxiliaries summed with compensation); rays that reach a focusing arrival
 * before their first caustic are traced again with FP64 auxiliaries
 * (IGA_RAY_AUX_FP64).  IGA_FP32C_FLAGGED: the same without that second pass:
 * such rays keep their FP32 auxiliaries and carry IGA_RAY_FOCUS instead (their
 * amplitudes from the focusing arrival on are ill-conditioned, off by up to a
 * few tenths of a dB); the other arrivals are the same as with IGA_FP32C. */
enum iga_precision { IGA_FP64 = 0, IGA_FP32C = 1, IGA_FP32C_FLAGGED = 2 };

/* Columns of an arrival row, in the reference's .arrivals.dat order
 * (main.infraga.3d.cpp:362-374): incl, az, n_b, x_0, y_0, time, cel,
 * turning ht, arrival incl, back az, trans. coeff. [dB], absorption [dB].
 * For IGA_GEOM_SPH columns 3 and 4 are lat_0, lon_0 [deg] and the celerity
 * uses the great-circle range (main.infraga.sph.cpp:379-391, 526-539). */
#define IGA_ARRIVAL_COLS 12

/* Optional per-arrival diagnostics (arrival_aux), IGA_AUX_COLS doubles per
 * arrival row, all from the ray's Jacobian auxiliaries (calc_amp = 1; zero
 * otherwise):
 *   0  |d(x,y)/d(inclination)| of the ground intercept [km/rad], formed as
 *      find_eigenray forms its Newton derivatives (geoac.eigenray.3d.cpp:334-348;
 *      spherical: d(lat,lon) of geoac.eigenray.sph.cpp:351-359 scaled to
 *      ground distance by r_grnd and r_grnd cos(lat))
 *   1  |d(x,y)/d(azimuth)| of the ground intercept [km/rad]
 *   2  ray-tube Jacobian D at the arrival row (geoac::jacobian); amplitude
 *      is proportional to |D|^-1/2, so |D| -> 0 marks a caustic
 *   3  caustics passed so far: sign changes of D between consecutive RK4 rows,
 *      counted as the write_caustics output does (main.infraga.3d.cpp:448-480) */
#define IGA_AUX_COLS 4

typedef struct iga_atmo_s* iga_atmo_t;

/* One stratified profile already in solver units (the values set_region
 * stores after conversion, atmo_io.3d.strat.cpp:106-124). */
typedef struct iga_profile {
    int n;                   /* number of altitude knots (>= 3) */
    const double* z;         /* [n] km, increasing */
    const double* c;         /* [n] km/s adiabatic sound speed */
    const double* u;         /* [n] km/s east wind */
    const double* v;         /* [n] km/s north wind */
    const double* rho;       /* [n] g/cm^3 */
} iga_profile;

/* Ray-fan parameters: the geoac globals (geoac.params.3d.cpp:27-41), the
 * topo::z0 ground height and the run_prop locals (main.infraga.3d.cpp:206-215). */
typedef struct iga_fan_params {
    int geometry;            /* IGA_GEOM_3D or IGA_GEOM_SPH */
    int precision;           /* IGA_FP64, IGA_FP32C or IGA_FP32C_FLAGGED */
    int bounces;             /* reflections to follow (>= 0) */
    int calc_amp;            /* 1: 18 equations with the Jacobian auxiliaries */
    int write_rays;          /* 1: sum time/absorption per step like the CLI's
                                write_rays=true path (all segments but the last of
                                each bounce, main.infraga.3d.cpp:451-453) */
    int block;               /* threads per CTA of the fan launch: 0 = 128, else 32, 64, 96 or 128
                                (iga_fan_tune picks one by timing the fan) */
    double src[3];           /* 3D: source x, y [km], altitude [km];
                                SPH: source latitude, longitude [deg], altitude [km] */
    double ds_min, ds_max, s_max;
    double alt_max, rng_max, x_min, x_max, y_min, y_max;
    double z_grnd;           /* topo::z0 */
    double freq;             /* Hz */
    double tweak_abs;        /* atmo::tweak_abs (abs_coeff=) */
    double turn_ht_min;      /* km */
    /* IGA_GEOM_SPH only: break_check region (geoac.params.sph.cpp:33-37, in
       degrees here) and run_prop's travel-time cap [hours] */
    double lat_min, lat_max, lon_min, lon_max;
    double time_max;
} iga_fan_params;

/* ---- library / device ---- */
const char* iga_strerror(int status);
const char* iga_last_cuda_error(void);   /* thread-local text of the last CUDA failure */
int iga_version(void);                    /* IGA_ABI_VERSION */
int iga_device_count(int* count);

/* ---- atmospheres ---- */

/* Replaces set_region(atmo_file, format, invert_winds)
 * (src/atmo/atmo_io.3d.strat.cpp:55-143 and atmo_io.sph.strat.cpp): parses a
 * .met profile ("zTuvdp", "zuvwTdp" or "zcuvd"), builds the FP64 natural cubic
 * spline slopes (interp::set, src/util/interpolation.cpp:103-136) on the host
 * and uploads the tables to the current CUDA device. */
int iga_atmo_load(const char* met_path, const char* format, int reverse_winds, iga_atmo_t* out);

/* Replaces set_region(prefix, x_file, y_file[, topo_file], format,
 * invert_winds) of the range-dependent solvers
 * (src/atmo/atmo_io.sph.rngdep.cpp:61-311, src/atmo/atmo_io.3d.rngdep.cpp:58-330).
 * geometry = IGA_GEOM_SPH: latitude and longitude node lists [deg] and terrain
 * rows "lat lon z" [deg, deg, km]; IGA_GEOM_3D: x and y node lists [km] and
 * terrain rows "x y z" [km].  Node profiles are {prefix}{n}.met with
 * n = i_x * n_y + i_y.  Builds the hybrid-spline node tables (interp::set for
 * hybrid_spline_3D, src/util/interpolation.cpp:910-1045) and the terrain
 * spline tables in FP64 on the host and uploads them.  topo_file may be NULL
 * (flat ground).  Such a handle runs FP64 fans of the geometry it was loaded
 * for. */
int iga_atmo_load_rngdep(const char* prefix, const char* x_file, const char* y_file, const char* topo_file,
                         const char* format, int reverse_winds, int geometry, iga_atmo_t* out);

/* Replaces set_region(atmo_file, topo_file, format, invert_winds) of
 * infraga-3d and infraga-sph (src/atmo/atmo_io.3d.strat.cpp:146-258,
 * src/atmo/atmo_io.sph.strat.cpp): a .met profile as iga_atmo_load over a
 * terrain file of rows "x y z" [km] (IGA_GEOM_3D) or "lat lon z" [deg, deg,
 * km] (IGA_GEOM_SPH), first coordinate major as for iga_atmo_load_rngdep.
 * The handle behaves as a range-dependent one of that geometry
 * (iga_atmo_region gives the terrain extent less 0.001 km or 1e-3 deg,
 * iga_atmo_terrain works, FP64 only) and runs the stratified solver's
 * equations over the terrain. */
int iga_atmo_load_topo(const char* met_path, const char* topo_file, const char* format, int reverse_winds,
                       int geometry, iga_atmo_t* out);

/* Horizontal propagation region of an atmosphere (geoac::set_limits): for a
 * range-dependent grid its node extent, intersected with the terrain extent,
 * less 1e-3 deg (spherical, degrees) or 0.001 km (3D, km) on each side; the
 * whole globe in degrees for a 1D profile. */
int iga_atmo_region(iga_atmo_t atmo, double* lat_min, double* lat_max, double* lon_min, double* lon_max);

/* Terrain height and gradient at a horizontal point of a range-dependent
 * handle loaded with a terrain file: topo::z and topo::dz
 * (src/atmo/atmo_state.sph.rngdep.cpp:58-97, atmo_state.3d.rngdep.cpp:45-80),
 * with the point clamped into the terrain grid.  Spherical: x, y = latitude,
 * longitude in RADIANS, z = height above r_earth [km], gradient per radian;
 * 3D: x, y [km], gradient per km.  IGA_E_UNSUPPORTED without terrain. */
int iga_atmo_terrain(iga_atmo_t atmo, double x, double y, double* z, double* dz_dx, double* dz_dy);

/* atmo::c, u, v, rho as the reference's point functions return them
 * (atmo_state.*.cpp: the splines at the clamped altitude, u and v scaled by
 * topo::bndlyr_sc over the handle's ground or terrain), at the horizontal point
 * (x, y) [km; IGA_GEOM_SPH: lat, lon in deg] and altitudes z[0..n) [km]; out
 * gets n rows of c [km/s], u, v [km/s], rho [g/cm^3].  params gives the
 * geometry and the flat ground height (z_grnd).  Host-side FP64; used for the
 * write_atmo profile dump (geoac::write_prof, geoac.interface.3d.cpp:47-66,
 * geoac.interface.sph.cpp:55-73). */
int iga_atmo_sample(iga_atmo_t atmo, const iga_fan_params* params, double x, double y, const double* z, int n,
                    double* out);

/* Same as iga_atmo_load from arrays already in solver units. */
int iga_atmo_create(const iga_profile* profile, iga_atmo_t* out);

/* Propagation limits the reference derives from the profile
 * (geoac::set_limits, atmo_io.3d.strat.cpp:24-37): z_ground = first knot,
 * z_top = last knot. */
int iga_atmo_limits(iga_atmo_t atmo, double* z_ground, double* z_top);

int iga_atmo_destroy(iga_atmo_t atmo);

/* Defaults of run_prop after set_region for a flat-ground 3D run
 * (main.infraga.3d.cpp:206-215, geoac.params.3d.cpp:27-41,
 * atmo_io.3d.strat.cpp:24-37): bounces 10, calc_amp 1, write_rays 0,
 * ds 0.001..0.05, s_max 1000, alt_max = z_top, rng_max 2000, x/y +-2000,
 * z_grnd = z_ground, freq 0.1, tweak_abs 1, turn_ht_min 0.2. */
int iga_fan_params_default(iga_atmo_t atmo, iga_fan_params* params);

/* Defaults for either geometry.  IGA_GEOM_3D: as iga_fan_params_default.
 * IGA_GEOM_SPH: run_prop of infraga-sph (main.infraga.sph.cpp:207-222,
 * geoac.params.sph.cpp:23-37, atmo_io.sph.strat.cpp:27-39): source at
 * latitude 30, longitude 0, altitude 0; rng_max 1000; latitude +-90,
 * longitude +-180; time_max 10 h; the other fields as for 3D.  On a
 * range-dependent handle (run_prop of infraga-sph-rngdep,
 * main.infraga.sph.rngdep.cpp:207-239): 2 bounces, the iga_atmo_region
 * limits, and the source at the centre of that region.  IGA_GEOM_3D on a
 * 3D range-dependent handle (main.infraga.3d.rngdep.cpp:210-242): x/y limits
 * from iga_atmo_region, source at its centre, rng_max 1000. */
int iga_fan_params_init(iga_atmo_t atmo, int geometry, iga_fan_params* params);

/* ---- ray fans ---- */

/* Replaces the per-ray loop body of run_prop (src/main.infraga.3d.cpp:421-541):
 * geoac::set_initial, prop_rk4 (src/util/rk4solver.cpp:14-85), travel_time,
 * atten, amp and set_refl (src/geoac/geoac.eqset.3d.strat.cpp) for every ray
 * of a fan at once.  theta_deg/phi_deg are the launch inclination and the
 * azimuth (degrees clockwise from north, as on the command line) of each ray.
 *
 * Host buffers.  arrivals receives up to `cap` rows of IGA_ARRIVAL_COLS
 * doubles, ordered by ray then bounce (the reference's file order);
 * *n_out = rows produced (if > cap, rows past cap are dropped and
 * IGA_E_TRUNCATED is returned).  ray_index (nullable, cap ints) gets the ray
 * of each row; ray_steps (nullable, n_rays) the accepted RK4 steps of each
 * ray (the sum of prop_rk4's returned k); ray_status (nullable, n_rays) an
 * iga_ray_status; total_steps (nullable) the sum over all rays;
 * arrival_aux (nullable, cap rows of IGA_AUX_COLS) the diagnostics above. */
int iga_fan_run(iga_atmo_t atmo, const iga_fan_params* params,
                const double* theta_deg, const double* phi_deg, int n_rays,
                double* arrivals, int cap, int* n_out, int* ray_index,
                long long* ray_steps, int* ray_status, long long* total_steps,
                double* arrival_aux);

/* Launch-shape autotuner (no counterpart in the reference, whose CPU loop has
 * no launch shape): runs the fan once per candidate CTA size (32, 64, 96 and
 * 128 threads; after one untimed warm-up run) and returns the fastest in
 * *best_block, to be passed as params->block to later runs of that fan (or
 * fans of the same size and kind).  seconds (nullable, 4 doubles) gets each
 * candidate's device time.  The persistent fan kernels give each resident
 * thread one ray at a time: small fans leave SMs idle with large CTAs, while
 * large fans fill the GPU either way. */
int iga_fan_tune(iga_atmo_t atmo, const iga_fan_params* params, const double* theta_deg, const double* phi_deg,
                 int n_rays, int* best_block, double* seconds);

/* Bytes of device workspace iga_fan_run_device needs (ray queue counters). */
size_t iga_fan_workspace_bytes(void);

/* Device-resident form of iga_fan_run for callers that keep inputs and
 * outputs in device memory.  All pointers are device pointers on the
 * atmosphere's device; the launch is asynchronous on `stream`
 * (a cudaStream_t, NULL = legacy default stream).
 *   d_arrivals  [n_rays * (bounces + 1) * IGA_ARRIVAL_COLS] doubles; row j of
 *               ray i at (i * (bounces + 1) + j)
 *   d_n_arr     [n_rays] ints, arrivals of each ray
 *   d_ray_steps [n_rays] long longs
 *   d_ray_status[n_rays] ints (nullable)
 *   d_arrival_aux [n_rays * (bounces + 1) * IGA_AUX_COLS] doubles (nullable),
 *               laid out like d_arrivals
 *   d_workspace iga_fan_workspace_bytes() bytes, 16-byte aligned; the call
 *               resets it on `stream` before the launch */
int iga_fan_run_device(iga_atmo_t atmo, const iga_fan_params* params,
                       const double* d_theta_deg, const double* d_phi_deg, int n_rays,
                       double* d_arrivals, int* d_n_arr, long long* d_ray_steps,
                       int* d_ray_status, double* d_arrival_aux, void* d_workspace, void* stream);

/* ---- sampled ray paths, terrain samples and caustics ---- */

/* Path row: the reference's .raypaths.dat columns (main.infraga.3d.cpp:381-388;
 * spherical: lat, lon [deg] instead of x, y) and the bounce of the row:
 *   x|lat, y|lon, z [km], trans. coeff. [dB] (0 without calc_amp),
 *   absorption [dB] (-2 x the running sum), time [s], bounce.
 * In IGA_PATH_TERRAIN mode column 2 is the ground height under the row
 * (.terrain.dat, main.infraga.3d.cpp:481-486) and column 3 is 0. */
#define IGA_PATH_COLS 7
/* Caustic row: x|lat, y|lon, z [km], time [s], bounce (.caustics-N.dat,
 * main.infraga.3d.cpp:470-475; the 3D range-dependent CLI also writes a
 * 0.0 column before the time, main.infraga.3d.rngdep.cpp:467-471). */
#define IGA_CAUSTIC_COLS 5
/* Back-projection row (.projection.dat of run_back_proj,
 * main.infraga.3d.cpp:673-690 and :711-735): x, y, z [km], time [s],
 * X_incl, Y_incl, Z_incl [km/deg], T_incl [s/deg], X_az, Y_az, Z_az [km/deg],
 * T_az [s/deg], group velocity x, y, z [km/s].  The T columns are the
 * reference's travel_time_var sums (geoac.eqset.3d.strat.cpp:597-670), kept
 * as written: they are decremented, and the last d|c_g| term multiplies where
 * it should add. */
#define IGA_PROJ_COLS 15
enum iga_path_mode {
    IGA_PATH_RAYS = 0,       /* rows m == 1 and m % 15 == 0 of every bounce (write_rays) */
    IGA_PATH_TERRAIN = 1,    /* rows m % 10 == 1 (write_topo) */
    IGA_PATH_PROJ = 2,       /* rows m == 1 and m % 5 == 0, IGA_PROJ_COLS wide (-back_proj);
                                3D stratified flat-ground and 3D range-dependent handles
                                (run_back_proj of main.infraga.3d.cpp:559-770 and
                                main.infraga.3d.rngdep.cpp:548-750), calc_amp = 1, no caustics */
    IGA_PATH_RESID = 3       /* one row per bounce segment (prop_rk4 call) at its row k - 1
                                (print_resid, main.infraga.3d.cpp:437-441): eikonal residual,
                                auxiliary-parameter residual, bounce, then zeros
                                (geoac::eval_eikonal / eval_eikonal_deriv,
                                geoac.eqset.3d.strat.cpp:393-432); 3D stratified flat-ground
                                handles, no caustics.  Without calc_amp the auxiliary
                                residual is 0: the reference reads it from solution
                                columns 6..17 that its 6-equation rows do not have. */
};

/* Replaces the write_rays / write_topo / write_caustics branches of run_prop's
 * per-ray loop (src/main.infraga.3d.cpp:443-497, main.infraga.sph.cpp:455-510,
 * main.infraga.3d.rngdep.cpp:440-488, main.infraga.sph.rngdep.cpp:450-503)
 * and, with IGA_PATH_PROJ, the projection rows of run_back_proj
 * (main.infraga.3d.cpp:701-741; the caller passes the reversed-wind
 * atmosphere, the receiver as src and turn_ht_min = -1e30):
 * for every ray of the fan, the RK4 rows m (1 <= m < k of each bounce
 * segment) that the reference samples, with time and absorption summed per
 * step as the reference does whenever it writes paths (params->write_rays is
 * taken as 1), and the caustic points (sign changes of the ray-tube Jacobian
 * between consecutive rows; needs calc_amp = 1).  FP64 only.
 *   ray_steps   nullable: the per-ray step counts an iga_fan_run of the same
 *               fan returned; without it the call first counts them itself
 *   path_rows   nullable: path_cap rows of IGA_PATH_COLS; *n_path (needed
 *               when path_rows is given) = rows produced; path_start
 *               (nullable, n_rays + 1) = first row of each ray and the total.
 *               The rows of ray i number at most
 *               (bounces + 1) + ray_steps[i] / 15 (IGA_PATH_RAYS; / 10 for
 *               IGA_PATH_TERRAIN, / 5 for IGA_PATH_PROJ) + 1; IGA_PATH_PROJ
 *               rows are IGA_PROJ_COLS wide; IGA_PATH_RESID gives at most
 *               bounces + 1 rows per ray.
 *   caustic_rows nullable: caustic_cap rows of IGA_CAUSTIC_COLS, ray by ray
 *               in step order; *n_caustic = rows produced; caustic_ray
 *               (nullable, caustic_cap) the ray of each row.
 * Returns IGA_E_TRUNCATED when either output had too little room (the counts
 * then give the room needed). */
int iga_fan_paths(iga_atmo_t atmo, const iga_fan_params* params,
                  const double* theta_deg, const double* phi_deg, int n_rays, int path_mode,
                  const long long* ray_steps,
                  double* path_rows, long long path_cap, long long* n_path, long long* path_start,
                  double* caustic_rows, long long caustic_cap, long long* n_caustic, int* caustic_ray);

/* ---- weakly non-linear waveform (-wnl_wvfrm) ---- */

/* Settings of run_wnl_wvfrm (main.infraga.3d.cpp:1087-1184) beyond the ray's:
 * fan carries the propagation settings (bounces, source, ds, limits, ground,
 * frequency of the absorption column, abs_coeff); its calc_amp and write_rays
 * are taken as 1, precision as IGA_FP64, and turn_ht_min is ignored (the
 * waveform driver has no turning-height cut). */
typedef struct iga_wnl_params {
    iga_fan_params fan;
    double ds_wvfrm;             /* geoac::ds_wvfrm: step scale of the Burgers solver (0.5) */
    double wvfrm_ref;            /* km of ray length where the source waveform is given (1.0) */
    double out_step;             /* km; below 1e4: a spectrum / waveform snapshot each time the
                                    ray length crosses a multiple of it (1e10: none) */
    double filt1_g, filt1_n1, filt1_n2;   /* wvfrm::filt1_* low-pass of the non-linear term (0.5, 4, 0.5) */
    double filt2_g, filt2_n1, filt2_n2;   /* wvfrm::filt2_* low-pass of the spectrum (0.75, 2, 1) */
    long long max_steps;         /* Heun steps per ray after which the ray is given up (status 2);
                                    no counterpart in the reference, whose loop is unbounded
                                    (1000000; 0 = that default) */
} iga_wnl_params;

/* Per-ray summary (info rows of IGA_WNL_INFO doubles, in this order). */
#define IGA_WNL_INFO 17
enum iga_wnl_info {
    IGA_WNL_STATUS = 0,     /* 0: waveform computed; 1: the ray never reached wvfrm_ref (u_out = 0);
                               2: max_steps reached (u_out: the waveform where it stopped) */
    IGA_WNL_STEPS = 1,      /* Heun steps of the Burgers solver over all bounces */
    IGA_WNL_SHIFTS = 2,     /* caustic phase shifts applied ("Caustic encountered.") */
    IGA_WNL_EVENTS = 3,     /* event rows produced (may exceed event_cap) */
    IGA_WNL_SNAPS = 4,      /* snapshots produced (may exceed snap_cap) */
    IGA_WNL_T_REF = 5,      /* travel time to the reference row: the time offset of .wvfrm_init.dat */
    IGA_WNL_P0 = 6,         /* max |p| of the source waveform [Pa] */
    IGA_WNL_SCALE = 7,      /* amplitude factor at the last row: p(t) = u_out * p0 * scale */
    IGA_WNL_LENGTH = 8,     /* ray length the waveform was carried along [km] (the reference's running sum) */
    IGA_WNL_C0 = 9, IGA_WNL_RHO0 = 10, IGA_WNL_NU0 = 11, IGA_WNL_CG0 = 12, IGA_WNL_D0 = 13,
                            /* sound speed, density, |nu|, |c_g| and Jacobian at the reference row */
    IGA_WNL_OOB = 14,       /* spline look-ups outside the ray's knots (the reference prints
                               "Cannot interpolate outside of given bounds" for each) */
    IGA_WNL_BETA0 = 15,     /* the non-linearity coefficient beta0 */
    IGA_WNL_TIME = 16       /* travel time summed per bounce to its row k - 1 (the driver's
                               travel_time_sum; the arrival row's time when the ray lands) */
};
/* Event row: type (0: the "Computing waveform at ray length" line of every
 * 10 km, 1: "Caustic encountered."), ray length [km], altitude [km], beta. */
#define IGA_WNL_EVENT_COLS 4

/* Defaults of run_wnl_wvfrm after set_region (fan as iga_fan_params_default; for
 * infraga-sph's waveform mode set fan with iga_fan_params_init(atmo,
 * IGA_GEOM_SPH, &params->fan) afterwards). */
int iga_wnl_params_default(iga_atmo_t atmo, iga_wnl_params* params);

/* Replaces run_wnl_wvfrm's bounce loop with geoac::wnl_wvfrm
 * (src/main.infraga.3d.cpp:1281-1347, src/geoac/geoac.eqset.3d.strat.cpp:753-1045;
 * with fan.geometry = IGA_GEOM_SPH, src/main.infraga.sph.cpp:1270-1325 and
 * geoac.eqset.sph.strat.cpp:855-1130, source latitude / longitude in degrees)
 * for n_rays rays of a stratified flat-ground atmosphere at once: each ray
 * is traced (FP64, calc_amp), the source waveform (wv_t, wv_p: len samples of
 * t [s] and p [Pa]; len a power of two from 16 to 8192) is given at ray length
 * wvfrm_ref and carried to the end of the last bounce by the reference's
 * Heun / FFT Burgers scheme with absorption, caustic phase shifts and filters.
 *   u_out       [n_rays][len] waveform at the end scaled by 1 / p0; the
 *               reference's .wvfrm_out.dat column is u_out * p0 * scale at
 *               t = (arrival time) + wv_t
 *   info        [n_rays][IGA_WNL_INFO] (iga_wnl_info)
 *   arrivals    nullable: [n_rays][bounces + 1][IGA_ARRIVAL_COLS] the fan's
 *               arrival rows (time / absorption summed per step, as the
 *               waveform driver does); n_arr, ray_status nullable [n_rays]
 *   events      nullable: [n_rays][event_cap][IGA_WNL_EVENT_COLS]
 *   snaps       nullable: [n_rays][snap_cap][1 + len + 2 (len / 2 + 1)]:
 *               the ray length label, u (scaled), then the spectrum U as
 *               (re, im) pairs (sc_waveform / sc_spectrum of out_step)
 * Returns IGA_E_TRUNCATED when events or snapshots had too little room (info
 * holds the counts needed). */
int iga_wnl_run(iga_atmo_t atmo, const iga_wnl_params* params, const double* theta_deg, const double* phi_deg,
                int n_rays, const double* wv_t, const double* wv_p, int len, double* u_out, double* info,
                double* arrivals, int* n_arr, int* ray_status, double* events, int event_cap, double* snaps,
                int snap_cap);

/* ---- eigenray search ---- */

/* One source-receiver pair of an eigenray search (receiver on the ground).
 * 3D: x, y [km]; IGA_GEOM_SPH (params->fan.geometry): latitude, longitude
 * [deg], as on infraga-sph's command line; altitude [km]. */
typedef struct iga_eig_pair {
    double src[3];           /* source x|lat, y|lon, altitude */
    double rcvr[2];          /* receiver x|lat, y|lon */
} iga_eig_pair;

/* Eigenray search settings: run_eig_search's locals and the geoac::eigenray
 * globals (main.infraga.3d.cpp:779-791, geoac.eigenray.3d.cpp:21-28).
 * fan carries the propagation settings (ds, s_max, limits, ground, frequency,
 * absorption, precision); its bounces/calc_amp/write_rays/src are ignored. */
typedef struct iga_eig_params {
    iga_fan_params fan;
    double incl_min, incl_max;   /* deg; search range (0.5, 45) */
    double incl_step_min;        /* deg; geoac::dth_sml (0.001) */
    double incl_step_max;        /* deg; geoac::dth_big (0.1) */
    double damping;              /* geoac::damping (1e-3) */
    double tolerance;            /* km; geoac::tolerance (0.1) */
    double az_err_lim;           /* deg; az_dev_lim (2) */
    int bnc_min, bnc_max;        /* bounce counts searched (0, 0) */
    int iterations;              /* Newton iteration limit (25) */
    int chunk;                   /* sweep inclinations traced per search per GPU round (0 = automatic) */
    int streams;                 /* pair groups searched concurrently, each on its own host thread and
                                    CUDA stream (0 = automatic = 1: on large searches the sweep launches
                                    already fill the GPU, and more groups measured slower) */
} iga_eig_params;

/* Defaults of run_eig_search after set_region (fan as iga_fan_params_default;
 * on a range-dependent handle as iga_fan_params_init for its geometry). */
int iga_eig_params_default(iga_atmo_t atmo, iga_eig_params* params);

/* Replaces run_eig_search's search loop (src/main.infraga.3d.cpp:939-950):
 * for every pair and every bounce count in [bnc_min, bnc_max], the inclination
 * sweep with azimuth correction of geoac::est_eigenray
 * (src/geoac/geoac.eigenray.3d.cpp:34-144) and the damped Newton refinement of
 * geoac::find_eigenray (:146-371), all searches running together (every ray
 * trace of a round is one GPU launch).  Output rows (IGA_ARRIVAL_COLS) are the
 * reference's eigenray .arrivals.dat rows, ordered by pair, bounce count, then
 * discovery; pair_index (nullable) gets each row's pair; total_steps
 * (nullable) the RK4 steps of every trace.  Capacity/truncation as iga_fan_run.
 * The reference's find_eigenray follows only the first reflection during its
 * Newton iterations (an unconditional break, geoac.eigenray.3d.cpp:206) while
 * its final trace and output use all bounces; that is reproduced.
 * fan.precision = IGA_FP32C traces the rays in FP32-compensated form (the
 * fan kernel's arithmetic) while the bracket and Newton updates stay in FP64;
 * the eigenrays found then agree with the FP64 search to within the search
 * tolerance (0.1 km at the receiver) rather than to rounding.
 * fan.geometry = IGA_GEOM_SPH (fan from iga_fan_params_init(atmo,
 * IGA_GEOM_SPH, ...)) runs infraga-sph's search instead
 * (src/geoac/geoac.eigenray.sph.cpp:42-380, main.infraga.sph.cpp:965-990):
 * great-circle ranges and bearings, the fixed sweep step until 3 azimuth
 * corrections, Newton iterations through every bounce, rows with latitude /
 * longitude in columns 3-4 (FP64 only; stratified profiles). */
int iga_eig_run(iga_atmo_t atmo, const iga_eig_params* params, const iga_eig_pair* pairs, int n_pairs,
                double* eigenrays, int cap, int* n_out, int* pair_index, long long* total_steps);

/* Replaces run_eig_direct's call of geoac::find_eigenray
 * (src/main.infraga.3d.cpp:1079-1080, src/geoac/geoac.eigenray.3d.cpp:146-371):
 * the damped Newton refinement alone, from the launch estimate incl_est
 * [deg] and az_est [deg clockwise from north] for `bounces` reflections, with
 * params' damping, tolerance and iteration limit.  *found = 1 and eigenray
 * (IGA_ARRIVAL_COLS doubles, the row iga_eig_run would give) are set when the
 * arrival came within tolerance of the receiver; *found = 0 otherwise. */
int iga_eig_direct(iga_atmo_t atmo, const iga_eig_params* params, const iga_eig_pair* pair, double incl_est,
                   double az_est, int bounces, double* eigenray, int* found, long long* total_steps);

/* Allocation-free form of iga_fan_run_device.  No counterpart in the
 * reference (which has no GPU path); it exists for callers that must not
 * allocate device memory themselves: applications that reserve their whole
 * device budget up front and keep cudaMalloc off the request path (it can
 * block and synchronise the device, which breaks their latency targets), and
 * host frameworks whose own allocator owns all device memory, where a library
 * allocation would bypass its accounting.  Inputs and outputs are the caller's
 * device buffers exactly as for iga_fan_run_device; only the ray-queue scratch
 * differs: instead of a caller workspace it uses a fixed
 * IGA_FAN_STATIC_SCRATCH_BYTES array compiled into the library, which every
 * device that loads the library keeps until the process exits.
 *   - FP64 only (IGA_E_UNSUPPORTED for IGA_FP32C, whose absorption table is
 *     built and uploaded on first use of a frequency).
 *   - Returns IGA_E_INVALID when the fan's scratch need
 *     (iga_fan_workspace_bytes()) exceeds IGA_FAN_STATIC_SCRATCH_BYTES.
 *   - The first call on a device looks up that device's address of the array
 *     (one-time set-up, serialised internally); make that first call before
 *     any stream capture starts.  That first call is also when the driver
 *     loads the library's device code and its static array and reserves the
 *     local (stack) memory the fan kernel needs: one-time allocations by the
 *     driver, not by this library.  Make one warm-up call during set-up, before
 *     latency-critical work; later calls leave device memory use unchanged.
 *   - The address is kept per device for the life of the process.  A
 *     cudaDeviceReset of that device invalidates it, together with every
 *     atmosphere handle on the device: reload the library's handles and do not
 *     call this entry point on a device that was reset.
 *   - All calls share the one array (the call clears it on `stream` before
 *     launching), so calls whose work overlaps on the GPU race: issue them on
 *     one stream or otherwise order them.
 *   - Calls no cudaMalloc, cudaFree or other allocating routine. */
#define IGA_FAN_STATIC_SCRATCH_BYTES 256
int iga_fan_run_device_noalloc(iga_atmo_t atmo, const iga_fan_params* params,
                               const double* d_theta_deg, const double* d_phi_deg, int n_rays,
                               double* d_arrivals, int* d_n_arr, long long* d_ray_steps,
                               int* d_ray_status, double* d_arrival_aux, void* stream);

/* ---- request server (continuous batching on one GPU) ----
 * No counterpart in the reference (its CLI runs one job per process).  A
 * server keeps the callers' atmosphere handles resident, queues fan and
 * eigenray requests, admits them as slots (CUDA streams) and device memory
 * (hbm_budget) free up, and runs admitted requests concurrently on the GPU.
 * A request's results are those of iga_fan_run / iga_eig_run for the same
 * inputs, alone or in any mix. */
typedef struct iga_server_s* iga_server_t;

typedef struct iga_server_config {
    int device;              /* CUDA device of the server and of the atmospheres it serves */
    int max_inflight;        /* concurrent fan requests (streams); default 8 */
    int eig_workers;         /* concurrent eigenray requests; default 2 */
    int small_rays;          /* fans up to this size use high-priority streams and no CTA cap; 4096 */
    double big_fan_sm_frac;  /* larger fans use at most this fraction of the resident CTA slots; 0.75 */
    size_t hbm_budget;       /* device bytes all admitted requests may hold; default 8 GiB */
} iga_server_config;

typedef struct iga_server_stats {
    long long completed, pending;
    double p50_s, p99_s;             /* submit -> results on the host, all completed requests */
    double fan_p50_s, fan_p99_s, eig_p50_s, eig_p99_s;
    long long ray_steps, rays, eigenrays;
    double wall_s;                   /* first submit -> last completion */
    size_t bytes_in_use;
} iga_server_stats;

int iga_server_config_default(iga_server_config* config);
int iga_server_create(const iga_server_config* config, iga_server_t* out);
/* Queue a fan (inputs copied; returns at once).  id identifies the request. */
int iga_server_submit_fan(iga_server_t server, iga_atmo_t atmo, const iga_fan_params* params,
                          const double* theta_deg, const double* phi_deg, int n_rays, long long* id);
int iga_server_submit_eig(iga_server_t server, iga_atmo_t atmo, const iga_eig_params* params,
                          const iga_eig_pair* pairs, int n_pairs, long long* id);
/* done = 1 once the request's results are on the host.  timeout_s: 0 polls,
 * < 0 waits without limit. */
int iga_server_wait(iga_server_t server, long long id, double timeout_s, int* done);
/* Copy a finished request's rows (IGA_ARRIVAL_COLS each; fan: ray by ray,
 * index = ray; eigen: as iga_eig_run, index = pair) and release it.  With
 * cap < n_out it returns IGA_E_TRUNCATED and keeps the request. */
int iga_server_fetch(iga_server_t server, long long id, double* rows, int cap, int* n_out, int* index,
                     long long* total_steps, double* latency_s);
int iga_server_get_stats(iga_server_t server, iga_server_stats* stats);
/* Finishes the requests on the GPU, drops the queued ones, frees the server. */
int iga_server_destroy(iga_server_t server);

#ifdef __cplusplus
}
#endif
#endif /* INFRAGA_GPU_H_ */

// Launch arguments shared by the 3D stratified fan kernels and the C ABI.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "device_common.cuh"

namespace iga {

// Everything a fan launch needs, by value (kernel parameter space).
struct Fan3DArgs {
    // atmosphere knot table (device, kStride doubles per knot)
    const double* knots;
    int n_knots;
    int uniform;
    double z_lo, z_hi, inv_dz;
    // rays
    const double* theta_deg;
    const double* phi_deg;
    int n_rays;
    int bounces;
    int write_rays;
    int length;              // int(s_max / ds_min): prop_rk4's row budget
    // outputs
    double* arrivals;        // [n_rays][bounces+1][12]
    int* n_arr;
    long long* ray_steps;
    int* ray_status;         // nullable
    double* aux;             // nullable: [n_rays][bounces+1][4] per-arrival diagnostics
    unsigned int* queue;     // [0] next ray (device ray queue)
    int grid_cap;            // > 0: at most this many CTAs (the request server shares the GPU)
    int block;               // > 0: threads per CTA of the fan launch (a multiple of 32 up to the kernel's
                             // compiled maximum); 0: that maximum
    // sampled per-step output (run_prop's write_rays / write_topo / write_caustics);
    // all null on the plain fan path
    double* path_rows;       // [path_off[n_rays]][kPathCols]
    const long long* path_off;   // [n_rays + 1]: row range of each ray
    long long* path_n;       // [n_rays]: rows the ray produced (may exceed its range: dropped)
    int path_mode;           // kPathRays or kPathTerrain
    double* caus_rows;       // [caus_cap][kCausCols], appended in any order
    unsigned long long* caus_count;
    long long caus_cap;
    // geometry / limits
    double src_x, src_y, src_z;
    double ds_min, ds_max, s_max;
    double alt_max, rng_max, x_min, x_max, y_min, y_max;
    double z0;               // flat ground height (topo::z0)
    double z_bl;             // boundary-layer top (topo::z_bndlyr = z0 + 2)
    double bl;               // topo::bndlyr_param
    double inv_bl;
    double freq, tweak_abs, turn_ht_min;
    // per-launch constants evaluated on the host (source and ground point)
    double c0;               // c at the source
    double u0s, v0s;         // winds at the source (boundary-layer scaled)
    double rho0;             // rho at the source
    double c_gnd;            // c at the ground height
    double dcz_g, duz_g, dvz_g;   // z-derivatives of c, u, v at the ground (set_refl)
    double c_ratio;          // c_gnd / c0 (arrival inclination)
    SBConst sb;
    // spherical geometry only (src_x/src_y hold the source latitude and
    // longitude in radians; z-like quantities above are altitudes)
    double r_earth;          // globe::r0
    double r_grnd;           // topo::z = r_earth + z0 (flat ground radius)
    double cos_lat_src;
    double lat_min, lat_max, lon_min, lon_max;   // radians (break_check)
    double time_max_h;       // run_prop's travel-time cap [hours]
    double hav_rng;          // sin^2(rng_max / (2 r_earth)): haversine range threshold
    int rng_exact_only;      // 1: rng_max >= pi r_earth or the threshold is unusable
    double refl_k1;          // c0 / c_grnd * dc/dr at the ground (set_refl dnu_r_ds)
    double refl_k2;          // c_grnd^2 / c0 / r_grnd
    double refl_k3;          // -1 / c_grnd
    double refl_mcr;         // -c0 / c_grnd
    // range-dependent atmosphere and terrain (spherical range-dependent kernel)
    const double* hyb_tab;   // [nx][ny][nz][64] node records (atmo_rngdep.h)
    const double* hyb_x;     // node latitudes [rad]
    const double* hyb_y;     // node longitudes [rad]
    const double* hyb_z;     // knot altitudes [km]
    int hyb_nx, hyb_ny, hyb_nz;
    const double* topo_tab;  // [nx][ny][4] terrain f, f_lat, f_lon, f_lat,lon (null: flat ground at z0)
    const double* topo_x;
    const double* topo_y;
    int topo_nx, topo_ny;
    double topo_zmax;        // topo::z_max of ground_check (max terrain + 0.01, or z0)
    double x_cut;            // r - r_earth above which exp(-(r - z_g)/bl) < 1e-173 everywhere
    // FP32-compensated path only
    const double* knots_c;   // [n_knots][kStrideC]: per segment z_k, 1/dz and the power-basis
                             // cubic coefficients a0..a3 of c, u, v in X = (z - z_k)/dz
                             // (last row: z only)
    const float* alpha_tab;  // Sutherland-Bass alpha(z) [dB/km, tweak_abs = 1] on a uniform grid
    int alpha_n;
    double alpha_z0, alpha_inv_h;
    const float* hyb_x32;    // [nx][ny][nz][kHybX32] FP32 copies of the hybrid records'
                             // second-derivative blocks (c, u, v: 9 values each)
    int retrace;             // FP32C: 1 = mark focusing rays for the FP64-auxiliary re-trace,
                             // 0 = flag them (kRayFocus) and keep tracing
};

constexpr int kHybX32 = 32;   // floats per record of hyb_x32 (3 x 9 used)

constexpr int kStrideC = 14;  // doubles per segment row of the FP32-compensated path's power-basis table

// Flag OR'ed into a ray's status (IGA_RAY_AUX_FP64): an FP32C ray traced
// again with FP64 auxiliaries after a focusing arrival.
constexpr int kRayAuxFp64 = 0x100;
// Flag OR'ed into a ray's status (IGA_RAY_FOCUS): an FP32C ray that met a
// focusing arrival and, without the re-trace pass, kept its FP32 auxiliaries.
constexpr int kRayFocus = 0x200;

// Sampled output rows.  Path rows: horizontal position (x, y [km] or lat, lon
// [deg]), altitude [km] (terrain mode: the ground height there), amplitude
// [dB] (0 without calc_amp or in terrain mode), absorption [dB] (-2 x the
// running sum), travel time [s], bounce.  Caustic rows: position (3), time,
// bounce, ray, and the ray's step index of the row (for ordering).
// Back-projection rows (kPathProj, 3D stratified flat-ground kernel only):
// x, y, z [km], time [s], X_incl (3) [km/deg], T_incl [s/deg], X_az (3),
// T_az, group velocity (3) [km/s].
constexpr int kPathCols = 7;
constexpr int kProjCols = 15;
constexpr int kCausCols = 7;
constexpr int kPathRays = 0;      // rows m == 1 and m % 15 == 0 of each bounce (raypaths)
constexpr int kPathTerrain = 1;   // rows m % 10 == 1 (terrain under the ray)
constexpr int kPathProj = 2;      // rows m == 1 and m % 5 == 0 (back projection)
constexpr int kPathResid = 3;     // one row per bounce segment: residuals at its row k - 1 (print_resid)
constexpr int kPathWnl = 4;       // every row m = 0..k of each bounce (weakly non-linear waveform), kWnlCols wide
// Waveform trace rows (kPathWnl, 3D stratified flat-ground kernel, calc_amp):
// x, y, z [km], nu_x, nu_y, nu_z, the ray-tube Jacobian D (geoac::jacobian),
// the travel time from the bounce's row 0 to this row (geoac::travel_time(solution, m)),
// bounce, m.
constexpr int kWnlCols = 10;

__host__ __device__ inline bool path_sampled(int mode, int m) {
    if (mode == kPathResid || mode == kPathWnl) return false;   // written by their own branches
    return mode == kPathRays ? (m == 1 || m % 15 == 0) : (mode == kPathTerrain ? (m % 10 == 1) : (m == 1 || m % 5 == 0));
}

__host__ __device__ inline int path_cols(int mode) {
    return mode == kPathProj ? kProjCols : (mode == kPathWnl ? kWnlCols : kPathCols);
}

// Upper bound on the path rows of a ray that took `steps` RK4 steps over at
// most `segments` bounce segments: each segment of K rows samples m in 1..K-1.
inline long long path_rows_bound(int mode, long long steps, int segments) {
    if (mode == kPathResid) return segments;
    if (mode == kPathWnl) return steps + segments;   // K + 1 rows per segment of K steps
    return (long long)segments + steps / (mode == kPathRays ? 15 : (mode == kPathTerrain ? 10 : 5)) + 1;
}

cudaError_t launch_fan3d_fp32c(const Fan3DArgs& a, bool calc_amp, cudaStream_t stream, int* grid_used);

cudaError_t launch_fan3d_fp64(const Fan3DArgs& a, bool calc_amp, cudaStream_t stream, int* grid_used);

// Spherical (global) stratified fan, FP64 (fansph_fp64.cu).
cudaError_t launch_fansph_fp64(const Fan3DArgs& a, bool calc_amp, cudaStream_t stream, int* grid_used);

// 3D Cartesian range-dependent fan with optional terrain, FP64 (fan3dr_fp64.cu).
cudaError_t launch_fan3dr_fp64(const Fan3DArgs& a, bool calc_amp, cudaStream_t stream, int* grid_used);

// Spherical range-dependent fan with optional terrain, FP64 (fansphr_fp64.cu).
cudaError_t launch_fansphr_fp64(const Fan3DArgs& a, bool calc_amp, cudaStream_t stream, int* grid_used);

// Spherical range-dependent fan with optional terrain, FP32-compensated
// (fansphr_fp32c.cu): the fan kernel and the FP64-auxiliary re-trace of its
// focusing rays, on `stream`.
cudaError_t launch_fansphr_fp32c(const Fan3DArgs& a, bool calc_amp, cudaStream_t stream, int* grid_used);

constexpr double kEarthRadiusKm = 6370.0;   // globe::r0 (util/globe.cpp:10)

}  // namespace iga

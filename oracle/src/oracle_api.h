// CPU oracle C API (test infrastructure only; loaded by tests/, smoke() and
// bench.py's cpu_baseline through ctypes; never linked into the product).
#pragma once
#ifdef __cplusplus
extern "C" {
#endif

#define ORC_ARR_COLS 12   // arrival row: incl az n_b x y time cel turn_ht arr_incl back_az amp_db atten_db
#define ORC_AUX_COLS 4    // per arrival: |d(x,y)/d theta|, |d(x,y)/d phi| [km/rad], Jacobian D, caustics so far

typedef struct orc_fan_cfg {
    double src[3];          // source x, y [km], altitude [km]
    double ds_min, ds_max, s_max;
    double alt_max, rng_max, x_min, x_max, y_min, y_max;
    double z_grnd;          // topo::z0
    double freq, tweak_abs, turn_ht_min;
    int bounces;
    int calc_amp;
    int write_rays;         // 1: per-step accumulation (all segments but the last)
    int reverse_winds;
    int n_threads;
} orc_fan_cfg;

// 3D Cartesian stratified ray fan, flat ground.  arrivals has room for
// n_rays * (bounces + 1) rows of ORC_ARR_COLS doubles; row j of ray i is at
// (i * (bounces + 1) + j).  n_arr[i] = arrivals written for ray i,
// steps[i] = accepted RK4 steps for ray i; aux (nullable) has ORC_AUX_COLS
// per arrival slot.  Returns 0, or -1 on a bad profile.
int orc_fan_3d(const char* met_path, const char* fmt, const orc_fan_cfg* cfg,
               const double* theta_deg, const double* phi_deg, int n_rays,
               double* arrivals, int* n_arr, long long* steps, double* aux);

#ifdef __cplusplus
}
#endif

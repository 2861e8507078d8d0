// FP64 ray-fan kernel: spherical (global) geometry, stratified atmosphere,
// flat ground at radius r_earth + z0.
//
// Same execution scheme as the 3D Cartesian kernel: one thread per ray,
// persistent grid pulling rays from a device queue, one RK4 step per loop
// iteration with ground hits, arrival records and reflections handled in the
// loop, the knot table in shared memory and row k-1 of each lane's ray in
// shared memory for the ground-intercept extrapolation.
//
// Physics follows the reference's spherical stratified equation set
// (src/geoac/geoac.eqset.sph.strat.cpp), its RK4 driver
// (src/util/rk4solver.cpp:14-85) and the per-ray loop of run_prop
// (src/main.infraga.sph.cpp:438-552).
#include "fan3d.cuh"
#include "fan3d_common.cuh"
#include "fansph_common.cuh"

namespace iga {

namespace {

#ifndef IGA_SPH_THREADS
#define IGA_SPH_THREADS 128
#endif
#ifndef IGA_SPH_MINB
#define IGA_SPH_MINB 2
#endif
constexpr int kThreads = IGA_SPH_THREADS;

// PATHS: also write the sampled per-step rows and caustic points of
// run_prop's write_rays / write_topo / write_caustics output
// (main.infraga.sph.cpp:455-510); the fan results are unchanged.
template <bool AMP, bool SMEM, bool PATHS>
__global__ void __launch_bounds__(kThreads, IGA_SPH_MINB) fansph_fp64_kernel(const __grid_constant__ Fan3DArgs a) {
    constexpr int N = DimSph<AMP>::n;
    extern __shared__ double s_mem[];
    double* s_prev = s_mem;
    const double* tab;
    if (SMEM) {
        double* s_tab = s_mem + N * blockDim.x;
        const int tot = a.n_knots * kStride;
        for (int i = threadIdx.x; i < tot; i += blockDim.x) s_tab[i] = a.knots[i];
        __syncthreads();
        tab = s_tab;
    } else {
        tab = a.knots;
    }
    double* prev = s_prev + threadIdx.x;   // element i at prev[i * blockDim.x]

    const int nb = a.bounces + 1;
    const double c_third = 1.0 / 3.0, c_sixth = 1.0 / 6.0;
    const double rad2deg = 180.0 / kPi;

    int ray = (int)atomicAdd(a.queue, 1u);
    if (ray >= a.n_rays) return;

    double y[N];
    int seg, bnc, kb, na, caustics;
    double D_prev = 0.0;
    long long steps;
    double s, tt, att, pt, pa, rmax;
    long long p_base = 0, p_cap = 0, p_n = 0;   // PATHS: this ray's row range and rows produced
    // PATHS, waveform trace rows: every row of every bounce (r, lat, lon, nu,
    // D, the bounce's travel time from its row 0, bounce, m)
    const bool wnl = PATHS && AMP && a.path_rows && a.path_mode == kPathWnl;
    double ttb = 0.0;
    auto wnl_row = [&](const double* yr, int m) {
        if (p_n < p_cap) {
            double* o = a.path_rows + (p_base + p_n) * kWnlCols;
            o[0] = yr[0]; o[1] = yr[1]; o[2] = yr[2];
            o[3] = yr[3]; o[4] = yr[4]; o[5] = yr[5];
            o[6] = row_jacobian_sph(tab, a, seg, yr);
            o[7] = ttb; o[8] = (double)bnc; o[9] = (double)m;
        }
        p_n++;
    };

    auto start_ray = [&](int r) {
        const double theta = a.theta_deg[r] * (kPi / 180.0);
        const double phi = kPi / 2.0 - a.phi_deg[r] * (kPi / 180.0);
        ray_init_sph<AMP>(a, theta, phi, y);
        seg = seg_guess(fmin(fmax(y[0] - a.r_earth, a.z_lo), a.z_hi), a.z_lo, a.inv_dz, a.n_knots);
        bnc = 0; kb = 0; na = 0; steps = 0; caustics = 0;
        s = 0.0; tt = 0.0; att = 0.0; pt = 0.0; pa = 0.0;
        rmax = 0.0;
        ttb = 0.0;
        if (PATHS && a.path_rows) { p_base = a.path_off[r]; p_cap = a.path_off[r + 1] - p_base; p_n = 0; }
    };
    start_ray(ray);

    while (true) {
        // ---- one RK4 step (rk4solver.cpp:30-55) ----
        if (wnl) wnl_row(y, kb);
        rmax = fmax(rmax, y[0] - a.r_earth);
        double ds = a.ds_max;   // set_ds (geoac.eqset.sph.strat.cpp:216-222)
        if (y[0] - a.r_earth < a.z_bl) ds -= (a.ds_max - a.ds_min) * exp(-(y[0] - a.r_grnd) / 0.2);
        s += ds;
        double acc[N], stg[N], f[N];
        rhs_sph<AMP>(tab, a, seg, y, f);
        if (AMP && (a.aux || (PATHS && a.caus_rows)) && kb >= 1) {   // caustics between rows 1..k-1 of the bounce
            const double D = ray_det_sph(f, y);
            if (kb >= 2 && D * D_prev < 0.0) {
                caustics++;
                if (PATHS && a.caus_rows) {   // row kb; time through segment (kb-1, kb)
                    const unsigned long long w = atomicAdd(a.caus_count, 1ull);
                    if ((long long)w < a.caus_cap) {
                        double* o = a.caus_rows + w * kCausCols;
                        o[0] = y[1] * rad2deg; o[1] = y[2] * rad2deg; o[2] = y[0] - a.r_earth; o[3] = tt + pt;
                        o[4] = (double)bnc; o[5] = (double)ray; o[6] = (double)(steps + kb);
                    }
                }
            }
            D_prev = D;
        }
#pragma unroll
        for (int i = 0; i < N; i++) { const double t = ds * f[i]; acc[i] = y[i] + t * c_sixth; stg[i] = y[i] + t * 0.5; }
        // stages 2..4 with one copy of the right-hand side (instruction-cache footprint)
#pragma unroll 1
        for (int st = 0; st < 3; st++) {
            rhs_sph<AMP>(tab, a, seg, stg, f);
            const double w = st < 2 ? c_third : c_sixth;
            const double c = st == 0 ? 0.5 : 1.0;
#pragma unroll
            for (int i = 0; i < N; i++) { const double t = ds * f[i]; acc[i] += t * w; stg[i] = y[i] + t * c; }
        }
        kb++;

        // ---- stop checks (rk4solver.cpp:57-75; break_check / ground_check,
        // geoac.eqset.sph.strat.cpp:484-506).  break_check wraps the longitude
        // of the new row in place before anything reads it. ----
        bool esc = s > a.s_max;
        if (!esc) {
            if (acc[2] > kPi) acc[2] -= 2.0 * kPi;
            else if (acc[2] < -kPi) acc[2] += 2.0 * kPi;
            esc = (acc[1] < -kPi / 2.0 || acc[1] > kPi / 2.0) || (acc[0] - a.r_earth > a.alt_max) ||
                  beyond_range(a, acc[1], acc[2]) || (acc[1] < a.lat_min || acc[1] > a.lat_max) ||
                  (acc[2] < a.lon_min || acc[2] > a.lon_max);
        }
        const bool gnd = !esc && (acc[0] - a.r_earth <= a.z0) && (acc[0] < a.r_grnd);

        double dt, da;
        seg_increment_sph(tab, a, seg, y, acc, dt, da);
        if (wnl) ttb += dt;
        if (a.write_rays) {   // all segments but the bounce's last (main.infraga.sph.cpp:466-468)
            tt += pt; att += pa; pt = dt; pa = da;
        } else {              // per-bounce sum added at the end (main.infraga.sph.cpp:496-497)
            pt += dt; pa += da;
        }

        bool capped = false, bad = false;
        if (!esc && !gnd) {
            if (kb >= a.length - 1) { capped = true; esc = true; }
            else if (!isfinite(acc[0]) || !isfinite(acc[1]) || !isfinite(acc[3])) { bad = true; esc = true; }
        }
        if (!esc && !gnd) {
#pragma unroll
            for (int i = 0; i < N; i++) { prev[i * blockDim.x] = y[i]; y[i] = acc[i]; }
            if (PATHS && a.path_rows && path_sampled(a.path_mode, kb)) {
                if (p_n < p_cap) {
                    double* o = a.path_rows + (p_base + p_n) * kPathCols;
                    o[0] = y[1] * rad2deg; o[1] = y[2] * rad2deg;
                    o[2] = a.path_mode == kPathRays ? y[0] - a.r_earth : a.r_grnd - a.r_earth;
                    int sg = seg;
                    o[3] = (AMP && a.path_mode == kPathRays)
                               ? amp_db_sph(tab, a, sg, y, a.theta_deg[ray] * (kPi / 180.0),
                                            kPi / 2.0 - a.phi_deg[ray] * (kPi / 180.0), nullptr)
                               : 0.0;
                    o[4] = -2.0 * (att + pa); o[5] = tt + pt; o[6] = (double)bnc;
                }
                p_n++;
            }
            continue;
        }

        // ---- end of a bounce segment (main.infraga.sph.cpp:459-548) ----
        const int K = capped ? a.length : kb;
        steps += K;
        if (wnl) wnl_row(acc, kb);   // row k: the first row beyond the segment's end
        if (!a.write_rays) { tt += pt; att += pa; }
        pt = 0.0; pa = 0.0;
        ttb = 0.0;
        int status = -1;
        if (rmax < a.z0 + a.turn_ht_min) status = 2;
        else if (esc) status = bad ? 4 : (capped ? 5 : 1);
        else if (K < 2) status = 3;
        else if (tt / 3600.0 > a.time_max_h) status = 6;
        if (status < 0) {
            // arrival record from the first below-ground row
            double* out = a.arrivals + ((size_t)ray * nb + na) * 12;
            const double th_deg = a.theta_deg[ray], ph_deg = a.phi_deg[ray];
            SphAtm mk;
            sph_atm<false>(tab, a, seg, acc[0], mk);
            const double incl = -asin(mk.c / a.c0 * acc[3]) * rad2deg;
            double baz = 90.0 - atan2(-acc[4], -acc[5]) * rad2deg;
            if (baz < -180.0) baz += 360.0;
            else if (baz > 180.0) baz -= 360.0;
            out[0] = th_deg;
            out[1] = ph_deg;
            out[2] = (double)bnc;
            out[3] = acc[1] * rad2deg;
            out[4] = acc[2] * rad2deg;
            out[5] = tt;
            out[6] = gc_dist(a.r_earth, acc[1], acc[2], a.src_x, a.src_y, a.cos_lat_src) / tt;
            out[7] = rmax;
            out[8] = incl;
            out[9] = baz;
            double jac = 0.0;
            out[10] = AMP ? amp_db_sph(tab, a, seg, acc, th_deg * (kPi / 180.0), kPi / 2.0 - ph_deg * (kPi / 180.0), &jac)
                          : 0.0;
            out[11] = -2.0 * att;
            if (a.aux) {
                double* ax = a.aux + ((size_t)ray * nb + na) * 4;
                if (AMP) write_aux_sph(ax, a, acc, jac, caustics);
                else ax[0] = ax[1] = ax[2] = ax[3] = 0.0;
            }
            na++;
            // reflection from rows k-2 (prev) and k-1 (y): approx_intercept
            // and set_refl (geoac.eqset.sph.strat.cpp:108-213) on flat ground,
            // where the terrain slopes a = b = 0 and their derivatives vanish
            const double dr_grnd = a.r_grnd - y[0];
            const double dr_k = y[0] - prev[0];
            double p[N];
#pragma unroll
            for (int i = 0; i < N; i++) p[i] = y[i] + (y[i] - prev[i * blockDim.x]) / dr_k * dr_grnd;
            y[0] = a.r_grnd; y[1] = p[1]; y[2] = p[2];
            y[3] = -p[3]; y[4] = p[4]; y[5] = p[5];
            if (AMP) {
                const double dnu_r = (((a.refl_k1 + p[4] * a.dvz_g) + p[5] * a.duz_g) + a.refl_k2 * (p[4] * p[4] + p[5] * p[5])) *
                                     a.refl_k3;
                const double ds0_dth = a.refl_mcr * p[6] / p[3];
                const double ds0_dph = a.refl_mcr * p[12] / p[3];
                y[6] = -p[6]; y[7] = p[7]; y[8] = p[8];
                y[9] = -p[9] + (-2.0 * dnu_r) * ds0_dth;
                y[10] = p[10]; y[11] = p[11];
                y[12] = -p[12]; y[13] = p[13]; y[14] = p[14];
                y[15] = -p[15] + (-2.0 * dnu_r) * ds0_dph;
                y[16] = p[16]; y[17] = p[17];
            }
            bnc++;
            if (bnc > a.bounces) status = 0;
        }
        if (status < 0) {
            s = 0.0; kb = 0;
            continue;
        }
        a.n_arr[ray] = na;
        a.ray_steps[ray] = steps;
        if (a.ray_status) a.ray_status[ray] = status;
        if (PATHS && a.path_rows) a.path_n[ray] = p_n;
        ray = (int)atomicAdd(a.queue, 1u);
        if (ray >= a.n_rays) break;
        start_ray(ray);
    }
}

template <bool AMP, bool SMEM, bool PATHS>
cudaError_t launch_impl(const Fan3DArgs& a, cudaStream_t stream, int* grid_used) {
    // threads per block: the caller's choice (a multiple of 32 up to kThreads) or kThreads
    const int threads = a.block > 0 ? a.block : kThreads;
    auto kern = fansph_fp64_kernel<AMP, SMEM, PATHS>;
    const size_t smem = (size_t)DimSph<AMP>::n * threads * sizeof(double) +
                        (SMEM ? (size_t)a.n_knots * kStride * sizeof(double) : 0);
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int dev = 0, n_sm = 0, per_sm = 0;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem)) != cudaSuccess) return e;
    if (per_sm < 1) per_sm = 1;
    long long want = ((long long)a.n_rays + threads - 1) / threads;
    long long grid = (long long)n_sm * per_sm;
    if (want < grid) grid = want;
    if (a.grid_cap > 0 && grid > a.grid_cap) grid = a.grid_cap;
    if (grid < 1) grid = 1;
    if (grid_used) *grid_used = (int)grid;
    kern<<<(unsigned)grid, threads, smem, stream>>>(a);
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_fansph_fp64(const Fan3DArgs& a, bool calc_amp, cudaStream_t stream, int* grid_used) {
    const size_t smem = (size_t)a.n_knots * kStride * sizeof(double);
    const bool fits = smem <= 64 * 1024;
    if (a.path_rows || a.caus_rows) {
        if (calc_amp) return fits ? launch_impl<true, true, true>(a, stream, grid_used) : launch_impl<true, false, true>(a, stream, grid_used);
        return fits ? launch_impl<false, true, true>(a, stream, grid_used) : launch_impl<false, false, true>(a, stream, grid_used);
    }
    if (calc_amp) return fits ? launch_impl<true, true, false>(a, stream, grid_used) : launch_impl<true, false, false>(a, stream, grid_used);
    return fits ? launch_impl<false, true, false>(a, stream, grid_used) : launch_impl<false, false, false>(a, stream, grid_used);
}

}  // namespace iga

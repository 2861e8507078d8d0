// FP64 ray-fan kernel: 3D Cartesian, stratified atmosphere, flat ground.
//
// One thread traces one ray at a time through all of its bounces; threads
// pull rays from a device queue (persistent grid), so a warp keeps all 32
// lanes busy while rays remain even though ray lengths differ by 10-100x.
// The loop body is one RK4 step; the rare events (ground hit, arrival record,
// reflection, new ray) are handled inside it, so lanes that hit the ground
// never wait for the rest of the warp to finish their bounce.
//
// Physics follows the reference 3D stratified equation set
// (src/geoac/geoac.eqset.3d.strat.cpp) and its RK4 driver
// (src/util/rk4solver.cpp:14-85); see the per-function notes below.  Without
// terrain the reference's d(nu_x)/ds, d(nu_y)/ds and the x/y components of
// the mu equations are identically zero (eval_src_eq, lines 353, 367, 382),
// and its flat-ground reflection leaves them unchanged, so those six values
// are per-ray constants here and only 12 of the 18 equations are integrated.
//
// The 1D spline table (altitude knots, interleaved c/u/v/rho values and
// slopes) is staged in shared memory once per CTA.
#include "fan3d.cuh"
#include "fan3d_common.cuh"

namespace iga {

namespace {

#ifndef IGA_FAN_THREADS
#define IGA_FAN_THREADS 128
#endif
#ifndef IGA_FAN_MINB
#define IGA_FAN_MINB 3
#endif
constexpr int kThreads = IGA_FAN_THREADS;


// PATHS: also write the sampled per-step rows (raypaths / terrain samples)
// and caustic points of run_prop's write_rays / write_topo / write_caustics
// output (main.infraga.3d.cpp:443-497); the fan results are unchanged.
template <bool AMP, bool SMEM, bool PATHS>
__global__ void __launch_bounds__(kThreads, IGA_FAN_MINB) fan3d_fp64_kernel(const __grid_constant__ Fan3DArgs a) {
    constexpr int N = Dim<AMP>::n;
    // dynamic shared memory: [N][kThreads] row k-1 of each lane's ray, then
    // (SMEM) the knot table
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

    int ray = (int)atomicAdd(a.queue, 1u);
    if (ray >= a.n_rays) return;

    double y[N];
    RayConst rc;
    int seg, bnc, kb, na, caustics;
    double D_prev = 0.0;
    long long steps;
    // tt/att: the ray's time and absorption sums; pt/pa: the bounce's partial
    // sums (bulk mode) or the pending last-segment increments (write_rays mode)
    double s, tt, att, pt, pa, zmax;
    long long p_base = 0, p_cap = 0, p_n = 0;   // PATHS: this ray's row range and rows produced
    // PATHS, back projection: travel-time variations (sums and pending increments as tt / pt)
    double tvt = 0.0, tvp = 0.0, ptvt = 0.0, ptvp = 0.0;
    const bool proj = PATHS && AMP && a.path_rows && a.path_mode == kPathProj;
    // PATHS, waveform trace rows: every row of every bounce, with the bounce's
    // travel time from its row 0 (ttb)
    const bool wnl = PATHS && AMP && a.path_rows && a.path_mode == kPathWnl;
    double ttb = 0.0;
    auto wnl_row = [&](const double* yr, int m) {
        if (p_n < p_cap) {
            double* o = a.path_rows + (p_base + p_n) * kWnlCols;
            o[0] = yr[0]; o[1] = yr[1]; o[2] = yr[2];
            o[3] = rc.nx; o[4] = rc.ny; o[5] = yr[3];
            o[6] = row_jacobian(tab, a, seg, yr, rc);
            o[7] = ttb; o[8] = (double)bnc; o[9] = (double)m;
        }
        p_n++;
    };

    auto start_ray = [&](int r) {
        const double theta = a.theta_deg[r] * kPi / 180.0;
        const double phi = kPi / 2.0 - a.phi_deg[r] * kPi / 180.0;
        ray_init<AMP>(a, theta, phi, y, rc);
        seg = seg_guess(fmin(fmax(y[2], a.z_lo), a.z_hi), a.z_lo, a.inv_dz, a.n_knots);
        bnc = 0; kb = 0; na = 0; steps = 0; caustics = 0;
        s = 0.0; tt = 0.0; att = 0.0; pt = 0.0; pa = 0.0;
        zmax = a.z0;
        tvt = tvp = ptvt = ptvp = 0.0;
        ttb = 0.0;
        if (PATHS && a.path_rows) { p_base = a.path_off[r]; p_cap = a.path_off[r + 1] - p_base; p_n = 0; }
    };
    start_ray(ray);

    while (true) {
        // ---- one RK4 step (rk4solver.cpp:30-55) ----
        if (wnl) wnl_row(y, kb);
        zmax = fmax(zmax, y[2]);
        double ds = a.ds_max;   // set_ds (geoac.eqset.3d.strat.cpp:214-220)
        if (y[2] < a.z_bl) ds -= (a.ds_max - a.ds_min) * exp(-(y[2] - a.z0) / 0.2);
        s += ds;
        double acc[N], stg[N], f[N];
        rhs<AMP>(tab, a, seg, y, rc, f);
        if (AMP && (a.aux || (PATHS && a.caus_rows)) && kb >= 1) {   // caustics between rows 1..k-1 of the bounce
            const double D = ray_jacobian(f, y);
            if (kb >= 2 && D * D_prev < 0.0) {
                caustics++;
                if (PATHS && a.caus_rows) {   // row kb; time through segment (kb-1, kb)
                    const unsigned long long w = atomicAdd(a.caus_count, 1ull);
                    if ((long long)w < a.caus_cap) {
                        double* o = a.caus_rows + w * kCausCols;
                        o[0] = y[0]; o[1] = y[1]; o[2] = y[2]; o[3] = tt + pt;
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
            rhs<AMP>(tab, a, seg, stg, rc, f);
            const double w = st < 2 ? c_third : c_sixth;
            const double c = st == 0 ? 0.5 : 1.0;
#pragma unroll
            for (int i = 0; i < N; i++) { const double t = ds * f[i]; acc[i] += t * w; stg[i] = y[i] + t * c; }
        }
        kb++;

        double dt, da;
        seg_increment(tab, a, seg, y, acc, rc, dt, da);
        if (wnl) ttb += dt;
        if (a.write_rays) {   // all segments but the bounce's last (main.infraga.3d.cpp:451-453)
            tt += pt; att += pa; pt = dt; pa = da;
            if (proj) {       // run_back_proj sums travel_time_var the same way (main.infraga.3d.cpp:706-708)
                double vt, vp;
                seg_time_var(tab, a, seg, y, acc, rc, vt, vp);
                tvt += ptvt; tvp += ptvp; ptvt = vt; ptvp = vp;
            }
        } else {              // per-bounce sum added at the end (main.infraga.3d.cpp:486-487)
            pt += dt; pa += da;
        }

        // ---- stop checks (rk4solver.cpp:57-75, break/ground_check :438-453) ----
        const double rx = acc[0] - a.src_x, ry = acc[1] - a.src_y;
        bool esc = (s > a.s_max) || (sqrt(rx * rx + ry * ry) > a.rng_max) ||
                   (acc[0] > a.x_max) || (acc[0] < a.x_min) || (acc[1] > a.y_max) || (acc[1] < a.y_min) ||
                   (acc[2] > a.alt_max);
        const bool gnd = !esc && (acc[2] < a.z0);
        bool capped = false, bad = false;
        if (!esc && !gnd) {
            if (kb >= a.length - 1) { capped = true; esc = true; }
            else if (!isfinite(acc[2]) || !isfinite(acc[3])) { bad = true; esc = true; }
        }
        if (!esc && !gnd) {
#pragma unroll
            for (int i = 0; i < N; i++) { prev[i * blockDim.x] = y[i]; y[i] = acc[i]; }
            if (proj && path_sampled(a.path_mode, kb)) {
                // projection row (main.infraga.3d.cpp:711-735): derivatives per degree
                // (x pi/180), the group velocity at the row
                if (p_n < p_cap) {
                    double* o = a.path_rows + (p_base + p_n) * kProjCols;
                    const double d2r = kPi / 180.0;
                    o[0] = y[0]; o[1] = y[1]; o[2] = y[2]; o[3] = tt + pt;
                    o[4] = y[4] * d2r; o[5] = y[5] * d2r; o[6] = y[6] * d2r; o[7] = (tvt + ptvt) * d2r;
                    o[8] = y[8] * d2r; o[9] = y[9] * d2r; o[10] = y[10] * d2r; o[11] = (tvp + ptvp) * d2r;
                    const double num = sqrt(rc.nx * rc.nx + rc.ny * rc.ny + y[3] * y[3]);
                    const double ze = fmin(fmax(y[2], a.z_lo), a.z_hi);
                    int sg = seg_walk(tab, a.n_knots, ze, seg);
                    const double* r0 = tab + sg * kStride;
                    const Cubic q = cubic_at(r0, ze);
                    const double c = cubic_f(r0, q, 2), sc = bl_scale(a, y[2]);
                    o[12] = c * rc.nx / num + cubic_f(r0, q, 4) * sc;
                    o[13] = c * rc.ny / num + cubic_f(r0, q, 6) * sc;
                    o[14] = c * y[3] / num;
                }
                p_n++;
            } else if (PATHS && a.path_rows && path_sampled(a.path_mode, kb)) {
                // row m = kb of the bounce, above the ground: z = max(z, z_g) = z
                if (p_n < p_cap) {
                    double* o = a.path_rows + (p_base + p_n) * kPathCols;
                    o[0] = y[0]; o[1] = y[1];
                    o[2] = a.path_mode == kPathRays ? y[2] : a.z0;
                    int sg = seg;
                    o[3] = (AMP && a.path_mode == kPathRays)
                               ? amp_db(tab, a, sg, y, rc, a.theta_deg[ray] * kPi / 180.0,
                                        kPi / 2.0 - a.phi_deg[ray] * kPi / 180.0, nullptr)
                               : 0.0;
                    o[4] = -2.0 * (att + pa); o[5] = tt + pt; o[6] = (double)bnc;
                }
                p_n++;
            }
            continue;
        }

        // ---- end of a bounce segment (main.infraga.3d.cpp:436-538) ----
        const int K = capped ? a.length : kb;
        steps += K;
        if (wnl) wnl_row(acc, kb);   // row k: the first row beyond the segment's end
        if (PATHS && a.path_rows && a.path_mode == kPathResid) {
            // print_resid (main.infraga.3d.cpp:437-441): residuals at row k - 1
            if (p_n < p_cap) {
                double* o = a.path_rows + (p_base + p_n) * kPathCols;
                eikonal_resid<AMP>(tab, a, seg, y, rc, o[0], o[1]);
                o[2] = (double)bnc; o[3] = 0.0; o[4] = 0.0; o[5] = 0.0; o[6] = 0.0;
            }
            p_n++;
        }
        if (!a.write_rays) { tt += pt; att += pa; }
        pt = 0.0; pa = 0.0;
        ptvt = 0.0; ptvp = 0.0;
        ttb = 0.0;
        int status = -1;
        if (zmax < a.z0 + a.turn_ht_min) status = 2;
        else if (esc) status = bad ? 4 : (capped ? 5 : 1);
        else if (K < 2) status = 3;
        if (status < 0) {
            // arrival record from the first below-ground row
            double* out = a.arrivals + ((size_t)ray * nb + na) * 12;
            const double incl = -asin(a.c_ratio * acc[3]) * 180.0 / kPi;
            double baz = 90.0 - atan2(-rc.ny, -rc.nx) * 180.0 / kPi;
            if (baz < -180.0) baz += 360.0;
            else if (baz > 180.0) baz -= 360.0;
            const double ex = acc[0] - a.src_x, ey = acc[1] - a.src_y;
            const double th_deg = a.theta_deg[ray], ph_deg = a.phi_deg[ray];
            out[0] = th_deg;
            out[1] = ph_deg;
            out[2] = (double)bnc;
            out[3] = acc[0];
            out[4] = acc[1];
            out[5] = tt;
            out[6] = sqrt(ex * ex + ey * ey) / tt;
            out[7] = zmax;
            out[8] = incl;
            out[9] = baz;
            double jac = 0.0;
            out[10] = AMP ? amp_db(tab, a, seg, acc, rc, th_deg * kPi / 180.0, kPi / 2.0 - ph_deg * kPi / 180.0, &jac) : 0.0;
            out[11] = -2.0 * att;
            if (a.aux) {
                double* ax = a.aux + ((size_t)ray * nb + na) * 4;
                if (AMP) write_aux(ax, a, acc, rc, jac, caustics);
                else ax[0] = ax[1] = ax[2] = ax[3] = 0.0;
            }
            na++;
            // reflection from rows k-2 (prev) and k-1 (y): geoac::approx_intercept
            // and geoac::set_refl (geoac.eqset.3d.strat.cpp:110-209), flat ground
            const double dz_grnd = a.z0 - y[2];
            const double dz_k = y[2] - prev[2 * blockDim.x];
            double p[N];
#pragma unroll
            for (int i = 0; i < N; i++) p[i] = y[i] + (y[i] - prev[i * blockDim.x]) / dz_k * dz_grnd;
            y[0] = p[0]; y[1] = p[1]; y[2] = a.z0; y[3] = -p[3];
            if (AMP) {
                y[4] = p[4]; y[5] = p[5]; y[6] = -p[6];
                y[8] = p[8]; y[9] = p[9]; y[10] = -p[10];
                const double ds0_dth = -a.c0 / a.c_gnd * p[6] / p[3];
                const double ds0_dph = -a.c0 / a.c_gnd * p[10] / p[3];
                const double dnuz_ds = -1.0 / a.c_gnd * (a.c0 / a.c_gnd * a.dcz_g + rc.nx * a.duz_g + rc.ny * a.dvz_g);
                y[7] = -p[7] + (-2.0 * dnuz_ds) * ds0_dth;
                y[11] = -p[11] + (-2.0 * dnuz_ds) * ds0_dph;
            }
            bnc++;
            if (bnc > a.bounces) status = 0;
        }
        if (status < 0) {
            s = 0.0; kb = 0;
            continue;
        }
        // ray finished: record and take the next one from the queue
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
    auto kern = fan3d_fp64_kernel<AMP, SMEM, PATHS>;
    const size_t smem = (size_t)Dim<AMP>::n * threads * sizeof(double) +
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

cudaError_t launch_fan3d_fp64(const Fan3DArgs& a, bool calc_amp, cudaStream_t stream, int* grid_used) {
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

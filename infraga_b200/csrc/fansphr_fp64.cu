// FP64 ray-fan kernel: spherical (global) geometry, range-dependent
// atmosphere (hybrid 3D splines), flat ground or terrain.
//
// Execution scheme as in the other fan kernels (one thread per ray,
// persistent grid on a device ray queue, one RK4 step per loop iteration,
// ground hits / arrivals / reflections in the loop, row k-1 in shared
// memory).  The atmosphere tables (atmo_rngdep.h) are read through the
// read-only cache: a ray reads the 4 corner records of its cell (2 x 512 B
// each, two z knots) per evaluation and stays in the same cell for many
// steps, so the working set is L1/L2-resident; the node coordinate arrays
// are staged in shared memory.
//
// Physics: the reference's spherical range-dependent equation set
// (src/geoac/geoac.eqset.sph.rngdep.cpp) with atmo_state.sph.rngdep.cpp
// (no boundary-layer vertical wind: topo_use_BLw=false, the default), its RK4
// driver (src/util/rk4solver.cpp:14-85) and run_prop
// (src/main.infraga.sph.rngdep.cpp:412-545).
//
// ST instantiations run infraga-sph's stratified profile over terrain
// (topo_file=): c, u, v, rho from the 1D knot table at the clamped altitude
// (atmo_state.sph.strat.cpp:166-245, calc_uvw :498-800) with the same terrain,
// boundary-layer scaling, equations (geoac.eqset.sph.strat.cpp differs from
// the range-dependent set only in where the atmosphere comes from) and bounce
// loop; run_prop of infraga-sph records the arrival inclination as -asin(...)
// (main.infraga.sph.cpp:523) where the range-dependent one has +asin.
#include "eig3d.cuh"
#include "fan3d.cuh"
#include "fansph_common.cuh"
#include "rngdep_eval.cuh"
#include "fansphr_common.cuh"

namespace iga {

namespace {

#ifndef IGA_SPHR_THREADS
#define IGA_SPHR_THREADS 128
#endif
#ifndef IGA_SPHR_MINB
#define IGA_SPHR_MINB 1
#endif
constexpr int kThreads = IGA_SPHR_THREADS;

// PATHS: also write the sampled per-step rows and caustic points of
// run_prop's write_rays / write_topo / write_caustics output
// (main.infraga.sph.rngdep.cpp:450-503); the fan results are unchanged.
template <bool AMP, bool PATHS, bool ST>
__global__ void __launch_bounds__(kThreads, IGA_SPHR_MINB) fansphr_fp64_kernel(const __grid_constant__ Fan3DArgs a) {
    constexpr int N = DimSph<AMP>::n;
    extern __shared__ double s_mem[];
    double* s_prev = s_mem;
    // node coordinates in shared memory
    double* s_hz = s_mem + N * blockDim.x;
    double* s_hx = s_hz + a.hyb_nz;
    double* s_hy = s_hx + a.hyb_nx;
    double* s_tx = s_hy + a.hyb_ny;
    double* s_ty = s_tx + a.topo_nx;
    for (int i = threadIdx.x; i < a.hyb_nz; i += blockDim.x) s_hz[i] = a.hyb_z[i];
    for (int i = threadIdx.x; i < a.hyb_nx; i += blockDim.x) s_hx[i] = a.hyb_x[i];
    for (int i = threadIdx.x; i < a.hyb_ny; i += blockDim.x) s_hy[i] = a.hyb_y[i];
    for (int i = threadIdx.x; i < a.topo_nx; i += blockDim.x) s_tx[i] = a.topo_x[i];
    for (int i = threadIdx.x; i < a.topo_ny; i += blockDim.x) s_ty[i] = a.topo_y[i];
    __syncthreads();
    Views vw;
    vw.hyb = HybView{a.hyb_tab, s_hx, s_hy, s_hz, a.hyb_nx, a.hyb_ny, a.hyb_nz};
    vw.topo = TopoView{a.topo_tab, s_tx, s_ty, a.topo_nx, a.topo_ny};
    vw.has_topo = a.topo_tab != nullptr;
    double* prev = s_prev + threadIdx.x;   // element i at prev[i * blockDim.x]

    const int nb = a.bounces + 1;
    const double c_third = 1.0 / 3.0, c_sixth = 1.0 / 6.0;

    int ray = (int)atomicAdd(a.queue, 1u);
    if (ray >= a.n_rays) return;

    double y[N];
    Cells cl{0, 0, 0, 0, 0};
    int bnc, kb, na, caustics;
    double D_prev = 0.0;
    long long steps;
    double s, tt, att, pt, pa, rmax;
    long long p_base = 0, p_cap = 0, p_n = 0;   // PATHS: this ray's row range and rows produced
    const double rad2deg = 180.0 / kPi;

    auto start_ray = [&](int r) {
        const double theta = a.theta_deg[r] * (kPi / 180.0);
        const double phi = kPi / 2.0 - a.phi_deg[r] * (kPi / 180.0);
        ray_init_sph<AMP>(a, theta, phi, y);
        bnc = 0; kb = 0; na = 0; steps = 0; caustics = 0;
        s = 0.0; tt = 0.0; att = 0.0; pt = 0.0; pa = 0.0;
        rmax = 0.0;
        if (PATHS && a.path_rows) { p_base = a.path_off[r]; p_cap = a.path_off[r + 1] - p_base; p_n = 0; }
    };
    start_ray(ray);

    while (true) {
        rmax = fmax(rmax, y[0] - a.r_earth);
        double ds = a.ds_max;   // set_ds (geoac.eqset.sph.rngdep.cpp:227-233)
        if (y[0] - a.r_earth < a.z_bl)
            ds -= (a.ds_max - a.ds_min) * exp(-(y[0] - topo_r(a, vw, cl, y[1], y[2])) / 0.2);
        s += ds;
        double acc[N], stg[N], f[N];
        rhs_sphr<AMP, ST>(a, vw, cl, y, f);
        if (AMP && (a.aux || (PATHS && a.caus_rows)) && kb >= 1) {
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
            rhs_sphr<AMP, ST>(a, vw, cl, stg, f);
            const double w = st < 2 ? c_third : c_sixth;
            const double c = st == 0 ? 0.5 : 1.0;
#pragma unroll
            for (int i = 0; i < N; i++) { const double t = ds * f[i]; acc[i] += t * w; stg[i] = y[i] + t * c; }
        }
        kb++;

        bool esc = s > a.s_max;
        if (!esc) {
            if (acc[2] > kPi) acc[2] -= 2.0 * kPi;
            else if (acc[2] < -kPi) acc[2] += 2.0 * kPi;
            esc = (acc[1] < -kPi / 2.0 || acc[1] > kPi / 2.0) || (acc[0] - a.r_earth > a.alt_max) ||
                  beyond_range(a, acc[1], acc[2]) || (acc[1] < a.lat_min || acc[1] > a.lat_max) ||
                  (acc[2] < a.lon_min || acc[2] > a.lon_max);
        }
        // ground_check (geoac.eqset.sph.rngdep.cpp:496-503)
        const bool gnd = !esc && (acc[0] - a.r_earth <= a.topo_zmax) && (acc[0] < topo_r(a, vw, cl, acc[1], acc[2]));

        double dt, da;
        seg_increment_sphr<ST>(a, vw, cl, y, acc, dt, da);
        if (a.write_rays) { tt += pt; att += pa; pt = dt; pa = da; }
        else { pt += dt; pa += da; }

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
                    Cells c2 = cl;
                    o[0] = y[1] * rad2deg; o[1] = y[2] * rad2deg;
                    o[2] = a.path_mode == kPathRays ? y[0] - a.r_earth : topo_r(a, vw, c2, y[1], y[2]) - a.r_earth;
                    o[3] = (AMP && a.path_mode == kPathRays)
                               ? amp_db_sphr<ST>(a, vw, c2, y, a.theta_deg[ray] * (kPi / 180.0),
                                             kPi / 2.0 - a.phi_deg[ray] * (kPi / 180.0), nullptr)
                               : 0.0;
                    o[4] = -2.0 * (att + pa); o[5] = tt + pt; o[6] = (double)bnc;
                }
                p_n++;
            }
            continue;
        }

        // ---- end of a bounce segment (main.infraga.sph.rngdep.cpp:499-541) ----
        const int K = capped ? a.length : kb;
        steps += K;
        if (!a.write_rays) { tt += pt; att += pa; }
        pt = 0.0; pa = 0.0;
        int status = -1;
        if (a.topo_tab == nullptr && rmax < a.z0 + a.turn_ht_min) status = 2;
        else if (esc) status = bad ? 4 : (capped ? 5 : 1);
        else if (K < 2) status = 3;
        else if (tt / 3600.0 > a.time_max_h) status = 6;
        if (status < 0) {
            double* out = a.arrivals + ((size_t)ray * nb + na) * 12;
            const double th_deg = a.theta_deg[ray], ph_deg = a.phi_deg[ray];
            AtmPt mk;
            atm_point<ST>(a, vw, cl, acc[0], acc[1], acc[2], mk);
            // the range-dependent run_prop records +asin(...) (main.infraga.sph.rngdep.cpp:514),
            // infraga-sph -asin(...) (main.infraga.sph.cpp:523)
            const double incl = (ST ? -1.0 : 1.0) * asin(mk.c / a.c0 * acc[3]) * 180.0 / kPi;
            double baz = 90.0 - atan2(-acc[4], -acc[5]) * 180.0 / kPi;
            if (baz < -180.0) baz += 360.0;
            else if (baz > 180.0) baz -= 360.0;
            out[0] = th_deg;
            out[1] = ph_deg;
            out[2] = (double)bnc;
            out[3] = acc[1] * (180.0 / kPi);
            out[4] = acc[2] * (180.0 / kPi);
            out[5] = tt;
            out[6] = gc_dist(a.r_earth, acc[1], acc[2], a.src_x, a.src_y, a.cos_lat_src) / tt;
            out[7] = rmax;
            out[8] = incl;
            out[9] = baz;
            double jac = 0.0;
            out[10] = AMP ? amp_db_sphr<ST>(a, vw, cl, acc, th_deg * (kPi / 180.0), kPi / 2.0 - ph_deg * (kPi / 180.0), &jac) : 0.0;
            out[11] = -2.0 * att;
            if (a.aux) {
                double* ax = a.aux + ((size_t)ray * nb + na) * 4;
                if (AMP) write_aux_sph(ax, a, acc, jac, caustics);
                else ax[0] = ax[1] = ax[2] = ax[3] = 0.0;
            }
            na++;
            reflect_sphr<N, AMP, ST>(a, vw, cl, y, prev, blockDim.x);
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

template <bool AMP, bool PATHS, bool ST>
cudaError_t launch_impl(const Fan3DArgs& a, cudaStream_t stream, int* grid_used) {
    // threads per block: the caller's choice (a multiple of 32 up to kThreads) or kThreads
    const int threads = a.block > 0 ? a.block : kThreads;
    auto kern = fansphr_fp64_kernel<AMP, PATHS, ST>;
    const size_t smem = ((size_t)DimSph<AMP>::n * threads + a.hyb_nz + a.hyb_nx + a.hyb_ny + a.topo_nx + a.topo_ny) *
                        sizeof(double);
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

// One eigenray-search trace per thread (find_eigenray / est_eigenray on this
// solver, geoac.eigenray.sph.cpp:42-380): n_seg prop_rk4 segments from the
// launch source with terrain reflections between them.  Record mode sums
// time and absorption per step and the turning height over rows 1..k-1 from
// 0 (:230-268) and forms the arrival columns (:283-296), with the arrival
// inclination's c taken at a radius equal to the source ALTITUDE (clamped to
// the lowest knot under the source, :284); an amplitude trace also returns
// what the Newton derivatives read under the last row (:335-345): c at the
// source and on the ground, the ground radius and the terrain gradient.
// Same block size as the fan kernel (reflect_sphr reads row k-2 from shared
// memory with that stride).
template <bool AMP, bool ST>
__global__ void __launch_bounds__(kThreads, IGA_SPHR_MINB) tracesphr_fp64_kernel(const __grid_constant__ Fan3DArgs a,
                                                                              const TraceReq* __restrict__ reqs,
                                                                              TraceRes18* __restrict__ out, int n, unsigned int* __restrict__ queue,
                                                                              SegRes* __restrict__ seg_out,
                                                                              int seg_stride) {
    constexpr int N = DimSph<AMP>::n;
    extern __shared__ double s_mem[];
    double* s_prev = s_mem;
    double* s_hz = s_mem + N * blockDim.x;
    double* s_hx = s_hz + a.hyb_nz;
    double* s_hy = s_hx + a.hyb_nx;
    double* s_tx = s_hy + a.hyb_ny;
    double* s_ty = s_tx + a.topo_nx;
    for (int i = threadIdx.x; i < a.hyb_nz; i += blockDim.x) s_hz[i] = a.hyb_z[i];
    for (int i = threadIdx.x; i < a.hyb_nx; i += blockDim.x) s_hx[i] = a.hyb_x[i];
    for (int i = threadIdx.x; i < a.hyb_ny; i += blockDim.x) s_hy[i] = a.hyb_y[i];
    for (int i = threadIdx.x; i < a.topo_nx; i += blockDim.x) s_tx[i] = a.topo_x[i];
    for (int i = threadIdx.x; i < a.topo_ny; i += blockDim.x) s_ty[i] = a.topo_y[i];
    __syncthreads();
    // persistent: each thread takes the next request when its trace ends, so
    // lanes whose trace finished early do not idle until the warp's longest one
    for (int r = (int)atomicAdd(queue, 1u); r < n; r = (int)atomicAdd(queue, 1u)) {
        Views vw;
        vw.hyb = HybView{a.hyb_tab, s_hx, s_hy, s_hz, a.hyb_nx, a.hyb_ny, a.hyb_nz};
        vw.topo = TopoView{a.topo_tab, s_tx, s_ty, a.topo_nx, a.topo_ny};
        vw.has_topo = a.topo_tab != nullptr;
        double* prev = s_prev + threadIdx.x;
        const TraceReq q = reqs[r];
        const bool record = (q.flags & kRecord) != 0, stop = (q.flags & kStopOnEscape) != 0;
        const double c_third = 1.0 / 3.0, c_sixth = 1.0 / 6.0;

        double y[N];
        Cells cl{0, 0, 0, 0, 0};
        ray_init_sph<AMP>(a, q.theta, q.phi, y);
        double tt = 0.0, att = 0.0, rmax = 0.0;
        long long steps = 0;
        double acc[N];
        bool esc = false;
        for (int sg = 0; sg < q.n_seg; sg++) {
            double s = 0.0, pt = 0.0, pa = 0.0;
            int kb = 0;
            bool capped = false;
#pragma unroll
            for (int i = 0; i < N; i++) prev[i * blockDim.x] = y[i];
            while (true) {
                if (record && kb >= 1) rmax = fmax(rmax, y[0] - a.r_earth);
                double ds = a.ds_max;
                if (y[0] - a.r_earth < a.z_bl)
                    ds -= (a.ds_max - a.ds_min) * exp(-(y[0] - topo_r(a, vw, cl, y[1], y[2])) / 0.2);
                s += ds;
                double stg[N], f[N];
                rhs_sphr<AMP, ST>(a, vw, cl, y, f);
#pragma unroll
                for (int i = 0; i < N; i++) { const double t = ds * f[i]; acc[i] = y[i] + t * c_sixth; stg[i] = y[i] + t * 0.5; }
                // stages 2..4 with one copy of the right-hand side (instruction-cache footprint)
#pragma unroll 1
                for (int st = 0; st < 3; st++) {
                    rhs_sphr<AMP, ST>(a, vw, cl, stg, f);
                    const double w = st < 2 ? c_third : c_sixth;
                    const double c = st == 0 ? 0.5 : 1.0;
#pragma unroll
                    for (int i = 0; i < N; i++) { const double t = ds * f[i]; acc[i] += t * w; stg[i] = y[i] + t * c; }
                }
                kb++;
                esc = s > a.s_max;
                if (!esc) {
                    if (acc[2] > kPi) acc[2] -= 2.0 * kPi;
                    else if (acc[2] < -kPi) acc[2] += 2.0 * kPi;
                    esc = (acc[1] < -kPi / 2.0 || acc[1] > kPi / 2.0) || (acc[0] - a.r_earth > a.alt_max) ||
                          beyond_range(a, acc[1], acc[2]) || (acc[1] < a.lat_min || acc[1] > a.lat_max) ||
                          (acc[2] < a.lon_min || acc[2] > a.lon_max);
                }
                const bool gnd = !esc && (acc[0] - a.r_earth <= a.topo_zmax) && (acc[0] < topo_r(a, vw, cl, acc[1], acc[2]));
                if (record) {
                    double dt, da;
                    seg_increment_sphr<ST>(a, vw, cl, y, acc, dt, da);
                    tt += pt; att += pa; pt = dt; pa = da;
                }
                if (!esc && !gnd) {
                    if (kb >= a.length - 1) { capped = true; esc = true; }
                    else if (!isfinite(acc[0]) || !isfinite(acc[1]) || !isfinite(acc[3])) esc = true;
                }
                if (!esc && !gnd) {
#pragma unroll
                    for (int i = 0; i < N; i++) { prev[i * blockDim.x] = y[i]; y[i] = acc[i]; }
                    continue;
                }
                break;
            }
            steps += capped ? a.length : kb;
            if (seg_out) {
                SegRes& g = seg_out[(size_t)r * seg_stride + sg];
                g.x = acc[1]; g.y = acc[2]; g.steps = steps; g.escaped = esc ? 1 : 0;
            }
            if (sg == q.n_seg - 1 || (esc && stop)) break;
            reflect_sphr<N, AMP, ST>(a, vw, cl, y, prev, blockDim.x);
        }
        TraceRes18& o = out[r];
#pragma unroll
        for (int i = 0; i < 18; i++) o.y[i] = i < N ? acc[i] : 0.0;
        o.steps = steps;
        o.escaped = esc ? 1 : 0;
        o.tt = o.att = o.zmax = o.amp_db = o.incl = o.baz = 0.0;
        o.c_src = a.c0; o.c_grnd = 0.0; o.z_grnd = 0.0; o.dzg[0] = 0.0; o.dzg[1] = 0.0;
        if (AMP && !record) {   // topo::z (a radius), topo::dz and atmo::c on the ground under the last row
            double rg = a.r_grnd;
            if (vw.has_topo) {
                TopoVal t;
                topo_eval(vw.topo, acc[1], acc[2], 1, t, cl.tx, cl.ty);
                rg = a.r_earth + t.z; o.dzg[0] = t.d[0]; o.dzg[1] = t.d[1];
            }
            o.z_grnd = rg;
            o.c_grnd = c_at<ST>(a, vw, cl, rg, acc[1], acc[2]);
        }
        if (record) {
            o.tt = tt; o.att = att; o.zmax = rmax;
            o.amp_db = AMP ? amp_db_sphr<ST>(a, vw, cl, acc, q.theta, q.phi, nullptr) : 0.0;
            const double c_k = c_at<ST>(a, vw, cl, acc[0], acc[1], acc[2]);
            const double c_s = c_at<ST>(a, vw, cl, a.src_z, a.src_x, a.src_y);   // r = the source altitude
            o.incl = -asin(c_k / c_s * acc[3]) * 180.0 / kPi;
            double baz = 90.0 - atan2(-acc[4], -acc[5]) * (180.0 / kPi);
            while (baz < -180.0) baz += 360.0;
            while (baz > 180.0) baz -= 360.0;
            o.baz = baz;
        }
    }
}

template <bool AMP, bool ST>
cudaError_t launch_trace_impl(const Fan3DArgs& a, const TraceReq* d_req, TraceRes18* d_res, int n, cudaStream_t st,
                              SegRes* seg_out, int seg_stride, unsigned int* d_queue) {
    if (n <= 0) return cudaSuccess;
    auto kern = tracesphr_fp64_kernel<AMP, ST>;
    const size_t smem = ((size_t)DimSph<AMP>::n * kThreads + a.hyb_nz + a.hyb_nx + a.hyb_ny + a.topo_nx + a.topo_ny) *
                        sizeof(double);
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int grid = 0;
    if ((e = trace_grid(kern, kThreads, smem, n, grid)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(d_queue, 0, sizeof(unsigned int), st)) != cudaSuccess) return e;
    kern<<<grid, kThreads, smem, st>>>(a, d_req, d_res, n, d_queue, seg_out, seg_stride);
    return cudaGetLastError();
}

// a.knots set (no hybrid tables): stratified profile over terrain
template <bool ST>
cudaError_t launch_fan(const Fan3DArgs& a, bool calc_amp, cudaStream_t stream, int* grid_used) {
    if (a.path_rows || a.caus_rows)
        return calc_amp ? launch_impl<true, true, ST>(a, stream, grid_used) : launch_impl<false, true, ST>(a, stream, grid_used);
    return calc_amp ? launch_impl<true, false, ST>(a, stream, grid_used) : launch_impl<false, false, ST>(a, stream, grid_used);
}

}  // namespace

cudaError_t launch_fansphr_fp64(const Fan3DArgs& a, bool calc_amp, cudaStream_t stream, int* grid_used) {
    return a.knots ? launch_fan<true>(a, calc_amp, stream, grid_used) : launch_fan<false>(a, calc_amp, stream, grid_used);
}

cudaError_t launch_trace_sphr(const Fan3DArgs& a, const TraceReq* d_req, TraceRes18* d_res, int n, bool amp,
                              cudaStream_t st, SegRes* seg_out, int seg_stride, unsigned int* d_queue) {
    if (a.knots)
        return amp ? launch_trace_impl<true, true>(a, d_req, d_res, n, st, seg_out, seg_stride, d_queue)
                   : launch_trace_impl<false, true>(a, d_req, d_res, n, st, seg_out, seg_stride, d_queue);
    return amp ? launch_trace_impl<true, false>(a, d_req, d_res, n, st, seg_out, seg_stride, d_queue)
               : launch_trace_impl<false, false>(a, d_req, d_res, n, st, seg_out, seg_stride, d_queue);
}

}  // namespace iga
